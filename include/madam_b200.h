/* Extensions of the B200 destriping library (libmadam_b200/libmadam.so).
 *
 * The reference has no status codes (errors call abort_mpi,
 * src/mpi_wrappers.f90:120-137) and returns its products only as FITS files
 * (src/output.f90).  These entry points return a status (0 = success) and
 * give the products of the last call as arrays.
 */
#ifndef MADAM_B200_H
#define MADAM_B200_H

#include "madam.h"

#ifdef __cplusplus
extern "C" {
#endif

/* destripe() with a status (reference src/smadam.F90:64-590). */
int madam_b200_destripe(int comm, char *parstring, long ndet, char *detstring,
                        double *detweights, long nsamp, long nnz, void *timestamps, void *pix,
                        void *pixweights, void *signal, long nperiod, long *periods, long *npsd,
                        long npsdtot, double *psdstarts, long npsdbin, double *psdfreqs,
                        long npsdval, double *psdvals);

/* FP32-TOD precision form of destripe() (reference src/smadam.F90:64-590,
 * which takes float64 signals only): the same arguments with `signal` as
 * float32 [ndet][nsamp] (host or device memory, like pix).  The PCG
 * projections read float32 pointing (consecutive samples of one baseline in
 * one pixel summed into pairs) and a float32 copy of the map; pixel
 * matrices, binning, baselines and all PCG inner products stay float64.
 * Maps and baselines agree with destripe() on the same samples to about
 * 1e-6 relative (tested at 1e-4).  A cleaned TOD (write_tod) goes back into
 * `signal` as float32.  No reference counterpart. */
int madam_b200_destripe_fp32(int comm, char *parstring, long ndet, char *detstring,
                             double *detweights, long nsamp, long nnz, void *timestamps, void *pix,
                             void *pixweights, float *signal, long nperiod, long *periods,
                             long *npsd, long npsdtot, double *psdstarts, long npsdbin,
                             double *psdfreqs, long npsdval, double *psdvals);

/* destripe_with_cache() with a status (reference src/smadam.F90:593-918). */
int madam_b200_destripe_with_cache(int comm, long ndet, long nsamp, long nnz, void *timestamps,
                                   void *pix, void *pixweights, void *signal, char *outpath);

/* clear_caches() with a status (reference src/smadam.F90:921-951).  Also
 * returns the device memory the solve kept in the device's memory pool. */
int madam_b200_clear_caches(void);

/* Batched Monte Carlo: nrhs realisations of destripe_with_cache (reference
 * src/smadam.F90:593-918, which takes one realisation per call) that share
 * one pointing.  signals: float64 [nrhs][ndet][nsamp], host or device memory
 * like pix.  Every realisation is solved as destripe_with_cache would solve
 * it right after the caching destripe(..., mcmode=T) call; the cache is left
 * unchanged.  Results: "map_batch", "binmap_batch" (float64
 * [nrhs][npix][nmap]), "aa_batch" (float64 [nrhs][ndet][noba]),
 * "noiter_batch", "rrinit_batch", "rr_final_batch" (float64 [nrhs]).  No
 * files are written.  No reference counterpart as one call. */
int madam_b200_destripe_with_cache_batch(int comm, long ndet, long nsamp, long nnz,
                                         void *timestamps, void *pix, void *pixweights,
                                         long nrhs, void *signals);

/* The batched Monte Carlo solve in the FP32-TOD precision form: signals are
 * float32 [nrhs][ndet][nsamp] (host or device memory, like pix); the
 * projections read float32 copies of p.detw and of the map (and the
 * scatter's pointing as pairs), while pixel matrices, baselines and all
 * inner products stay float64.  Results as for
 * madam_b200_destripe_with_cache_batch; they agree with the float64 solve of
 * the same samples to about 1e-6 relative (tested at 1e-4).  No reference
 * counterpart. */
int madam_b200_destripe_with_cache_batch_fp32(int comm, long ndet, long nsamp, long nnz,
                                              void *timestamps, void *pix, void *pixweights,
                                              long nrhs, float *signals);

/* Serving: a job queue over one GPU.  No reference counterpart (the
 * reference runs one destripe per call and per MPI job).
 *
 * serve_open starts nworkers worker threads, each with its own engine and
 * CUDA stream, and a device-memory budget of mem_fraction of the free memory;
 * NULL on error (message in err).  serve_submit queues one destripe() job
 * with the reference's destripe arguments (src/smadam.F90:64-101; mcmode is
 * refused) and returns its id, or -1 (message in err).  The caller's buffers
 * must stay valid until the job is done.  Jobs start first come, first
 * served, when their estimated footprint fits the budget beside the running
 * jobs, and overlap on the device (the library's memory pool is trimmed to
 * the budget after each job, and a job that runs out of device memory is
 * requeued once); their products do not depend on what else
 * runs (beyond rounding).  A job's setup runs on its worker; its PCG then
 * iterates in shared rounds with the other jobs past their setup, driven by
 * one stepper thread: per round each job's A p and preconditioner, the CG
 * vector algebra and inner products of all jobs in shared launches, and one
 * host synchronisation for every job's convergence test (a job with a
 * covariance-matrix output, or kfirst off, runs on its worker alone).
 * serve_wait waits up to timeout_s seconds (< 0: no limit) and
 * returns the job state: 0 queued, 1 running, 2 done, 3 failed, -1 unknown.
 * serve_result_size / serve_result_copy give a done job's "map", "binmap"
 * (float64 [npix][nmap]), "hits", "mask" (int32 [npix]), "aa" (float64
 * [ndet][noba]), "scalars" (float64 [24]), "rr_history" (float64);
 * serve_job_info gives out[0..5] = submit, start and end time (s), samples,
 * PCG iterations, admitted bytes, and with nout >= 9 out[6..8] = the job's
 * setup, PCG and finalisation wall times (ms; the PCG's includes the shared
 * rounds it waited in); serve_error the message of a failed job;
 * serve_release frees a finished job; serve_stats gives out[0..2] = PCG
 * rounds run, job-rounds (jobs summed over the rounds) and the most jobs in
 * one round; serve_close waits for the running jobs, drops the queued ones
 * and frees the server. */
void *madam_b200_serve_open(int nworkers, double mem_fraction, char *err, long errlen);
long madam_b200_serve_submit(void *srv, char *parstring, long ndet, char *detstring,
                             double *detweights, long nsamp, long nnz, void *timestamps, void *pix,
                             void *pixweights, void *signal, long nperiod, long *periods,
                             long *npsd, long npsdtot, double *psdstarts, long npsdbin,
                             double *psdfreqs, long npsdval, double *psdvals, char *err,
                             long errlen);
/* serve_submit for a float32 signal: the job runs in the FP32-TOD form of
 * madam_b200_destripe_fp32. */
long madam_b200_serve_submit_fp32(void *srv, char *parstring, long ndet, char *detstring,
                                  double *detweights, long nsamp, long nnz, void *timestamps,
                                  void *pix, void *pixweights, float *signal, long nperiod,
                                  long *periods, long *npsd, long npsdtot, double *psdstarts,
                                  long npsdbin, double *psdfreqs, long npsdval, double *psdvals,
                                  char *err, long errlen);
int madam_b200_serve_wait(void *srv, long job, double timeout_s);
long madam_b200_serve_result_size(void *srv, long job, const char *name);
int madam_b200_serve_result_copy(void *srv, long job, const char *name, void *dst, long nbytes);
int madam_b200_serve_job_info(void *srv, long job, double *out, long nout);
int madam_b200_serve_error(void *srv, long job, char *buf, long buflen);
int madam_b200_serve_release(void *srv, long job);
int madam_b200_serve_stats(void *srv, double *out, long nout);
int madam_b200_serve_close(void *srv);

/* Sharded runs: communicators standing in for the reference's MPI
 * communicator (mpi_wrappers.f90).  Each rank (one process per GPU) passes
 * its own TOD (detectors and/or time spans) to destripe / destripe_with_cache
 * with `comm` = the handle returned here; the pixel matrices, hits, maps and
 * the PCG inner products are summed across the ranks (the reference's
 * collect_map / collect_cc / collect_hits / sum_mpi), so every rank ends with
 * the whole maps and its own baselines; rank 0 writes the FITS files.
 * Leakage matrices need every rank to hold the same detectors, as in the
 * reference.  comm_nccl_id fills 128 bytes of NCCL unique id (rank 0, to be
 * sent to the other ranks); comm_init_nccl makes an NCCL communicator (NVLink
 * / NVSwitch, libnccl.so.2 loaded on first use); comm_init_host one whose
 * reductions call fn(host buffer, n, op) (op 0 sum, 1 max), e.g. over a CPU
 * process group.  Both return a handle > 0, or -1 (message from
 * comm_error); comm 0 or an unknown handle means a single rank.  The batched
 * solve and the job server run on one rank.  No reference counterpart beyond
 * the MPI communicator. */
int madam_b200_comm_nccl_id(char *id);
int madam_b200_comm_init_nccl(int rank, int nranks, const char *id);
typedef void (*madam_b200_allreduce_fn)(double *buf, long n, int op);
int madam_b200_comm_init_host(int rank, int nranks, madam_b200_allreduce_fn fn);
int madam_b200_comm_free(int handle);
int madam_b200_comm_error(char *buf, long buflen);

/* Status of the last call (0 = success) and its error message; replaces the
 * reference's abort_mpi messages (src/mpi_wrappers.f90:120-137). */
int madam_b200_last_error(char *buf, long buflen);

/* Products of the last call, in place of the FITS writers of
 * src/output.f90:114-1180.  Names: "map", "binmap" (float64 [npix][nmap],
 * full sky, NESTED, nside_map), "hits", "mask" (int32 [npix]), "crit"
 * (float32 [npix]), "cc", "cca" (float64 [npix][nmap][nmap], inverse pixel
 * matrices at nside_map / nside_cross), "aa", "yba", "nna" (float64
 * [ndet][noba]: baselines, RHS, F^T N^-1 F), "fcov" (float64
 * [npsdtot][nof/2+1]), "invcov" (float64 [npsdtot][nof]), "rr_history"
 * (float64 [niter]), "band_widths" (int64), "scalars" (float64 [24]),
 * "leakmatrix:<d>" (float64 [npix][nmap][nmap], row i column j: the leakage
 * matrix of detector d, write_leakmatrix), the subsets of bin_subsets
 * (smadam.F90:954-1257) as "subsets" (float64 [nsub][4]: pass, survey, detector
 * set, nmap) with "subset_binmap:<k>", "subset_hits:<k>", "subset_mask:<k>"
 * (int32), "subset_cc:<k>", "subset_leak:<k>:<d>",
 * "timings" (float64 [9], milliseconds), "nan_checks" (float64 [7], with
 * checknan: detectors with NaN parameters, NaN counts of yba, the binned
 * cross map, the pointing weights, and r, z, p at the first CG step; the
 * reference prints these checks, smadam_routines.f90:456-502, 978-1033).
 * result_size returns elements or
 * -1; result_copy fails when nbytes is too small. */
long madam_b200_result_size(const char *name);
int madam_b200_result_copy(const char *name, void *dst, long nbytes);

/* Times `iters` PCG iterations (after `warmup`) restarted from the RHS of the
 * last solve, inputs resident in HBM; out[0..7] = total ms, ms per
 * iteration, kernel launches per iteration, scatter / filter / gather /
 * preconditioner / update ms per iteration.  No reference counterpart. */
int madam_b200_bench_iterations(int warmup, int iters, double *out, long nout);

/* Number of kernels the library has launched.  No reference counterpart. */
unsigned long long madam_b200_kernel_launches(void);

/* Host check of the integer division used in the kernels (0 = pass).  No
 * reference counterpart. */
int madam_b200_selftest_fastdiv(void);

/* Hit counts and inverse pixel matrices (the "hits" and "cc" products of
 * destripe) of a pointing that is already in device memory, computed
 * without allocating any device memory.  No counterpart in the reference
 * (whose pixel_matrix / count_hits, src/smadam_routines.f90:111-246,
 * 349-422, and invert_pixelmatrix_map, src/map_routines.f90:218-321, run
 * inside destripe).
 *
 * All arrays are device memory owned by the caller: detweights [ndet],
 * pix int64 [ndet][nsamp] (NESTED at nside; negative = flagged, skipped),
 * pixweights float64 [ndet][nsamp][nnz], hits int32 [12 nside^2], cc
 * float64 [12 nside^2][nnz][nnz].  Every array must be device memory of the
 * current device (or managed memory).  A pixel matrix is rejected, and its
 * cc entries zeroed, by the reference's invert_pixelmatrix_map test with
 * allow_decoupling = F and incomplete_matrices = F (fixed; the reference
 * defaults): pixmode 0 rejects det(C) < pixlim, pixmode 1 rejects
 * det(C) (3 / trace C)^3 < pixlim, pixmode 2 rejects rcond (smallest over
 * largest eigenvalue) < pixlim.  Work is queued on `stream` (NULL = legacy
 * default stream) and is complete once that stream is synchronised.
 * Limits: nside <= 64 (the accumulators are a fixed 2.75 MB device array of
 * 49152 pixels; larger maps return status 1 and say so); nnz 1 or 3.  The
 * first call on a device looks up that array's address and loads the code of
 * all this entry point's kernels (for every nnz), so make it before any
 * stream capture; later calls load and allocate nothing.  Calls that overlap
 * on one device share the array and race.  A CUDA error already pending when
 * the call starts is reported as status 2 and left pending; no work is
 * queued.  Returns 0, 1 (invalid argument) or 2 (CUDA error); the message
 * goes to err (errlen bytes, may be NULL). */
int madam_b200_pixel_matrices_noalloc(long nside, long nnz, long ndet, long nsamp,
                                      const double *detweights, const long long *pix,
                                      const double *pixweights, long pixmode, double pixlim,
                                      int *hits, double *cc, void *stream, char *err,
                                      long errlen);

#ifdef __cplusplus
}
#endif

#endif
