/* Drop-in C-ABI of the Madam destriping library, implemented for NVIDIA B200
 * (sm_100a) by libmadam_b200/libmadam.so.
 *
 * The three entry points keep the reference's exact signatures and argument
 * meaning:
 *   destripe             reference src/madam.h:1-2, src/smadam.F90:64-101
 *   destripe_with_cache  reference src/smadam.F90:593-609 (exported, not in
 *                        the reference header)
 *   clear_caches         reference src/smadam.F90:921
 * Buffers: timestamps float64[nsamp]; pix int32[ndet][nsamp];
 * pixweights float32[ndet][nsamp][nnz]; signal float64[ndet][nsamp];
 * periods int64[nperiod] (start offsets); npsd int64[ndet];
 * psdstarts float64[npsdtot]; psdfreqs float64[npsdbin];
 * psdvals float64[npsdval].  Host or CUDA device pointers are accepted.
 * nnz is 1 (temperature) or 3 (I, Q, U); other values are refused, since
 * the reference's general pixel matrix (src/smadam_routines.f90:227) hands
 * its float32 weights to the float64 BLAS dsyr and so has no defined result.
 * pix is rewritten in place (flagged samples become 12*nside_max^2) and
 * signal is destriped in place when write_tod or subsets are set, as in the
 * reference.  `comm` is a Fortran MPI handle in the reference; here it is 0
 * (one rank) or a handle of madam_b200_comm_init_nccl / _host (madam_b200.h),
 * whose ranks each pass their own share of the data and get the whole maps,
 * as the reference's MPI ranks do.  Any other value runs one rank: an MPI
 * handle has no meaning to this library (library handles start at
 * 0x2D420001, away from Open MPI's and MPICH's Fortran handle values), so a
 * job of several MPI ranks must pass library communicators.  On an error the reference aborts the MPI job;
 * these void entry points print the message and return; the status is
 * available from madam_b200_last_error (madam_b200.h).
 */
#ifndef MADAM_H
#define MADAM_H

#ifdef __cplusplus
extern "C" {
#endif

void destripe(int comm, char *parstring, long ndet, char *detstring, double *detweights,
              long nsamp, long nnz, void *timestamps, void *pix, void *pixweights, void *signal,
              long nperiod, long *periods, long *npsd, long npsdtot, double *psdstarts,
              long npsdbin, double *psdfreqs, long npsdval, double *psdvals);

void destripe_with_cache(int comm, long ndet, long nsamp, long nnz, void *timestamps, void *pix,
                         void *pixweights, void *signal, char *outpath);

void clear_caches(void);

#ifdef __cplusplus
}
#endif

#endif
