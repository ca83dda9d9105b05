// The destriping engine: state of one destripe() solve on one GPU.
//
// Host orchestration follows destripe() (smadam.F90:64-590) and
// destripe_with_cache() (smadam.F90:593-918).  All sample- and map-domain
// work runs as CUDA kernels; the host keeps the small tables (baseline layout,
// PSDs, trimmed filter segments) and drives the PCG loop.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <future>
#include <initializer_list>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "band2.cuh"
#include "comm.h"
#include "common.cuh"
#include "params.h"

namespace madam {

constexpr int kRedBlocks = 1184;      // 148 SMs x 8, fixed for determinism
constexpr int kMaxBasis = 8;          // basis_order + 1 at most
// FP32-TOD forms: a reliable update (true float64 residual) each time the
// squared residual norm the float32 projections carried has dropped by this
// factor since the last one
constexpr double kReliableDrop = 1e-6;


// A job's CG vectors for the serving stepper's shared launches (pcg_shared).
struct PcgJob {
  double *aa, *r, *ro, *p, *ap, *z, *pw;
  const double *bw;
  const uint8_t *rmask;
  double *part, *scal;
  long long nb;
  int active;
};

// Shared launches over the PCG jobs of a device table of n entries, on st:
// step 0: aa += alpha p, ro = r, r -= alpha ap (k_update_ar of each job);
// step 1: r.z, ro.z, r.r and the CG scalars of each job, its rz and rr also
// to out[2 j], out[2 j + 1] (k_dots + k_finish mode 2); step 2: p = z + beta
// p, pw = p bw (k_update_p).  Same grids and reduction order as the
// single-job kernels; nbmax: the largest job's vector length.
void pcg_shared(cudaStream_t st, const PcgJob *tab, int n, long long nbmax, int step,
                double *out);

// Owning device allocation.
// Device memory of the engine: stream-ordered allocations on the stream of
// the engine the calling thread is working for (several engines may run in
// parallel host threads), served by the device's default memory pool, which keeps freed
// blocks for reuse (one destripe call allocates and frees several GB of
// temporaries; the pool turns the repeats into bookkeeping).
extern thread_local cudaStream_t g_alloc_stream;

// True when every non-null buffer is device memory of device `dev` (< 0: the
// current one) or managed memory, false when all are host memory; throws on a
// mix, or on device memory of another GPU.
bool inputs_on_device(int dev, std::initializer_list<const void *> ptrs);
void *dev_alloc(size_t bytes);
void dev_free(void *p);

template <typename T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { reset(); }
  void reset() {
    if (p) dev_free(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count == n && p) return;
    reset();
    if (count == 0) return;
    p = (T *)dev_alloc(count * sizeof(T));
    n = count;
  }
  void zero(cudaStream_t s) {
    if (n) MADAM_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  // at least count elements (kept when already as large)
  void reserve(size_t count) {
    if (count > n) alloc(count);
  }
  T *get() const { return p; }
};

// A filtered / preconditioned piece of one (detector, period): the baselines
// kept by trim_interval (noise_routines.f90:764-813).
struct Segment {
  int det, iv, isub;
  long k0;       // first baseline, index into the [det][noba_short] vectors
  long noba;
  int psd_filter;  // psd_index at the period start (convolve_interval)
  int psd_prec;    // psd_index at the segment start (preconditioning_band)
  int prec_ok;     // psd_index_det >= 0 and detector weight != 0
};

// Device table entry of the batched FFT convolution.
struct ConvSeg {
  long long x_off;   // input offset into the source vector
  long long y_off;   // output offset into the destination vector
  int n_in;          // input length (zero padded to the FFT length)
  int n_out;         // output length
  int spec;          // spectrum row
  int flags;         // bit 0: subtract input mean, bit 1: subtract output mean
};

// Per-segment band Cholesky factor location.
struct BandSeg {
  long long k0;      // first baseline of the segment
  long long l_off;   // offset of the factor in the band store
  int n;             // rows
  int nband;         // band width (kd + 1)
};

struct Timings {
  double setup_ms = 0, iterate_ms = 0, finalize_ms = 0, total_ms = 0;
  double scatter_ms = 0, gather_ms = 0, filter_ms = 0, precond_ms = 0, other_ms = 0;
};

struct FFTPlan;  // fft.cu
struct CgpWork;  // engine_host.inl

class Engine {
 public:
  Engine();
  ~Engine();

  // Full destripe().  Pointers are host or device memory (is_device).
  void run(const Params &par, std::vector<Detector> dets, long ndet, long nsamp,
           long nnz, double *timestamps, int32_t *pix, float *pixweights,
           double *signal, long nperiod, const long *periods, bool is_device);
  // destripe_with_cache(): new TOD, cached pixel matrices / filter / preconditioner
  // path_output of the cached parameters (destripe_with_cache's outpath)
  void set_output_path(const std::string &path) { par_.path_output = path; }
  void run_cached(long ndet, long nsamp, long nnz, double *timestamps,
                  int32_t *pix, float *pixweights, double *signal,
                  bool is_device);

  // Batched Monte Carlo: nrhs realisations of destripe_with_cache() sharing
  // the pointing, solved as one multi-right-hand-side PCG.  signals:
  // [nrhs][ndet][nsamp].  Each realisation is solved as destripe_with_cache
  // would solve it right after the caching destripe(); the cache is left as
  // it was.
  void run_cached_batch(long ndet, long nsamp, long nnz, double *timestamps, int32_t *pix,
                        float *pixweights, long nrhs, double *signals, bool is_device,
                        bool fp32 = false);

  // Precision of the next run(): false = FP64 TOD (destripe), true = the
  // FP32-TOD form (madam_b200_destripe_fp32): `signal` holds float32
  // samples, the PCG projections read float32 pointing sums and a float32
  // copy of the map; pixel matrices, baselines and reductions stay FP64.
  void set_fp32(bool v) { fp32_next_ = v; }
  bool fp32() const { return fp32_; }
  long long pairs() const { return use_pairs_ ? npairs_ : 0; }

  // Rank of a sharded run (comm.h), or nullptr for a single rank.
  void set_comm(Comm *c) { comm_ = c; }
  bool sharded() const { return comm_ && comm_->nranks > 1; }

  // Subchunk pass of the next run() (nsubchunk > 1): isub 1..nsub bins and
  // solves only that subchunk of every interval; 0 is the full-data pass.
  void set_subchunk(int isub, int nsub) {
    isubchunk_ = isub;
    nsubchunk_ = nsub;
  }
  void keep_subchunk_results(int isub);
  void clear_subchunk_results() {
    subchunk_d_.clear();
    subchunk_i_.clear();
  }

  bool cached() const { return cached_; }
  const Params &params() const { return par_; }

  // Named results (host copies).  Maps are full sky at nside_map.
  long result_size(const std::string &name);
  void result_copy(const std::string &name, void *dst, long nbytes);

  // destripe() in parts, for the serving stepper: run_setup (everything
  // before the PCG), the stepwise PCG (pcg_*), run_finish (maps, files)
  void run_setup(const Params &par, std::vector<Detector> dets, long ndet, long nsamp, long nnz,
                 double *timestamps, int32_t *pix, float *pixweights, double *signal,
                 long nperiod, const long *periods, bool is_device);
  void run_finish();
  void run_solve();                // the PCG (or write_covmat) as destripe() runs it
  bool stepwise_ok() const;        // the PCG can be stepped (kfirst, no covmat, one rank)
  bool pcg_begin();                // first residual; false: no iteration to do
  void pcg_use_stream(cudaStream_t s);  // launch the steps on s (nullptr: own stream)
  void pcg_apply();                // A p and alpha
  void pcg_precond();              // z = M r
  PcgJob pcg_job();
  bool pcg_after(double rz, double rr);  // after a round: true when the PCG stops
  void pcg_end();

  // Times `iters` PCG iterations on the state of the last solve (bench).
  void bench_iterations(int warmup, int iters, std::vector<double> &out);

  Timings timings;
  static constexpr int kSetupMarks = 10;
  double setup_marks_[kSetupMarks] = {0};
  long noiter = 0;
  double rrinit = 0, rr_final = 0;
  std::vector<double> rr_history;
  unsigned long long launches_iter = 0;

 private:
  // --- setup phases
  void bind_inputs(double *timestamps, int32_t *pix, float *pixweights,
                   double *signal, bool is_device, bool first_call);
  void init_layout(long nperiod, const long *periods);
  void flag_and_compact(bool first_call);
  void build_runs();
  void build_csr();
  void setup_scatter();
  void map_side_setup();
  void apply_inmask();
  void initialize_a();
  void build_segments();
  void build_filter();
  void filter_spectra(const std::vector<std::pair<long, int>> &tasks, long nh);
  void build_filter_finish();
  void construct_preconditioner();
  void build_guarded_chunks(const std::vector<PRun> &pruns, const std::vector<PRun> &cruns);
  // checknan diagnostics: [0] detectors with NaN parameters, NaN counts of
  // [1] yba, [2] the binned cross map, [3] the pointing weights, [4] r, [5] z,
  // [6] p at the first CG step
  static constexpr int kNanChecks = 7;
  std::vector<double> nan_checks_;
  unsigned long long count_nan(const double *v, long long n);
  unsigned long long count_nan(const float *v, long long n);
  void check_nan_setup();
  void check_nan_iterate(double rz, long long nb);
  std::vector<GChunk> make_gchunks(int Cg, int G, std::vector<int> &cls_begin,
                                   std::vector<int> &seg_off) const;
  int guard_chunk_len(long long npos) const;
  void iterate();
  void pcg_reset();
  bool pcg_stop_test(long istep, double rz, double rr);
  long pcg_istep_ = 0;
  double pcg_t0_ = 0, run_t0_ = 0, pcg_rr_true_ = 0;
  bool pcg_reliable_ = false;
  const double *pcg_bw_ = nullptr;
  const uint8_t *pcg_rmask_ = nullptr;
  cudaStream_t pcg_own_st_ = nullptr;
  void finalize(bool first_call);
  void writeback_host();
  void write_fits(bool first_call);

  // --- batched Monte Carlo
  void iterate_batch();
  void apply_A_batch();
  bool batch_timed_ = false;  // iterate_batch: phase events in apply_A_batch
  void apply_preconditioner_batch(const double *r, double *z);
  void build_batch_tables();
  template <int G>
  void project_group_T(long r0, int nr);
  template <int G, class T>
  void project_group_T2(long r0, int nr);
  // Launch-shape tuner of the batched projections: the grid of a kernel is
  // chosen once per (kernel, work items, right-hand-side width) by timing
  // one launch at each candidate (one to four waves of resident CTAs, and
  // the reduction grid) and kept for the process; a tuning pass runs only
  // while tune_batch_ is set (before the timed iterations).
  template <class L>
  unsigned tuned_grid(const void *kern, int key, long long items, int GW, L launch);
  bool tune_batch_ = false;
  bool tuned(int key, long long items, int GW);  // a shape tuned_grid has already timed
  DevBuf<double> pwT_, lmapT_, scatpT_, apnT_;  // right-hand-side-minor copies
  DevBuf<float> pwTf_, lmapTf_;                 // their float32 forms (FP32-TOD batch)
  long nrhs_ = 0;                        // right-hand sides of the last batch
  DevBuf<double> yb_, aab_, rb_, pb_, zb_, apb_, rob_, pwb_;  // [R][nb]
  DevBuf<double> lmapb_, scatpb_;        // [R][nloc_cross][nmap], scatter partials
  DevBuf<double> binb_, mapb_, binmapb_; // [R][nloc][nmap]
  DevBuf<double> partb_, scalb_;         // [R][3][kRedBlocks], [R][S_NSCAL]
  DevBuf<int> actb_, actu_;              // active / reliably updated right-hand sides
  // reliable updates of several right-hand sides at once: their A x through
  // the float64 batched projections on the pixel-sorted samples
  DevBuf<double> xsb_, pwsb_, apsb_, partsb_, scalsb_;
  DevBuf<int> actsb_;
  void true_residual_batch(const std::vector<long> &upd);
  long nrhs_alt_ = 0;  // the batch size while true_residual_batch runs its own
  std::vector<int> act_host_;
  std::vector<double> noiter_b_, rrinit_b_, rrfinal_b_;
  // band factor tables replicated per right-hand side (offsets k0 + r nb)
  std::vector<PSeg> band2_pseg_h_;
  std::vector<PChunk> band2_ch_h_;
  DevBuf<PSeg> p2segs_b_;
  DevBuf<PChunk> p2ch_b_;
  DevBuf<GChunk> p2gc_b_;
  std::vector<int> band2_gcls_begin_b_;
  DevBuf<double> p2y_b_;
  DevBuf<int> p2tf_b_, p2tb_b_;
  DevBuf<double> p2wp_b_, p2ws_b_;
  std::vector<int> band2_cls_begin_b_, band2_cls_seg_b_;
  int p2nseg_b_ = 0, p2nch_b_ = 0;
  DevBuf<ConvSeg> filt_segs_b_d_;
  long batch_tables_r_ = 0;              // right-hand sides the tables were built for
  bool suppress_fits_ = false;

  // --- iteration pieces
  void apply_A(const double *p, const double *pw, double *ap, bool timed);
  void bin_tod(bool accumulate_wamap);
  void subtract_baselines();
  void clean_tod();
  void apply_preconditioner(const double *r, double *z);
  // higher-order baselines (basis_order > 0)
  void initialize_a_basis();
  void basis_vectors();
  void scatter_basis(const double *amp, double sign, double *target, bool fine);
  void apply_A_basis(const double *p, double *ap, bool timed);
  void precondition_basis(const double *r, double *z);
  void clean_tod_basis();
  // the inverse noise covariance files (file_covmat) in place of the solve
  void write_covmat();
  void scatter_baselines(const double *pw, double *target, bool fine);
  void convolve(const double *x, double *y, const std::vector<ConvSeg> &segs,
                const double *spectra, DevBuf<ConvSeg> &dsegs);
  void cg_preconditioner_segments(const double *r, double *z);
  // global: the inner product spans the ranks of a sharded run
  void finish_dots(int nd, int mode, int slot0, int nblk = kRedBlocks, bool global = false);

  Params par_;
  std::vector<Detector> dets_;
  bool cached_ = false;
  cudaStream_t st_ = nullptr;
  cudaEvent_t ev_[8];
  // host-signal upload on a copy stream, overlapped with the pointing setup
  // (bind_inputs); wait_tod() orders the engine stream after it
  cudaStream_t cst_ = nullptr;
  cudaEvent_t ev_ptr_ = nullptr, ev_tod_ = nullptr;
  bool tod_pending_ = false;
  void wait_tod();
  void sync_tod();

  // sizes
  long ndet_ = 0, nsamp_ = 0, nnz_ = 0;
  int nmap_ = 0;
  long nside_max_ = 0, nosubmaps_tot_ = 0, nosubpix_max_ = 0, nosubpix_map_ = 0,
       nosubpix_cross_ = 0, ndeg_cross_ = 1, ndeg_shift_ = 0;
  long ninterval_ = 0, noba_short_ = 0, noba_pp_max_ = 0, nshort_ = 0;
  double dnshort_ = 0;
  FastDiv fdn_;
  int gather_kb_ = 0;
  DevBuf<int2> gather_chunks_;  // {first global baseline, baselines} per warp chunk
  long long ngather_chunks_ = 0;
  long long gather_tiles_det_ = 0;
  std::vector<long> intervals_, istart_iv_, noba_pp_, kstart_pp_;
  std::vector<uint32_t> bstart_;  // noba_short + 1
  std::vector<double> btime_;
  std::vector<double> detw_iv_;   // [det * ninterval + iv], 0 = skipped
  std::vector<double> bw_host_;   // per baseline detector weight

  // compaction
  std::vector<int> ksubmap_;
  std::vector<long> subtable1_, subtable2_;
  long nolocmaps_ = 0, nloc_ = 0, nloc_map_ = 0, nloc_cross_ = 0;
  long dummy_local_ = 0, dummy_global_ = 0;
  int tile_shift_ = 0;
  long ntiles_ = 0;

  // inputs
  bool in_device_ = false;
  int32_t *d_pix_caller_ = nullptr;
  double *h_signal_ = nullptr;
  int32_t *h_pix_ = nullptr;
  double *d_tod_ = nullptr;   // device signal (caller's or ours)
  DevBuf<double> tod_own_;
  DevBuf<int32_t> pix_;       // working pixel numbers
  DevBuf<float> wraw_;        // staging copy of host weights
  const float *d_w_ = nullptr;
  DevBuf<float4> point4_;     // nnz = 3: {w0, w1, w2, compacted pixel}
  DevBuf<int32_t> pixc_;      // nnz = 1: compacted pixel
  DevBuf<uint32_t> bstart_d_;
  DevBuf<double> bw_;         // per-baseline detector weight
  DevBuf<uint8_t> rmask_;
  // basis_order + 1 amplitudes per baseline: the F^T F inverses and the
  // per-amplitude detector weights / residual mask
  int nbasis_ = 1;  // at most kMaxBasis
  DevBuf<double> nna_inv_, bwn_;
  DevBuf<uint8_t> rmaskn_;
  DevBuf<double> times_d_;

  // runs for the privatised scatters
  DevBuf<Run> runs_;
  DevBuf<int> item_begin_;   // nwork + 1 run offsets
  DevBuf<int> item_tile_;    // tile of each work item
  long nruns_ = 0, nwork_ = 0;
  DevBuf<float4> sp4_;        // pixel-sorted pointing {w, baseline}
  DevBuf<int2> sp2_;          // pixel-sorted baseline (temperature only)
  DevBuf<int> csr_off_;       // nloc_cross + 1 offsets
  DevBuf<int4> scatter_chunks_;  // {pixel, first entry, entries, partial slot}
  DevBuf<int4> scatter_multi_;   // {pixel, first slot, chunks} of multi-chunk pixels
  DevBuf<double> scatter_partial_;
  long long nscatter_chunks_ = 0;
  int nscatter_multi_ = 0;
  long long csr_nvalid_ = 0;
  DevBuf<long long> istart_d_;
  DevBuf<int> kstart_d_;
  DevBuf<int32_t> pix_orig_;

  // map domain (compacted)
  DevBuf<double> cc_, cca_, map_, binmap_, wamap_, lmap_, lmap_fine_;
  DevBuf<int> hits_, mask_;
  DevBuf<float> crit_;
  DevBuf<int> flagcount_;

  // baseline domain
  DevBuf<double> aa_, yba_, nna_, r_, p_, z_, ap_, ro_, pw_, tmpv_;
  std::vector<double> nna_host_;
  std::vector<double> cc_raw_host_;
  DevBuf<double> part_, scal_;
  std::vector<double> scal_host_;

  // filter / preconditioner
  long nof_ = -1, npsdtot_ = 0;
  std::vector<int> psddet_;
  std::vector<double> psdstart_, psdstop_;
  std::vector<double> fcov_host_, invcov_host_;
  DevBuf<double> fcov_, fprec_, invcov_, delta_;
  std::vector<Segment> segs_;
  std::vector<ConvSeg> filt_segs_, fprec_segs_;
  DevBuf<ConvSeg> filt_segs_d_, fprec_segs_d_, tmp_segs_d_;
  bool use_diagonal_ = false;
  DevBuf<double> prec_diag_;
  std::vector<BandSeg> band_segs_;
  DevBuf<BandSeg> band_segs_d_;
  DevBuf<double> band_;
  std::vector<int> cg_prec_segs_;   // segments without a band factor
  std::vector<long> band_widths_;
  DevBuf<PSeg> p2segs_;
  DevBuf<PRun> p2runs_, p2cruns_;
  DevBuf<PChunk> p2ch_;
  DevBuf<int> p2tf_, p2tb_;  // per-chunk transfer offsets, forward / backward
  DevBuf<double> p2rows_, p2T_, p2wp_, p2ws_;
  int p2nseg_ = 0, p2nch_ = 0;
  long long band2_rows_ = 0;
  long band2_ntrans_ = 0;
  int band2_chunk_ = 0;
  std::vector<int> band2_cls_w_, band2_cls_begin_, band2_cls_seg_;
  // guarded solve (band2_solve_guarded): chunks of band2_gchunk_ rows with
  // guards of band2_guard_ positions, when every chunk's guard checks out
  bool band2_guarded_ = false;
  int band2_guard_ = 0, band2_gchunk_ = 0;
  std::vector<GChunk> band2_gch_h_;
  std::vector<PRun> band2_pruns_h_, band2_cruns_h_;
  std::vector<int> band2_gcls_begin_, band2_gseg_off_;
  DevBuf<GChunk> p2gc_;
  DevBuf<double> p2y_;  // forward solution L^-1 r, full baseline vector
  DevBuf<int> band2_err_;  // a staging wait of the guarded solve ran out
  void check_band_err();
  // setup trace: with MADAM_B200_TRACE set, each step's host time (after a
  // synchronisation of the stream) goes to stderr
  bool trace_on_ = false;
  double trace_t_ = 0;
  cudaEvent_t trace_ev_[2] = {nullptr, nullptr};
  void trace(const char *what);
  long n_band_fail_ = 0;
  std::unique_ptr<FFTPlan> fft_;
  std::future<void> filter_job_;  // host spectra of build_filter
  std::string filter_err_;
  // filter spectra computed on the device (build_filter); the host copy of
  // fcov and of the inverse-covariance kernels is made when asked for
  bool filter_dev_ = false, fcov_host_valid_ = false, invcov_valid_ = false;
  DevBuf<int> filter_flag_;
  std::vector<std::pair<long, int>> filter_tasks_;
  std::unique_ptr<SpectrumFile> spectrum_file_;  // file_spectrum's table
  std::vector<double> filter_sigma0_;
  const std::vector<double> &fcov_host();
  const std::vector<double> &invcov_host();
  std::unique_ptr<CgpWork> cgp_;

  // pixels flagged during the call (host write-back)
  DevBuf<long long> flagged_idx_;
  DevBuf<int32_t> flagged_val_;
  std::vector<int32_t> orig_pix_values_;
  bool tod_cleaned_ = false;

  // subsets and leakage matrices (subsets.inl)
  void run_subsets();
  void leak_matrices();
  void check_same_detectors();
  void subset_accumulate(const std::vector<uint8_t> &detflags, const std::vector<double2> &spans,
                         int nmaps, double *cc, double *bin, int *hits);
  std::vector<double> leak_product(const std::vector<double> &cinv,
                                   const std::vector<double> &cdet, int nmaps);
  std::vector<double> detector_matrix(long det, int nmaps);
  static std::vector<double> full_sym(const std::vector<double> &packed, int nmaps);
  // compacted per-pixel arrays (device or host) -> full sky, zeros elsewhere
  void expand_to_sky(const void *dev, size_t elem, long per_pix, long nosubpix, void *out);
  void expand_host(const void *host, size_t elem, long per_pix, long nosubpix, void *out);
  const double *times_in_ = nullptr;  // the caller's timestamps
  bool times_dev_ = false;
  DevBuf<double> times_own_;
  const double *subset_times_ = nullptr;
  std::vector<double2> subset_spans_;
  std::map<std::string, std::vector<double>> extra_d_;  // subset / leakage results
  std::map<std::string, std::vector<int>> extra_i_;
  int isubchunk_ = 0, nsubchunk_ = 0;
  // sharded runs: in-place reductions across the ranks (no-ops on one rank)
  Comm *comm_ = nullptr;
  void ar_sum(double *dev, size_t n) {
    if (sharded()) comm_->allreduce(dev, n, 0, st_);
  }
  void ar_sum(int *dev, size_t n) {
    if (sharded()) comm_->allreduce(dev, n, 0, st_);
  }
  void ar_max(int *dev, size_t n) {
    if (sharded()) comm_->allreduce(dev, n, 1, st_);
  }
  double ar_sum_host(double v);
  bool writes_files() const { return !comm_ || comm_->rank == 0; }
  int rank() const { return comm_ ? comm_->rank : 0; }
  std::map<std::string, std::vector<double>> subchunk_d_;  // products of subchunk passes
  std::map<std::string, std::vector<int>> subchunk_i_;

  // FP32-TOD form
  bool fp32_next_ = false, fp32_ = false;
  float *sig32_caller_ = nullptr;  // caller's float32 signal (host or device)
  bool build_pairs();
  void build_scatter_chunks();
  bool use_pairs_ = false;        // PCG projections over pointing pairs
  long long npairs_ = 0;
  DevBuf<float4> gp4_;            // time-ordered pairs {sum w, cross pixel}
  DevBuf<int> poff_;              // first pair of each baseline [nb + 1]
  DevBuf<int4> pair_chunks_;      // gather chunks over pairs {b0, nbl, first pair, pairs}
  long long npair_chunks_ = 0;
  DevBuf<float4> lmapf_;          // float32 map copy read by the FP32 gather
  DevBuf<double2> lmapg_;         // padded FP64 map copy {I, Q}, {U, 0}
  // reliable updates of the FP32-TOD forms: the true residual b - A x with
  // float64 projections over the exact sample pointing
  // (the single FP32-TOD solve projects through float32 only with nmap 3)
  bool refine() const { return fp32_ && nmap_ == 3; }
  void apply_A_exact(const double *x, double *ax);
  void true_residual(const double *x, const double *b, double *r);
  DevBuf<double> pwx_, lmapx_, apx_, partx_;
  DevBuf<double2> lmapgx_;
  // FP32-TOD form: the pixel-sorted samples and their scatter chunks, kept
  // beside the pairs for the exact scatter
  void build_sample_csr();
  void swap_csr();
  bool have_xcsr_ = false;
  DevBuf<float4> xsp4_;
  DevBuf<int2> xsp2_;
  DevBuf<int> xcsr_off_;
  DevBuf<int4> xscatter_chunks_, xscatter_multi_;
  DevBuf<double> xscatter_partial_;
  long long xnscatter_chunks_ = 0, xcsr_nvalid_ = 0;
  int xnscatter_multi_ = 0;
  long n_reliable_ = 0;           // reliable updates of the last solve
};

}  // namespace madam
