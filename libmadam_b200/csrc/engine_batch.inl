// Batched Monte Carlo: many destripe_with_cache() realisations (smadam.F90:
// 593-918) that share one pointing, solved together.
//
// The reference solves Monte Carlo realisations one destripe_with_cache call
// at a time.  Here the pointing-side setup (flagging, compaction, runs, the
// pixel-sorted pointing) is done once, every realisation gets its own binned
// map and right-hand side (bin_tod + initialize_a on top of the cached
// state), and the R systems are solved as one multi-right-hand-side PCG:
// each pass over the pointing serves a group of right-hand sides, the
// filter and the band preconditioner run over R copies of their segment
// tables, and every right-hand side keeps its own CG scalars, convergence
// test and iteration count (iterate_a, smadam_routines.f90:677-983, per
// realisation).  The per-realisation arithmetic is that of the single solve.

namespace {
constexpr int kScatterGroup = 8;  // right-hand sides per scatter pass (long baselines)
}  // namespace

void Engine::build_batch_tables() {
  // band factor tables and filter segments replicated for nrhs_ right-hand
  // sides (vector offsets r * nb), grouped by width class
  const long long nb = (long long)ndet_ * noba_short_;
  if (batch_tables_r_ == nrhs_) return;
  std::vector<PSeg> ps;
  std::vector<PChunk> ch;
  std::vector<int> tf, tb;
  band2_cls_begin_b_.clear();
  band2_cls_seg_b_.clear();
  for (size_t i = 0; i + 1 < band2_cls_seg_.size(); ++i) {
    band2_cls_begin_b_.push_back((int)ch.size());
    band2_cls_seg_b_.push_back((int)ps.size());
    for (long r = 0; r < nrhs_; ++r)
      for (int s = band2_cls_seg_[i]; s < band2_cls_seg_[i + 1]; ++s) {
        PSeg q = band2_pseg_h_[s];
        q.k0 += r * nb;
        q.ch_off = (int)ch.size();
        const int sn = (int)ps.size();
        ps.push_back(q);
        for (int c = band2_pseg_h_[s].ch_off; c < band2_pseg_h_[s].ch_off + q.nch; ++c) {
          PChunk k = band2_ch_h_[c];
          k.seg = sn;
          ch.push_back(k);
          tf.push_back(k.tf);
          tb.push_back(k.tb);
        }
      }
  }
  band2_cls_begin_b_.push_back((int)ch.size());
  band2_cls_seg_b_.push_back((int)ps.size());
  // the guarded chunks, replicated the same way (segment r * nseg_class + s),
  // at the chunk length of the whole batch's positions
  if (band2_guarded_) {
    long long npos = 0;
    for (const PSeg &q : band2_pseg_h_) npos += q.n;
    std::vector<int> gb1, soff;
    const std::vector<GChunk> one =
        make_gchunks(guard_chunk_len(npos * nrhs_), band2_guard_, gb1, soff);
    std::vector<GChunk> gcs;
    band2_gcls_begin_b_.clear();
    for (size_t i = 0; i + 1 < band2_cls_seg_.size(); ++i) {
      band2_gcls_begin_b_.push_back((int)gcs.size());
      const int sbase = band2_cls_seg_b_[i];
      const int ns = band2_cls_seg_[i + 1] - band2_cls_seg_[i];
      for (long r = 0; r < nrhs_; ++r)
        for (int s = band2_cls_seg_[i]; s < band2_cls_seg_[i + 1]; ++s)
          for (int c = soff[s]; c < soff[s + 1]; ++c) {
            GChunk k = one[c];
            k.seg = sbase + (int)r * ns + (s - band2_cls_seg_[i]);
            gcs.push_back(k);
          }
    }
    band2_gcls_begin_b_.push_back((int)gcs.size());
    p2gc_b_.alloc(std::max<size_t>(1, gcs.size()));
    if (!gcs.empty())
      MADAM_CUDA(cudaMemcpyAsync(p2gc_b_.get(), gcs.data(), gcs.size() * sizeof(GChunk),
                                 cudaMemcpyHostToDevice, st_));
  }
  p2nseg_b_ = (int)ps.size();
  p2nch_b_ = (int)ch.size();
  if (!ps.empty()) {
    p2segs_b_.alloc(ps.size());
    p2ch_b_.alloc(ch.size());
    p2tf_b_.alloc(tf.size());
    p2tb_b_.alloc(tb.size());
    p2wp_b_.alloc((size_t)ch.size() * kBand2State);
    p2ws_b_.alloc((size_t)ch.size() * kBand2State);
    MADAM_CUDA(cudaMemcpyAsync(p2segs_b_.get(), ps.data(), ps.size() * sizeof(PSeg),
                               cudaMemcpyHostToDevice, st_));
    MADAM_CUDA(cudaMemcpyAsync(p2ch_b_.get(), ch.data(), ch.size() * sizeof(PChunk),
                               cudaMemcpyHostToDevice, st_));
    MADAM_CUDA(cudaMemcpyAsync(p2tf_b_.get(), tf.data(), tf.size() * sizeof(int),
                               cudaMemcpyHostToDevice, st_));
    MADAM_CUDA(cudaMemcpyAsync(p2tb_b_.get(), tb.data(), tb.size() * sizeof(int),
                               cudaMemcpyHostToDevice, st_));
  }
  // the filter segments (also those of the fprecond preconditioner)
  const std::vector<ConvSeg> &fs = filt_segs_;
  std::vector<ConvSeg> cs;
  for (long r = 0; r < nrhs_; ++r)
    for (ConvSeg c : fs) {
      c.x_off += r * nb;
      c.y_off += r * nb;
      cs.push_back(c);
    }
  if ((long)cs.size() > 65535) fail("too many filter segments in one batch (reduce nrhs)");
  filt_segs_b_d_.alloc(std::max<size_t>(1, cs.size()));
  if (!cs.empty())
    MADAM_CUDA(cudaMemcpyAsync(filt_segs_b_d_.get(), cs.data(), cs.size() * sizeof(ConvSeg),
                               cudaMemcpyHostToDevice, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  batch_tables_r_ = nrhs_;
}

void Engine::apply_preconditioner_batch(const double *r, double *z) {
  // preconditioning_band (noise_routines.f90:1159-1256) for every right-hand side
  const long long nb = (long long)ndet_ * noba_short_;
  const long long nt = nb * nrhs_;
  if (par_.precond_width_max < 1) {
    MADAM_CUDA(cudaMemcpyAsync(z, r, nt * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    return;
  }
  if (use_diagonal_) {
    for (long k = 0; k < nrhs_; ++k)
      MADAM_LAUNCH(k_mul, grid_for(nb), 256, 0, st_, z + k * nb, r + k * nb, prec_diag_.get(), nb);
    return;
  }
  MADAM_CUDA(cudaMemcpyAsync(z, r, nt * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  const long nfs = (long)filt_segs_.size() * nrhs_;
  if (par_.use_fprecond) {
    if (nfs > 0) fft_->convolve(st_, filt_segs_b_d_.get(), nfs, fprec_.get(), npsdtot_, r, z);
    return;
  }
  if (band2_guarded_) {
    p2y_b_.alloc(std::max<long long>(1, nt));
    band2_solve_guarded(st_, p2segs_b_.get(), p2gc_b_.get(), band2_cls_w_.data(),
                        band2_gcls_begin_b_.data(), (int)band2_cls_w_.size(), p2runs_.get(),
                        p2cruns_.get(), p2rows_.get(), r, p2y_b_.get(), z, band2_err_.get());
  } else {
    band2_solve(st_, p2segs_b_.get(), p2nseg_b_, p2ch_b_.get(), p2nch_b_, p2tf_b_.get(),
                p2tb_b_.get(), band2_cls_w_.data(), band2_cls_begin_b_.data(),
                band2_cls_seg_b_.data(), (int)band2_cls_w_.size(), p2runs_.get(),
                p2cruns_.get(), p2rows_.get(), p2T_.get(), r, z, p2wp_b_.get(), p2ws_b_.get());
  }
  for (long k = 0; k < nrhs_; ++k) {
    band_solve(st_, band_segs_d_.get(), (int)band_segs_.size(), band_.get(), r + k * nb,
               z + k * nb);
    cg_preconditioner_segments(r + k * nb, z + k * nb);
  }
}

namespace {
std::mutex g_tune_mu;
// (device, kernel, items, GW) -> grid
std::map<std::tuple<int, int, long long, int>, unsigned> g_tuned;
int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}
}  // namespace

bool Engine::tuned(int key, long long items, int GW) {
  const auto id = std::make_tuple(current_device(), key, items, GW);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  return g_tuned.count(id) > 0;
}

template <class L>
unsigned Engine::tuned_grid(const void *kern, int key, long long items, int GW, L launch) {
  const auto id = std::make_tuple(current_device(), key, items, GW);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(id);
    if (it != g_tuned.end()) {
      launch(it->second);
      return it->second;
    }
  }
  if (!tune_batch_) {
    launch((unsigned)kRedBlocks);
    return (unsigned)kRedBlocks;
  }
  int per_sm = 0, dev = 0, nsm = 0;
  MADAM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0));
  MADAM_CUDA(cudaGetDevice(&dev));
  MADAM_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  std::vector<unsigned> cand{(unsigned)kRedBlocks};
  for (int w = 1; w <= 4 && per_sm > 0; ++w) {
    const unsigned g = (unsigned)(w * per_sm * nsm);
    if (std::find(cand.begin(), cand.end(), g) == cand.end()) cand.push_back(g);
  }
  launch(cand[0]);  // warm: caches and the kernel's first load
  float best = 1e30f;
  unsigned best_g = cand[0];
  for (unsigned g : cand) {
    MADAM_CUDA(cudaEventRecord(ev_[0], st_));
    launch(g);
    MADAM_CUDA(cudaEventRecord(ev_[1], st_));
    MADAM_CUDA(cudaEventSynchronize(ev_[1]));
    float ms = 0;
    MADAM_CUDA(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
    if (ms < best) {
      best = ms;
      best_g = g;
    }
  }
  if (best_g != cand.back()) launch(best_g);  // the outputs of the chosen shape last
  if (g_trace_alloc)
    std::fprintf(stderr, "madam_b200 trace: tuned kernel %d (GW %d): grid %u, %.3f ms\n", key,
                 GW, best_g, best);
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tuned[id] = best_g;
  return best_g;
}

template <int G>
void Engine::project_group_T(long r0, int nr) {
  if (fp32_) project_group_T2<G, float>(r0, nr);
  else project_group_T2<G, double>(r0, nr);
}

template <int G, class T>
void Engine::project_group_T2(long r0, int nr) {
  // A p's projections for right-hand sides [r0, r0 + nr), nr <= 32 G, on
  // right-hand-side-minor copies (batch_kernels.inl).  T = float in the
  // FP32-TOD form: p.detw and the map the gather reads are float32.
  constexpr int GW = 32 * G;
  const long long nb = (long long)ndet_ * noba_short_;
  const long long ncross = std::max<long>(1, nloc_cross_);
  const bool f32 = std::is_same<T, float>::value;
  // grow-only: the float32 and float64 passes (reliable updates) and the
  // 32- and 64-wide groups share these buffers
  T *pwT;
  if (f32) {
    pwTf_.reserve((size_t)nb * GW);
    pwT = (T *)pwTf_.get();
    lmapTf_.reserve((size_t)ncross * nmap_ * GW);
  } else {
    pwT_.reserve((size_t)nb * GW);
    pwT = (T *)pwT_.get();
  }
  lmapT_.reserve((size_t)ncross * nmap_ * GW);
  scatpT_.reserve((size_t)std::max<size_t>(1, scatter_partial_.n / nmap_) * nmap_ * GW);
  apnT_.reserve((size_t)nb * GW);
  const unsigned tb = (unsigned)std::min<long long>(4736, (nb + 31) / 32);
  if (batch_timed_) MADAM_CUDA(cudaEventRecord(ev_[2], st_));
  MADAM_LAUNCH((k_transpose_rhs<G, T>), dim3(tb, G), 256, 0, st_, pwb_.get(), nb, (int)r0, nr,
               pwT);
  // 1) baseline -> map, combine, ccmultiply
  if (nloc_cross_ > 0 && nscatter_chunks_ > 0 && f32) {
    // FP32-TOD form: all GW right-hand sides in one pass, entry-order sums
    if (nmap_ == 3)
      tuned_grid((const void *)k_scatter_T_seq<3, GW>, 1, nscatter_chunks_, GW, [&](unsigned g) {
        MADAM_LAUNCH((k_scatter_T_seq<3, GW>), g, 256, 0, st_, scatter_chunks_.get(),
                     nscatter_chunks_, sp4_.get(), sp2_.get(), (const float *)pwT, lmapT_.get(),
                     scatpT_.get());
      });
    else
      tuned_grid((const void *)k_scatter_T_seq<1, GW>, 2, nscatter_chunks_, GW, [&](unsigned g) {
        MADAM_LAUNCH((k_scatter_T_seq<1, GW>), g, 256, 0, st_, scatter_chunks_.get(),
                     nscatter_chunks_, sp4_.get(), sp2_.get(), (const float *)pwT, lmapT_.get(),
                     scatpT_.get());
      });
  } else if (nloc_cross_ > 0 && nscatter_chunks_ > 0) {
    // one launch per 32 right-hand sides (fewer registers, more warps)
    for (int g0 = 0; g0 < GW; g0 += 32) {
      if (nmap_ == 3)
        MADAM_LAUNCH((k_scatter_T<3, GW, T>), kRedBlocks, 256, 0, st_, scatter_chunks_.get(),
                     nscatter_chunks_, sp4_.get(), sp2_.get(), (const T *)pwT, g0,
                     lmapT_.get(), scatpT_.get());
      else
        MADAM_LAUNCH((k_scatter_T<1, GW, T>), kRedBlocks, 256, 0, st_, scatter_chunks_.get(),
                     nscatter_chunks_, sp4_.get(), sp2_.get(), (const T *)pwT, g0,
                     lmapT_.get(), scatpT_.get());
    }
  }
  if (nloc_cross_ > 0 && nscatter_chunks_ > 0 && nscatter_multi_ > 0) {
    const long long tot = (long long)nscatter_multi_ * nmap_ * GW;
    if (nmap_ == 3)
      MADAM_LAUNCH((k_scatter_combine_T<3, G>), grid_for(tot), 256, 0, st_,
                   scatter_multi_.get(), nscatter_multi_, scatpT_.get(), lmapT_.get());
    else
      MADAM_LAUNCH((k_scatter_combine_T<1, G>), grid_for(tot), 256, 0, st_,
                   scatter_multi_.get(), nscatter_multi_, scatpT_.get(), lmapT_.get());
  }
  float *mf = f32 ? lmapTf_.get() : nullptr;
  if (nloc_cross_ > 0) {
    if (nmap_ == 3)
      MADAM_LAUNCH((k_ccmult_T<3, G>), grid_for((long long)nloc_cross_ * GW), 256, 0, st_,
                   cca_.get(), lmapT_.get(), (long long)nloc_cross_, mf);
    else
      MADAM_LAUNCH((k_ccmult_T<1, G>), grid_for((long long)nloc_cross_ * GW), 256, 0, st_,
                   cca_.get(), lmapT_.get(), (long long)nloc_cross_, mf);
  }
  // 3) map -> baseline sums, then ap and p.ap per right-hand side
  if (batch_timed_) MADAM_CUDA(cudaEventRecord(ev_[3], st_));
  const T *mT = f32 ? (const T *)lmapTf_.get() : (const T *)lmapT_.get();
  if (f32 && use_pairs_ && nmap_ == 3 && npair_chunks_ > 0) {
    // FP32-TOD form: over the pointing pairs (fewer map rows to read); the
    // chunks cover every baseline, so apnT is written for all of them
    tuned_grid((const void *)k_gather_T_pairs<G>, 3, npair_chunks_, GW, [&](unsigned g) {
      MADAM_LAUNCH(k_gather_T_pairs<G>, g, 256, 0, st_, pair_chunks_.get(), npair_chunks_,
                   gp4_.get(), poff_.get(), lmapTf_.get(), apnT_.get());
    });
  } else if (nmap_ == 3)
    tuned_grid((const void *)k_gather_T<3, G, T>, f32 ? 4 : 5, ngather_chunks_, GW,
               [&](unsigned g) {
                 MADAM_LAUNCH((k_gather_T<3, G, T>), g, 256, 0, st_, gather_chunks_.get(),
                              ngather_chunks_, point4_.get(), pixc_.get(), bstart_d_.get(),
                              noba_short_, nsamp_, mT, (int)ndeg_shift_, (int)nloc_,
                              apnT_.get());
               });
  else
    MADAM_LAUNCH((k_gather_T<1, G, T>), kRedBlocks, 256, 0, st_, gather_chunks_.get(),
                 ngather_chunks_, point4_.get(), pixc_.get(), bstart_d_.get(), noba_short_,
                 nsamp_, mT, (int)ndeg_shift_, (int)nloc_, apnT_.get());
  MADAM_LAUNCH(k_gather_finish_T<G>, kRedBlocks, 256, 0, st_, apnT_.get(), nb, bw_.get(),
               nna_.get(), rmask_.get(), pb_.get(), apb_.get(), (int)r0, nr, partb_.get());
  if (batch_timed_) MADAM_CUDA(cudaEventRecord(ev_[4], st_));
}

void Engine::apply_A_batch() {
  // A p for every right-hand side (iterate_a 798-878)
  const long long nb = (long long)ndet_ * noba_short_;
  const long long tstride = (long long)std::max<long>(1, nloc_cross_) * nmap_;
  const long long pstride = (long long)scatter_partial_.n;
  // noise prior ap = C_a^-1 p (cinvmul, 829-845); the projections add to it
  const long long nt = nb * nrhs_;
  if (batch_timed_) MADAM_CUDA(cudaEventRecord(ev_[0], st_));
  if (par_.kfilter) {
    MADAM_CUDA(cudaMemcpyAsync(apb_.get(), pb_.get(), nt * sizeof(double),
                               cudaMemcpyDeviceToDevice, st_));
    const long nfs = (long)filt_segs_.size() * nrhs_;
    if (nfs > 0) fft_->convolve(st_, filt_segs_b_d_.get(), nfs, fcov_.get(), npsdtot_, pb_.get(),
                                apb_.get());
  } else if (par_.diagfilter != 0) {
    for (long k = 0; k < nrhs_; ++k)
      MADAM_LAUNCH(k_diagfilter, grid_for(nb), 256, 0, st_, apb_.get() + k * nb, nna_.get(),
                   pb_.get() + k * nb, par_.diagfilter, nb);
  } else {
    MADAM_CUDA(cudaMemsetAsync(apb_.get(), 0, nt * sizeof(double), st_));
  }
  if (batch_timed_) MADAM_CUDA(cudaEventRecord(ev_[1], st_));
  if (ngather_chunks_ > 0) {
    // right-hand-side-minor projections, 64 right-hand sides a pass
    for (long r0 = 0; r0 < nrhs_; r0 += 64) {
      const int nr = (int)std::min<long>(64, nrhs_ - r0);
      if (nr > 32) project_group_T<2>(r0, nr);
      else project_group_T<1>(r0, nr);
    }
    MADAM_LAUNCH(k_finish_b, (unsigned)nrhs_, 1024, 0, st_, partb_.get(), kRedBlocks, 1,
                 scalb_.get(), 1, 0, actb_.get());
    return;
  }
  // baselines longer than a gather chunk: right-hand-side-major scatter,
  // single-RHS gathers
  if (nloc_cross_ > 0 && nscatter_chunks_ > 0) {
    for (long r0 = 0; r0 < nrhs_; r0 += kScatterGroup) {
      const int nr = (int)std::min<long>(kScatterGroup, nrhs_ - r0);
      if (nmap_ == 3)
        MADAM_LAUNCH((k_scatter_chunks_b<3, kScatterGroup>), kRedBlocks, 256, 0, st_,
                     scatter_chunks_.get(), nscatter_chunks_, sp4_.get(), sp2_.get(), pwb_.get(),
                     nb, (int)r0, nr, lmapb_.get(), tstride, scatpb_.get(), pstride);
      else
        MADAM_LAUNCH((k_scatter_chunks_b<1, kScatterGroup>), kRedBlocks, 256, 0, st_,
                     scatter_chunks_.get(), nscatter_chunks_, sp4_.get(), sp2_.get(), pwb_.get(),
                     nb, (int)r0, nr, lmapb_.get(), tstride, scatpb_.get(), pstride);
    }
    if (nscatter_multi_ > 0) {
      const dim3 g((unsigned)std::min<long long>(1184, (nscatter_multi_ + 255) / 256),
                   (unsigned)nrhs_);
      if (nmap_ == 3)
        MADAM_LAUNCH(k_scatter_combine_b<3>, g, 256, 0, st_, scatter_multi_.get(),
                     nscatter_multi_, scatpb_.get(), pstride, lmapb_.get(), tstride);
      else
        MADAM_LAUNCH(k_scatter_combine_b<1>, g, 256, 0, st_, scatter_multi_.get(),
                     nscatter_multi_, scatpb_.get(), pstride, lmapb_.get(), tstride);
    }
  }
  if (nloc_cross_ > 0) {
    const dim3 g((unsigned)std::min<long long>(1184, (nloc_cross_ + 255) / 256),
                 (unsigned)nrhs_);
    if (nmap_ == 3)
      MADAM_LAUNCH(k_ccmult_b<3>, g, 256, 0, st_, cca_.get(), lmapb_.get(),
                   (long long)nloc_cross_);
    else
      MADAM_LAUNCH(k_ccmult_b<1>, g, 256, 0, st_, cca_.get(), lmapb_.get(),
                   (long long)nloc_cross_);
  }
  for (long k = 0; k < nrhs_; ++k) {
    double *pk = pb_.get() + k * nb, *apk = apb_.get() + k * nb;
    double *mk = lmapb_.get() + k * tstride, *partk = partb_.get() + k * 3 * kRedBlocks;
    if (gather_kb_ > 0) {
      if (nmap_ == 3)
        MADAM_LAUNCH(k_gather_tiled<3>, kRedBlocks, 256, 0, st_, point4_.get(), pixc_.get(),
                     bstart_d_.get(), noba_short_, nsamp_, gather_kb_, gather_tiles_det_,
                     (int)ndet_, bw_.get(), pk, nna_.get(), mk, (int)ndeg_shift_, (int)nloc_,
                     rmask_.get(), apk, partk);
      else
        MADAM_LAUNCH(k_gather_tiled<1>, kRedBlocks, 256, 0, st_, point4_.get(), pixc_.get(),
                     bstart_d_.get(), noba_short_, nsamp_, gather_kb_, gather_tiles_det_,
                     (int)ndet_, bw_.get(), pk, nna_.get(), mk, (int)ndeg_shift_, (int)nloc_,
                     rmask_.get(), apk, partk);
    } else if (nmap_ == 3) {
      MADAM_LAUNCH(k_gather<3>, kRedBlocks, 256, 0, st_, point4_.get(), pixc_.get(),
                   bstart_d_.get(), nb, noba_short_, nsamp_, bw_.get(), pk, nna_.get(), mk,
                   (int)ndeg_shift_, (int)nloc_, rmask_.get(), apk, partk);
    } else {
      MADAM_LAUNCH(k_gather<1>, kRedBlocks, 256, 0, st_, point4_.get(), pixc_.get(),
                   bstart_d_.get(), nb, noba_short_, nsamp_, bw_.get(), pk, nna_.get(), mk,
                   (int)ndeg_shift_, (int)nloc_, rmask_.get(), apk, partk);
    }
  }
  MADAM_LAUNCH(k_finish_b, (unsigned)nrhs_, 1024, 0, st_, partb_.get(), kRedBlocks, 1,
               scalb_.get(), 1, 0, actb_.get());
}

// The true residuals r_k = y_k - A aa_k of the right-hand sides in upd (the
// FP32-TOD batch's reliable updates) in one float64 pass: their aa rows go
// through apply_A_batch as a batch of their own, with the pixel-sorted
// samples in the scatter and float64 projections (the arithmetic of the
// single solve's exact operator, apply_A_exact), instead of one single-RHS
// operator per right-hand side.
template <class B>
static void swap_buf(B &a, B &b) {
  std::swap(a.p, b.p);
  std::swap(a.n, b.n);
}

void Engine::true_residual_batch(const std::vector<long> &upd) {
  const long long nb = (long long)ndet_ * noba_short_;
  const long ns = (long)upd.size();
  xsb_.reserve((size_t)ns * nb);
  pwsb_.reserve((size_t)ns * nb);
  apsb_.reserve((size_t)ns * nb);
  partsb_.reserve((size_t)ns * 3 * kRedBlocks);
  scalsb_.reserve((size_t)ns * S_NSCAL);
  scalsb_.zero(st_);
  actsb_.reserve(ns);
  std::vector<int> one(ns, 1);
  MADAM_CUDA(cudaMemcpyAsync(actsb_.get(), one.data(), ns * sizeof(int), cudaMemcpyHostToDevice,
                             st_));
  for (long i = 0; i < ns; ++i) {
    MADAM_CUDA(cudaMemcpyAsync(xsb_.get() + i * nb, aab_.get() + upd[i] * nb,
                               nb * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    MADAM_LAUNCH(k_mul, grid_for(nb), 256, 0, st_, pwsb_.get() + i * nb, xsb_.get() + i * nb,
                 bw_.get(), nb);
  }
  auto swap_all = [&]() {
    swap_buf(pb_, xsb_);
    swap_buf(pwb_, pwsb_);
    swap_buf(apb_, apsb_);
    swap_buf(partb_, partsb_);
    swap_buf(scalb_, scalsb_);
    swap_buf(actb_, actsb_);
    if (have_xcsr_) swap_csr();
    std::swap(nrhs_, nrhs_alt_);
  };
  nrhs_alt_ = ns;
  const bool f32 = fp32_, timed = batch_timed_;
  fp32_ = false;
  batch_timed_ = false;
  swap_all();
  try {
    apply_A_batch();
  } catch (...) {
    swap_all();
    fp32_ = f32;
    batch_timed_ = timed;
    throw;
  }
  swap_all();
  fp32_ = f32;
  batch_timed_ = timed;
  for (long i = 0; i < ns; ++i) {
    MADAM_LAUNCH(k_residual, grid_for(nb), 256, 0, st_, rb_.get() + upd[i] * nb,
                 yb_.get() + upd[i] * nb, apsb_.get() + i * nb, nb);
    ++n_reliable_;
  }
}

void Engine::iterate_batch() {
  // iterate_a (smadam_routines.f90:677-983) for every right-hand side
  double t0 = now_ms();
  const long long nb = (long long)ndet_ * noba_short_;
  const long long nt = nb * nrhs_;
  const long R = nrhs_;
  for (auto *b : {&rb_, &pb_, &zb_, &apb_, &rob_, &pwb_, &aab_}) b->alloc(nt);
  partb_.alloc((size_t)R * 3 * kRedBlocks);
  scalb_.alloc((size_t)R * S_NSCAL);
  scalb_.zero(st_);
  actb_.alloc(R);
  actu_.alloc(R);
  lmapb_.alloc((size_t)R * std::max<long>(1, nloc_cross_) * nmap_);
  scatpb_.alloc((size_t)R * std::max<size_t>(1, scatter_partial_.n));
  build_batch_tables();
  act_host_.assign(R, 1);
  auto upload_act = [&]() {
    MADAM_CUDA(cudaMemcpyAsync(actb_.get(), act_host_.data(), R * sizeof(int),
                               cudaMemcpyHostToDevice, st_));
  };
  upload_act();
  noiter_b_.assign(R, 0.0);
  rrinit_b_.assign(R, 0.0);
  rrfinal_b_.assign(R, 1.0);
  MADAM_CUDA(cudaMemcpyAsync(rb_.get(), yb_.get(), nt * sizeof(double), cudaMemcpyDeviceToDevice,
                             st_));
  aab_.zero(st_);
  apply_preconditioner_batch(rb_.get(), zb_.get());
  const dim3 gv((unsigned)std::min<long long>(4736, (nb + 255) / 256), (unsigned)R);
  const dim3 gd(kRedBlocks, (unsigned)R);
  MADAM_LAUNCH(k_update_p_b, gv, 256, 0, st_, pb_.get(), zb_.get(), pwb_.get(), bw_.get(), nb,
               scalb_.get(), 1, actb_.get());
  MADAM_LAUNCH(k_dots_b, gd, 256, 0, st_, rb_.get(), zb_.get(), rb_.get(), rb_.get(), nullptr,
               nullptr, 2, rmask_.get(), nb, actb_.get(), partb_.get());
  MADAM_LAUNCH(k_finish_b, (unsigned)R, 1024, 0, st_, partb_.get(), kRedBlocks, 2, scalb_.get(),
               0, S_RZ, actb_.get());
  std::vector<double> sc((size_t)R * S_NSCAL);
  auto fetch = [&]() {
    MADAM_CUDA(cudaMemcpyAsync(sc.data(), scalb_.get(), sc.size() * sizeof(double),
                               cudaMemcpyDeviceToHost, st_));
    MADAM_CUDA(cudaStreamSynchronize(st_));
  };
  fetch();
  long nact = 0;
  for (long k = 0; k < R; ++k) {
    const double rzinit = sc[k * S_NSCAL + S_RZ];
    rrinit_b_[k] = sc[k * S_NSCAL + S_RR];
    if (rzinit < fsp(1e-30f) || std::isnan(rzinit)) act_host_[k] = 0;
    nact += act_host_[k];
  }
  upload_act();
  // launch shapes of the batched projections, tuned once per shape on this
  // batch's data before the iterations (apply_A_batch's outputs are
  // overwritten by the first iteration); counted in the setup time
  if (ngather_chunks_ > 0) {
    const double tt = now_ms();
    tune_batch_ = true;
    try {
      apply_A_batch();
    } catch (...) {
      tune_batch_ = false;
      throw;
    }
    tune_batch_ = false;
    if (fp32_) {
      // the float64 pass of the reliable updates: its buffers now, so that
      // the iterations do not allocate
      const long long ncr = std::max<long>(1, nloc_cross_);
      const size_t xpart = have_xcsr_ ? xscatter_partial_.n : scatter_partial_.n;
      for (auto *b : {&xsb_, &pwsb_, &apsb_}) b->reserve((size_t)R * nb);
      partsb_.reserve((size_t)R * 3 * kRedBlocks);
      scalsb_.reserve((size_t)R * S_NSCAL);
      actsb_.reserve(R);
      pwT_.reserve((size_t)nb * 64);
      lmapT_.reserve((size_t)ncr * nmap_ * 64);
      scatpT_.reserve(std::max<size_t>(1, xpart / nmap_) * nmap_ * 64);
      apnT_.reserve((size_t)nb * 64);
    }
    MADAM_CUDA(cudaStreamSynchronize(st_));
    timings.setup_ms += now_ms() - tt;
    t0 += now_ms() - tt;
  }
  // FP32-TOD batch: reliable updates per right-hand side (see iterate())
  const bool refine_b = fp32_;
  std::vector<double> rr_true(rrinit_b_);
  n_reliable_ = 0;
  long istep = 0;
  // phase times (CUDA events; the projections' of the last 64-RHS group when
  // there are several)
  batch_timed_ = ngather_chunks_ > 0 && nrhs_ <= 64;
  while (istep < par_.iter_max && nact > 0) {
    ++istep;
    apply_A_batch();
    MADAM_LAUNCH(k_update_ar_b, gv, 256, 0, st_, aab_.get(), rb_.get(), rob_.get(), pb_.get(),
                 apb_.get(), nb, scalb_.get(), actb_.get());
    if (batch_timed_) MADAM_CUDA(cudaEventRecord(ev_[5], st_));
    apply_preconditioner_batch(rb_.get(), zb_.get());
    if (batch_timed_) MADAM_CUDA(cudaEventRecord(ev_[6], st_));
    MADAM_LAUNCH(k_dots_b, gd, 256, 0, st_, rb_.get(), zb_.get(), rob_.get(), zb_.get(),
                 rb_.get(), rb_.get(), 3, rmask_.get(), nb, actb_.get(), partb_.get());
    MADAM_LAUNCH(k_finish_b, (unsigned)R, 1024, 0, st_, partb_.get(), kRedBlocks, 3,
                 scalb_.get(), 2, 0, actb_.get());
    fetch();
    if (batch_timed_) {
      float tm[4];
      MADAM_CUDA(cudaEventElapsedTime(&tm[0], ev_[0], ev_[1]));
      MADAM_CUDA(cudaEventElapsedTime(&tm[1], ev_[2], ev_[3]));
      MADAM_CUDA(cudaEventElapsedTime(&tm[2], ev_[3], ev_[4]));
      MADAM_CUDA(cudaEventElapsedTime(&tm[3], ev_[5], ev_[6]));
      timings.filter_ms += tm[0];
      timings.scatter_ms += tm[1];
      timings.gather_ms += tm[2];
      timings.precond_ms += tm[3];
    }
    if (refine_b) {
      const double tr0 = now_ms();
      std::vector<long> upd;
      for (long k = 0; k < R; ++k) {
        if (!act_host_[k]) continue;
        const double rr = sc[k * S_NSCAL + S_RR];
        if ((rr / rrinit_b_[k] < par_.cglimit && istep > par_.iter_min) ||
            rr < kReliableDrop * rr_true[k])
          upd.push_back(k);
      }
      if (!upd.empty()) {
        // the true residuals of those right-hand sides, their z (the
        // single-solve preconditioner on their slices), and rz, rz2 and rr
        // of those alone (mode 3 keeps rz_old)
        std::vector<int> mask(R, 0);
        const double ta = now_ms();
        if (upd.size() >= 4 && ngather_chunks_ > 0) {
          true_residual_batch(upd);
        } else {
          for (long k : upd)
            true_residual(aab_.get() + k * nb, yb_.get() + k * nb, rb_.get() + k * nb);
        }
        if (g_trace_alloc) MADAM_CUDA(cudaStreamSynchronize(st_));
        const double tb = now_ms();
        for (long k : upd) {
          apply_preconditioner(rb_.get() + k * nb, zb_.get() + k * nb);
          mask[k] = 1;
        }
        if (g_trace_alloc) {
          MADAM_CUDA(cudaStreamSynchronize(st_));
          std::fprintf(stderr,
                       "madam_b200 trace: iteration %ld reliable update of %zu: residual "
                       "%.2f ms, preconditioner %.2f ms\n",
                       istep, upd.size(), tb - ta, now_ms() - tb);
        }
        MADAM_CUDA(cudaMemcpyAsync(actu_.get(), mask.data(), R * sizeof(int),
                                   cudaMemcpyHostToDevice, st_));
        MADAM_LAUNCH(k_dots_b, gd, 256, 0, st_, rb_.get(), zb_.get(), rob_.get(), zb_.get(),
                     rb_.get(), rb_.get(), 3, rmask_.get(), nb, actu_.get(), partb_.get());
        MADAM_LAUNCH(k_finish_b, (unsigned)R, 1024, 0, st_, partb_.get(), kRedBlocks, 3,
                     scalb_.get(), 3, 0, actu_.get());
        fetch();
        for (long k : upd) rr_true[k] = sc[k * S_NSCAL + S_RR];
      }
      timings.other_ms += now_ms() - tr0;  // the reliable updates
    }
    bool changed = false;
    for (long k = 0; k < R; ++k) {
      if (!act_host_[k]) continue;
      const double rz = sc[k * S_NSCAL + S_RZ], rr = sc[k * S_NSCAL + S_RR];
      rrfinal_b_[k] = rr / rrinit_b_[k];
      noiter_b_[k] = (double)istep;
      if (rr / rrinit_b_[k] > 1e3)
        fail("CG is diverging (Monte Carlo realisation " + std::to_string(k) + ")");
      if ((rr / rrinit_b_[k] < par_.cglimit && istep > par_.iter_min) || rz == 0) {
        act_host_[k] = 0;
        --nact;
        changed = true;
      }
    }
    if (changed) upload_act();
    if (nact == 0) break;
    MADAM_LAUNCH(k_update_p_b, gv, 256, 0, st_, pb_.get(), zb_.get(), pwb_.get(), bw_.get(), nb,
                 scalb_.get(), 0, actb_.get());
  }
  MADAM_CUDA(cudaStreamSynchronize(st_));
  batch_timed_ = false;
  check_band_err();
  timings.iterate_ms = now_ms() - t0;
}

void Engine::run_cached_batch(long ndet, long nsamp, long nnz, double *timestamps, int32_t *pix,
                              float *pixweights, long nrhs, double *signals, bool is_device,
                              bool fp32) {
  g_alloc_stream = st_;
  if (!cached_) fail("destripe_with_cache called with empty caches.");
  if (nrhs < 1) fail("nrhs must be at least 1");
  if (sharded()) fail("the batched solve runs on one rank");
  if (nbasis_ > 1) fail("the batched solve takes basis_order 0");
  if (par_.temperature_only && nnz != 1)
    fail("temperature_only=T but pointing weights are polarized");
  if (ndet != ndet_ || nsamp != nsamp_ || nnz != nnz_)
    fail("destripe_with_cache: data shape differs from the cached call");
  const double t0 = now_ms();
  timings = Timings();
  rr_history.clear();
  noiter = 0;
  const long long n = (long long)ndet * nsamp;
  const long long nb = (long long)ndet_ * noba_short_;
  nrhs_ = nrhs;
  // pointing-side setup, once; fp32: float32 signals and projections (the
  // FP32-TOD form), which also compresses the scatter's pointing into pairs
  fp32_ = fp32;
  fp32_next_ = false;
  d_pix_caller_ = is_device ? pix : nullptr;
  bind_inputs(timestamps, pix, pixweights, signals, is_device, false);
  wait_tod();  // the realisations are copied on the engine stream below
  flag_and_compact(false);
  build_runs();
  if (par_.kfirst) build_csr();
  // the cached state every realisation starts from
  DevBuf<double> wamap0;
  wamap0.alloc(wamap_.n);
  if (wamap_.n)
    MADAM_CUDA(cudaMemcpyAsync(wamap0.get(), wamap_.get(), wamap_.n * sizeof(double),
                               cudaMemcpyDeviceToDevice, st_));
  const long long nv = (long long)nloc_ * nmap_;
  yb_.alloc((size_t)nrhs * nb);
  binb_.alloc((size_t)nrhs * std::max<long long>(1, nv));
  mapb_.alloc((size_t)nrhs * std::max<long long>(1, nv));
  binmapb_.alloc((size_t)nrhs * std::max<long long>(1, nv));
  DevBuf<float> t32;
  auto select_tod = [&](long k) {
    if (fp32) {
      float *src = (float *)signals + k * n;
      sig32_caller_ = src;
      const float *dsrc = src;
      if (!is_device) {
        t32.alloc(n);
        MADAM_CUDA(cudaMemcpyAsync(t32.get(), src, n * sizeof(float), cudaMemcpyHostToDevice,
                                   st_));
        dsrc = t32.get();
      }
      if (n > 0) MADAM_LAUNCH(k_f32_to_f64, grid_for(n), 256, 0, st_, dsrc, tod_own_.get(), n);
      d_tod_ = tod_own_.get();
      return;
    }
    if (is_device) {
      d_tod_ = signals + k * n;
    } else {
      MADAM_CUDA(cudaMemcpyAsync(tod_own_.get(), signals + k * n, n * sizeof(double),
                                 cudaMemcpyHostToDevice, st_));
      d_tod_ = tod_own_.get();
      h_signal_ = signals + k * n;
    }
  };
  // per realisation: binned map and right-hand side (bin_tod, initialize_a)
  for (long k = 0; k < nrhs; ++k) {
    select_tod(k);
    if (wamap_.n)
      MADAM_CUDA(cudaMemcpyAsync(wamap_.get(), wamap0.get(), wamap_.n * sizeof(double),
                                 cudaMemcpyDeviceToDevice, st_));
    bin_tod(true);
    if (nv)
      MADAM_CUDA(cudaMemcpyAsync(binb_.get() + k * nv, map_.get(), nv * sizeof(double),
                                 cudaMemcpyDeviceToDevice, st_));
    if (par_.kfirst) {
      std::vector<Segment> old = segs_;
      initialize_a();
      if (k == 0) {
        build_segments();
        bool same = old.size() == segs_.size();
        for (size_t i = 0; same && i < old.size(); ++i)
          same = old[i].k0 == segs_[i].k0 && old[i].noba == segs_[i].noba;
        if (!same) fail("destripe_with_cache: flagging differs from the cached call");
      }
      if (nb)
        MADAM_CUDA(cudaMemcpyAsync(yb_.get() + k * nb, yba_.get(), nb * sizeof(double),
                                   cudaMemcpyDeviceToDevice, st_));
    }
  }
  MADAM_CUDA(cudaStreamSynchronize(st_));
  timings.setup_ms = now_ms() - t0;
  if (par_.kfirst) iterate_batch();
  else {
    noiter_b_.assign(nrhs, 0.0);
    rrinit_b_.assign(nrhs, 0.0);
    rrfinal_b_.assign(nrhs, 0.0);
    aab_.alloc((size_t)nrhs * nb);
    aab_.zero(st_);
  }
  // per realisation: destriped and binned maps (subtract_baselines_a,
  // makemaps), optional TOD cleaning; no files
  const double tf = now_ms();
  suppress_fits_ = true;
  try {
    for (long k = 0; k < nrhs; ++k) {
      select_tod(k);
      tod_cleaned_ = false;
      if (nb)
        MADAM_CUDA(cudaMemcpyAsync(aa_.get(), aab_.get() + k * nb, nb * sizeof(double),
                                   cudaMemcpyDeviceToDevice, st_));
      if (nv) {
        MADAM_CUDA(cudaMemcpyAsync(map_.get(), binb_.get() + k * nv, nv * sizeof(double),
                                   cudaMemcpyDeviceToDevice, st_));
        MADAM_CUDA(cudaMemcpyAsync(binmap_.get(), binb_.get() + k * nv, nv * sizeof(double),
                                   cudaMemcpyDeviceToDevice, st_));
      }
      finalize(false);
      if (nv) {
        MADAM_CUDA(cudaMemcpyAsync(mapb_.get() + k * nv, map_.get(), nv * sizeof(double),
                                   cudaMemcpyDeviceToDevice, st_));
        MADAM_CUDA(cudaMemcpyAsync(binmapb_.get() + k * nv, binmap_.get(), nv * sizeof(double),
                                   cudaMemcpyDeviceToDevice, st_));
      }
    }
  } catch (...) {
    suppress_fits_ = false;
    throw;
  }
  suppress_fits_ = false;
  // leave the cache as it was
  if (wamap_.n)
    MADAM_CUDA(cudaMemcpyAsync(wamap_.get(), wamap0.get(), wamap_.n * sizeof(double),
                               cudaMemcpyDeviceToDevice, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  noiter = (long)*std::max_element(noiter_b_.begin(), noiter_b_.end());
  timings.finalize_ms = now_ms() - tf;
  timings.total_ms = now_ms() - t0;
}
