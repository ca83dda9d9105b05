// Engine methods: host orchestration of the destriping solve.  Included at
// the end of engine.cu so the kernels there are visible.

// Work vectors of the CG fallback preconditioner.
struct CgpWork {
  DevBuf<CgpSeg> segs;
  DevBuf<double> x, resid, prop, aprop, zres, prec, st;
  DevBuf<int> done, active;
  DevBuf<ConvSeg> csegs;
  std::vector<ConvSeg> hcsegs;
  long nseg = 0;
};

thread_local cudaStream_t g_alloc_stream = nullptr;

// allocations and frees that take longer than a millisecond of host time
// are reported with MADAM_B200_TRACE set
static const bool g_trace_alloc = std::getenv("MADAM_B200_TRACE") != nullptr;

void *dev_alloc(size_t bytes) {
  void *p = nullptr;
  const double t0 = g_trace_alloc ? now_ms() : 0;
  MADAM_CUDA(cudaMallocAsync(&p, bytes, g_alloc_stream));
  if (g_trace_alloc && now_ms() - t0 > 1.0)
    std::fprintf(stderr, "madam_b200 trace: slow alloc of %.3f GB: %.3f ms\n", bytes / 1e9,
                 now_ms() - t0);
  return p;
}

void dev_free(void *p) {
  const double t0 = g_trace_alloc ? now_ms() : 0;
  cudaFreeAsync(p, g_alloc_stream);
  if (g_trace_alloc && now_ms() - t0 > 1.0)
    std::fprintf(stderr, "madam_b200 trace: slow free: %.3f ms\n", now_ms() - t0);
}

Engine::Engine() {
  MADAM_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
  {
    int dev = 0;
    MADAM_CUDA(cudaGetDevice(&dev));
    cudaMemPool_t pool;
    MADAM_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t keep = UINT64_MAX;
    MADAM_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  g_alloc_stream = st_;
  for (auto &e : ev_) MADAM_CUDA(cudaEventCreate(&e));
  MADAM_CUDA(cudaStreamCreateWithFlags(&cst_, cudaStreamNonBlocking));
  MADAM_CUDA(cudaEventCreateWithFlags(&ev_ptr_, cudaEventDisableTiming));
  MADAM_CUDA(cudaEventCreateWithFlags(&ev_tod_, cudaEventDisableTiming));
}

void Engine::wait_tod() {
  if (!tod_pending_) return;
  MADAM_CUDA(cudaStreamWaitEvent(st_, ev_tod_, 0));
  tod_pending_ = false;
}

void Engine::sync_tod() {
  // a call that fails before it reads the signal still waits for the copy
  // from the caller's buffer
  if (!tod_pending_) return;
  cudaStreamSynchronize(cst_);
  cudaStreamWaitEvent(st_, ev_tod_, 0);
  tod_pending_ = false;
}

Engine::~Engine() {
  // members free their memory after this body: order those frees on the
  // legacy stream once the engine's streams are idle
  if (cst_) cudaStreamSynchronize(cst_);
  cudaStreamSynchronize(st_);
  g_alloc_stream = nullptr;
  for (auto &e : ev_) cudaEventDestroy(e);
  for (auto &e : trace_ev_)
    if (e) cudaEventDestroy(e);
  if (ev_ptr_) cudaEventDestroy(ev_ptr_);
  if (ev_tod_) cudaEventDestroy(ev_tod_);
  if (cst_) cudaStreamDestroy(cst_);
  if (st_) cudaStreamDestroy(st_);
}


static SampleMap sample_map(const long long *istart, const int *kstart, int niv,
                            long long nsamp, long noba, FastDiv fdn) {
  SampleMap m;
  m.istart = istart;
  m.kstart = kstart;
  m.ninterval = niv;
  m.nsamp = nsamp;
  m.noba_short = noba;
  m.fdn = fdn;
  return m;
}

void Engine::bind_inputs(double *timestamps, int32_t *pix, float *pixweights, double *signal,
                         bool is_device, bool first_call) {
  (void)first_call;
  (void)timestamps;
  const long long n = (long long)ndet_ * nsamp_;
  sync_tod();
  in_device_ = is_device;
  h_pix_ = is_device ? nullptr : pix;
  h_signal_ = is_device ? nullptr : signal;
  const cudaMemcpyKind kind = is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  pix_.alloc(n);
  pix_orig_.alloc(n);
  MADAM_CUDA(cudaMemcpyAsync(pix_orig_.get(), pix, n * sizeof(int32_t), kind, st_));
  MADAM_CUDA(cudaMemcpyAsync(pix_.get(), pix_orig_.get(), n * sizeof(int32_t),
                             cudaMemcpyDeviceToDevice, st_));
  if (fp32_) {
    // FP32-TOD form: float32 samples, widened once into the engine's copy
    sig32_caller_ = (float *)signal;
    h_signal_ = nullptr;
    if (is_device) {
      d_w_ = pixweights;
    } else {
      wraw_.alloc(n * nnz_);
      MADAM_CUDA(cudaMemcpyAsync(wraw_.get(), pixweights, n * nnz_ * sizeof(float),
                                 cudaMemcpyHostToDevice, st_));
      d_w_ = wraw_.get();
    }
    tod_own_.alloc(n);
    const float *src = (const float *)signal;
    DevBuf<float> t32;
    if (!is_device) {
      t32.alloc(n);
      MADAM_CUDA(cudaMemcpyAsync(t32.get(), signal, n * sizeof(float), cudaMemcpyHostToDevice,
                                 st_));
      src = t32.get();
    }
    if (n > 0) MADAM_LAUNCH(k_f32_to_f64, grid_for(n), 256, 0, st_, src, tod_own_.get(), n);
    d_tod_ = tod_own_.get();
    return;
  }
  sig32_caller_ = nullptr;
  if (is_device) {
    d_w_ = pixweights;
    d_tod_ = signal;
  } else {
    wraw_.alloc(n * nnz_);
    MADAM_CUDA(cudaMemcpyAsync(wraw_.get(), pixweights, n * nnz_ * sizeof(float),
                               cudaMemcpyHostToDevice, st_));
    d_w_ = wraw_.get();
    tod_own_.alloc(n);
    d_tod_ = tod_own_.get();
    // the signal is first read by the binning: its upload follows the
    // pointing's on the copy stream while the engine stream flags, compacts
    // and sorts the pointing
    if (n > 0) {
      MADAM_CUDA(cudaEventRecord(ev_ptr_, st_));
      MADAM_CUDA(cudaStreamWaitEvent(cst_, ev_ptr_, 0));
      // a page-locked buffer is read by a kernel (the copy engine would
      // queue the setup's small transfers behind this one), a pageable one
      // goes through the copy engine
      // the kernel reads all n values through the device alias, so the
      // last one must lie in the same page-locked, mapped range (a buffer
      // registered only in part goes through the copy engine instead)
      cudaPointerAttributes pa{}, pz{};
      bool mapped = cudaPointerGetAttributes(&pa, signal) == cudaSuccess &&
                    pa.type == cudaMemoryTypeHost && pa.devicePointer != nullptr &&
                    ((uintptr_t)pa.devicePointer % 16) == 0;
      cudaGetLastError();
      if (mapped) {
        const double *last = (const double *)signal + (n - 1);
        mapped = cudaPointerGetAttributes(&pz, last) == cudaSuccess &&
                 pz.type == cudaMemoryTypeHost && pz.devicePointer != nullptr &&
                 (const char *)pz.devicePointer ==
                     (const char *)pa.devicePointer + (n - 1) * sizeof(double);
        cudaGetLastError();
      }
      if (mapped)
        // one small CTA per SM: the bus, not the SMs, limits it, and the
        // setup kernels beside it keep their warp slots
        MADAM_LAUNCH(k_fetch_host, 148, 128, 0, cst_, (const double *)pa.devicePointer,
                     tod_own_.get(), n);
      else
        MADAM_CUDA(cudaMemcpyAsync(tod_own_.get(), signal, n * sizeof(double),
                                   cudaMemcpyHostToDevice, cst_));
      MADAM_CUDA(cudaEventRecord(ev_tod_, cst_));
      tod_pending_ = true;
    }
  }
}

void Engine::init_layout(long nperiod, const long *periods) {
  Params &p = par_;
  // check_files: interval lengths (read_data.f90:221-239)
  ninterval_ = nperiod;
  if (nperiod <= 0) fail("ERROR: intervals not known.");
  intervals_.assign(nperiod, 0);
  for (long ip = 0; ip < nperiod; ++ip) {
    const long len = (ip < nperiod - 1) ? periods[ip + 1] - periods[ip] : nsamp_ - periods[ip];
    if (p.basis_order > 0 && len < p.basis_order + 1) fail("Too short period");
    intervals_[ip] = len;
  }
  // init_parameters (parameter_control.f90:27-409)
  if (!p.radiometers) {
    for (auto &d : dets_)
      for (int ip = 0; ip < d.npsd && d.has_psd; ++ip) {
        auto &psd = d.psds[ip];
        size_t im = 0;
        for (size_t i = 1; i < psd.size(); ++i)
          if (psd[i] > psd[im]) im = i;
        for (size_t i = 0; i < im; ++i) psd[i] = psd[im];
      }
  }
  if (p.noise_weights_from_psd) {
    // measure_noise_weights (noise_routines.f90:65-127)
    const double fs = p.fsample;
    if (p.radiometers) {
      const double f = fs / 2;
      for (auto &d : dets_)
        for (int i = 0; i < d.npsd; ++i) {
          double v;
          interpolate_psd(d.psdfreqs, d.psds[i], &f, &v, 1);
          d.sigmas[i] = std::sqrt(v * fs);
          d.plateaus[i] = v;
        }
    } else {
      const long nbin = 10000;
      const double fstep = fs * .5 / nbin;
      std::vector<double> fr(nbin), dv(nbin);
      for (long i = 0; i < nbin; ++i) fr[i] = fstep * (i + 1);
      const double fbase = 1 / (p.dnshort / fs);
      const long ibase = (long)(fbase / fstep);
      const long ilo = (long)(1 / fstep), ihi = (long)(10 / fstep);
      for (auto &d : dets_)
        for (int ip = 0; ip < d.npsd; ++ip) {
          interpolate_psd(d.psdfreqs, d.psds[ip], fr.data(), dv.data(), nbin);
          double plateau = dv[ilo - 1];
          for (long i = ilo - 1; i <= ihi - 1; ++i) plateau = std::min(plateau, dv[i]);
          double rms = ibase * plateau;
          for (long i = ibase; i < nbin; ++i) rms += dv[i];
          d.sigmas[ip] = std::sqrt(rms / nbin * fs);
          d.plateaus[ip] = plateau;
          d.weights[ip] = 1 / (plateau * fs);
        }
    }
  }
  if (p.nsubchunk < 2) {
    p.nsubchunk = 0;
    p.isubchunk = 0;
  }
  if (p.isubchunk > p.nsubchunk) fail("ERROR: isubchunk > nsubchunk");
  // parameter_control.f90:128-131
  if (!p.file_covmat.empty()) {
    p.kfilter = true;
    p.kfirst = true;
    if (p.nsubchunk > 0) fail("file_covmat with nsubchunk > 1 is not supported");
  }
  if (p.good_baseline_fraction < 0 || p.good_baseline_fraction > 1)
    fail("ERROR: good_baseline_fraction must be in 0..1");
  if (p.nside_cross < 0) p.nside_cross = p.nside_map;
  auto pow2 = [](long v) { return v > 0 && (v & (v - 1)) == 0; };
  if (!pow2(p.nside_map)) fail("nside_map must be a power of two.");
  if (!pow2(p.nside_submap)) fail("nside_submap must be a power of two.");
  if (!pow2(p.nside_cross)) fail("nside_cross must be a power of two.");
  if (p.nside_map < p.nside_cross) fail("nside_cross > nside_map not supported by Madam/TOAST");
  if (p.pixlim_cross < 0) p.pixlim_cross = p.pixlim_map;
  if (p.pixmode_map < 0 || p.pixmode_map > 2) fail("Pixmode_map must be in range [0-2]");
  if (p.pixmode_cross < 0 || p.pixmode_cross > 4) fail("Pixmode_cross must be in range [0-4]");
  if (nmap_ == 1) p.temperature_only = true;
  else if (p.temperature_only) nmap_ = 1;
  if (nmap_ != 1 && nmap_ != 3) fail("only nnz = 1 or nnz = 3 is supported");
  if (p.mode_detweight == 0) {
    for (auto &d : dets_)
      for (int i = 0; i < d.npsd; ++i)
        d.weights[i] = (d.sigmas[i] == 0) ? 0 : 1.0 / d.plateaus[i] / p.fsample;
  } else if (p.mode_detweight == 1) {
    for (auto &d : dets_) std::fill(d.weights.begin(), d.weights.end(), 1.0);
  } else if (p.mode_detweight == 2) {
    auto horn = [](const std::string &nm) -> long {
      std::string s = nm.compare(0, 3, "LFI") == 0 ? nm.substr(3, 2)
                                                    : (nm.size() > 4 ? nm.substr(4, 1) : "");
      char *end = nullptr;
      const long h = std::strtol(s.c_str(), &end, 10);
      if (s.empty() || !end || *end != '\0') fail("ERROR : Failed to extract horn from " + nm);
      return h;
    };
    for (size_t a = 0; a + 1 < dets_.size(); ++a) {
      const long h1 = horn(dets_[a].name);
      for (size_t b = a + 1; b < dets_.size(); ++b) {
        if (horn(dets_[b].name) != h1) continue;
        auto &d1 = dets_[a];
        auto &d2 = dets_[b];
        if (d1.npsd != d2.npsd)
          fail("Detectors in the same horn do not have the same number of PSDs");
        std::vector<double> w(d1.npsd);
        for (int i = 0; i < d1.npsd; ++i)
          w[i] = (d1.plateaus[i] == 0 || d2.plateaus[i] == 0)
                     ? 0
                     : 2 / (d1.plateaus[i] + d2.plateaus[i]) / p.fsample;
        d1.weights = w;
        d2.weights = w;
      }
    }
  } else {
    fail("bad mode_detweight");
  }
  nside_max_ = std::max(p.nside_map, p.nside_cross);
  p.nside_submap = std::min({p.nside_submap, p.nside_map, p.nside_cross});
  nosubmaps_tot_ = 12 * p.nside_submap * p.nside_submap;
  nshort_ = (long)(p.dnshort + .5);
  if (!p.kfirst) {
    p.dnshort = 1e6;
    nshort_ = (long)(p.dnshort + .5);
    p.precond_width_min = 0;
    p.precond_width_max = 0;
    p.kfilter = false;
  } else {
    p.precond_width_max = std::max(p.precond_width_min, p.precond_width_max);
  }
  if (p.basis_order > 0 && p.kfilter) fail("Filter only implemented for basis_order==0");
  nbasis_ = (int)p.basis_order + 1;
  if (nbasis_ > kMaxBasis)
    fail("basis_order above " + std::to_string(kMaxBasis - 1) + " is not supported");
  if (nbasis_ > 1 && fp32_) fail("the float32 TOD form takes basis_order 0");
  dnshort_ = p.dnshort;
  noba_pp_.assign(ninterval_, 0);
  kstart_pp_.assign(ninterval_ + 1, 0);
  istart_iv_.assign(ninterval_ + 1, 0);
  noba_short_ = 0;
  long long acc = 0;
  for (long i = 0; i < ninterval_; ++i) {
    if (intervals_[i] <= 0) fail("empty pointing period");
    noba_pp_[i] = (long)((double)(intervals_[i] - 1) / dnshort_) + 1;
    kstart_pp_[i] = noba_short_;
    istart_iv_[i] = acc;
    noba_short_ += noba_pp_[i];
    acc += intervals_[i];
  }
  kstart_pp_[ninterval_] = noba_short_;
  istart_iv_[ninterval_] = acc;
  if (acc != nsamp_) fail("pointing periods do not cover the samples");
  if ((long long)ndet_ * noba_short_ >= (1LL << 31)) fail("too many baselines");
  if (nsamp_ >= (1LL << 32) - 1) fail("too many samples per detector");
  const long nsm = p.nside_submap;
  nosubpix_max_ = nside_max_ * nside_max_ / (nsm * nsm);
  nosubpix_map_ = p.nside_map * p.nside_map / (nsm * nsm);
  nosubpix_cross_ = p.nside_cross * p.nside_cross / (nsm * nsm);
  ndeg_cross_ = nosubpix_max_ / nosubpix_cross_;
  ndeg_shift_ = 0;
  while ((1L << ndeg_shift_) < ndeg_cross_) ++ndeg_shift_;
  noba_pp_max_ = 0;
  for (long v : noba_pp_) noba_pp_max_ = std::max(noba_pp_max_, v);
  // start_timeloop (parameter_control.f90:752-846): baseline lengths
  bstart_.assign(noba_short_ + 1, 0);
  long m = 0;
  long long pos = 0;
  for (long i = 0; i < ninterval_; ++i) {
    double dn = 0;
    long nn = 0;
    for (long k = 0; k < noba_pp_[i] - 1; ++k) {
      const double dn0 = dn;
      const long n0 = nn;
      dn = dn0 + dnshort_;
      nn = (long)(dn + .5);
      bstart_[m++] = (uint32_t)pos;
      pos += nn - n0;
    }
    const long last = intervals_[i] - nn;
    if (p.kfirst && (last < 0 || last > (long)dnshort_ + 1))
      fail("ERROR in start_timeloop: Lengths do not match.");
    bstart_[m++] = (uint32_t)pos;
    pos += last;
  }
  bstart_[m] = (uint32_t)pos;
  // gather tiling: kb baselines per CTA tile when baselines are short
  {
    long maxlen = 0;
    for (long k = 0; k < noba_short_; ++k) maxlen = std::max<long>(maxlen, bstart_[k + 1] - bstart_[k]);
    gather_kb_ = 0;
    if (maxlen > 0 && maxlen <= kGatherTile / 2) {
      gather_kb_ = (int)std::max<long>(1, kGatherTile / maxlen);
      gather_kb_ = std::min(gather_kb_, 256);
      gather_tiles_det_ = (noba_short_ + gather_kb_ - 1) / gather_kb_;
    }
  }
  // gather chunks: runs of consecutive baselines of one detector with at most
  // kGatherChunk samples and 32 baselines (every baseline must fit one)
  {
    long maxlen = 0;
    for (long k = 0; k < noba_short_; ++k)
      maxlen = std::max<long>(maxlen, bstart_[k + 1] - bstart_[k]);
    std::vector<int2> ck;
    if (maxlen <= kGatherChunk && (long long)ndet_ * noba_short_ < (1LL << 31)) {
      std::vector<int2> one;  // chunks of detector 0, repeated per detector
      long k = 0;
      while (k < noba_short_) {
        long k1 = k + 1;
        while (k1 < noba_short_ && k1 - k < 32 && bstart_[k1 + 1] - bstart_[k] <= kGatherChunk)
          ++k1;
        one.push_back(make_int2((int)k, (int)(k1 - k)));
        k = k1;
      }
      ck.reserve(one.size() * ndet_);
      for (long d = 0; d < ndet_; ++d)
        for (const int2 &c : one) ck.push_back(make_int2((int)(d * noba_short_ + c.x), c.y));
    }
    ngather_chunks_ = (long long)ck.size();
    gather_chunks_.alloc(std::max<size_t>(1, ck.size()));
    if (!ck.empty())
      MADAM_CUDA(cudaMemcpyAsync(gather_chunks_.get(), ck.data(), ck.size() * sizeof(int2),
                                 cudaMemcpyHostToDevice, st_));
  }
  // every baseline but the last of a period has length dnshort
  const double dnc = std::min(dnshort_, 4294967295.0);
  fdn_ = FastDiv((uint32_t)std::max(1.0, dnc));
  // device copies of the layout tables
  istart_d_.alloc(ninterval_ + 1);
  kstart_d_.alloc(ninterval_ + 1);
  std::vector<long long> is(istart_iv_.begin(), istart_iv_.end());
  std::vector<int> ks(kstart_pp_.begin(), kstart_pp_.end());
  MADAM_CUDA(cudaMemcpyAsync(istart_d_.get(), is.data(), is.size() * sizeof(long long),
                             cudaMemcpyHostToDevice, st_));
  MADAM_CUDA(cudaMemcpyAsync(kstart_d_.get(), ks.data(), ks.size() * sizeof(int),
                             cudaMemcpyHostToDevice, st_));
  bstart_d_.alloc(noba_short_ + 1);
  MADAM_CUDA(cudaMemcpyAsync(bstart_d_.get(), bstart_.data(), bstart_.size() * sizeof(uint32_t),
                             cudaMemcpyHostToDevice, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
}

void Engine::flag_and_compact(bool first_call) {
  const long long n = (long long)ndet_ * nsamp_;
  const SampleMap sm = sample_map(istart_d_.get(), kstart_d_.get(), (int)ninterval_, nsamp_,
                                  noba_short_, fdn_);
  if (first_call && n > 0) {
    // check_files (read_data.f90:241-272)
    MADAM_LAUNCH(k_flag_zero_weight, grid_for(n), 256, 0, st_, pix_.get(), d_w_, (int)nnz_, n);
    DevBuf<unsigned long long> cnt;
    cnt.alloc((size_t)ndet_ * ninterval_);
    cnt.zero(st_);
    MADAM_LAUNCH(k_count_good, grid_for(n), 256, 0, st_, pix_.get(), n, sm, (int)ninterval_,
                 cnt.get());
    DevBuf<long long> ivlen;
    ivlen.alloc(ninterval_);
    std::vector<long long> il(intervals_.begin(), intervals_.end());
    MADAM_CUDA(cudaMemcpyAsync(ivlen.get(), il.data(), il.size() * sizeof(long long),
                               cudaMemcpyHostToDevice, st_));
    MADAM_LAUNCH(k_flag_sparse, grid_for(n), 256, 0, st_, pix_.get(), n, sm, (int)ninterval_,
                 cnt.get(), ivlen.get());
    MADAM_CUDA(cudaStreamSynchronize(st_));
  }
  // init_pointing + where (pixels < 0) pixels = dummy_pixel + reduce_pixels
  dummy_global_ = 12 * nside_max_ * nside_max_;
  DevBuf<int> ksub;
  ksub.alloc(nosubmaps_tot_ + 1);
  ksub.zero(st_);
  if (n > 0)
    MADAM_LAUNCH(k_dummy_ksub, grid_for(n), 256, 0, st_, pix_.get(), n, (int)dummy_global_,
                 (int)nosubpix_max_, ksub.get());
  if (isubchunk_ > 0 && n > 0) {
    // a subchunk pass (smadam.F90:194-196; parameter_control.f90:820-835):
    // interval i contributes its samples [sublen (isub - 1), sublen isub) with
    // sublen = len / nsubchunk (the last subchunk takes the rest); the other
    // samples take the dummy pixel, which excludes them from every sum as the
    // reference's subchunk test does.  The hit submaps stay those of the
    // full data, as the reference compacts once before its passes.
    std::vector<long long> rg;
    long long off = 0;
    for (long iv = 0; iv < ninterval_; ++iv) {
      const long long len = intervals_[iv], sublen = len / nsubchunk_;
      const long long a = off + sublen * (isubchunk_ - 1);
      const long long b = isubchunk_ == nsubchunk_ ? off + len : a + sublen;
      rg.push_back(a);
      rg.push_back(b);
      off += len;
    }
    DevBuf<long long> drg;
    drg.alloc(rg.size());
    MADAM_CUDA(cudaMemcpyAsync(drg.get(), rg.data(), rg.size() * sizeof(long long),
                               cudaMemcpyHostToDevice, st_));
    MADAM_LAUNCH(k_subchunk_mask, grid_for(n), 256, 0, st_, pix_.get(), n, (long long)nsamp_,
                 drg.get(), (int)ninterval_, (int)dummy_global_);
  }
  ar_max(ksub.get(), nosubmaps_tot_ + 1);  // the hit submaps of every rank
  std::vector<int> ks(nosubmaps_tot_ + 1);
  MADAM_CUDA(cudaMemcpyAsync(ks.data(), ksub.get(), ks.size() * sizeof(int),
                             cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  ks[nosubmaps_tot_] = 1;
  if (first_call) {
    ksubmap_ = ks;
    subtable1_.assign(nosubmaps_tot_ + 1, -1);
    subtable2_.assign(nosubmaps_tot_ + 1, -1);
    long k = -1;
    for (long i = 0; i <= nosubmaps_tot_; ++i)
      if (ksubmap_[i]) {
        ++k;
        subtable1_[i] = i - k;
        subtable2_[k] = i - k;
      }
    nolocmaps_ = 0;
    for (long i = 0; i < nosubmaps_tot_; ++i) nolocmaps_ += ksubmap_[i] ? 1 : 0;
    nloc_ = nolocmaps_ * nosubpix_max_;
    nloc_map_ = nloc_;
    nloc_cross_ = nolocmaps_ * nosubpix_cross_;
    dummy_local_ = (nosubmaps_tot_ - subtable1_[nosubmaps_tot_]) * nosubpix_max_;
    if (nloc_ >= (1L << 30)) fail("map too large");
    int ts = 0;
    while ((1L << (ts + 1)) <= std::min<long>(nosubpix_max_, kTileMax)) ++ts;
    tile_shift_ = ts;
    ntiles_ = (nloc_ + (1L << ts) - 1) >> ts;
  } else {
    for (long i = 0; i <= nosubmaps_tot_; ++i)
      if ((ks[i] != 0) != (ksubmap_[i] != 0))
        fail("destripe_with_cache: the pointing hits other submaps than the cached call");
  }
  DevBuf<int> sub1;
  sub1.alloc(nosubmaps_tot_ + 1);
  std::vector<int> s1(subtable1_.begin(), subtable1_.end());
  MADAM_CUDA(cudaMemcpyAsync(sub1.get(), s1.data(), s1.size() * sizeof(int),
                             cudaMemcpyHostToDevice, st_));
  if (nmap_ == 3 && nnz_ == 3) {
    point4_.alloc(n);
    if (n > 0)
      MADAM_LAUNCH(k_compact<3>, grid_for(n), 256, 0, st_, pix_.get(), d_w_, n, sub1.get(),
                   (int)nosubpix_max_, point4_.get(), nullptr);
  } else {
    pixc_.alloc(n);
    if (n > 0)
      MADAM_LAUNCH(k_compact<1>, grid_for(n), 256, 0, st_, pix_.get(), d_w_, n, sub1.get(),
                   (int)nosubpix_max_, nullptr, pixc_.get());
  }
  MADAM_CUDA(cudaStreamSynchronize(st_));
  // the staging copy of host weights is done with, unless the covariance
  // files read the raw weights later
  if (!in_device_ && par_.file_covmat.empty()) wraw_.reset();
  // detector weights per (det, period) and per baseline
  if (first_call) {
    detw_iv_.assign((size_t)ndet_ * ninterval_, 0.0);
    for (long d = 0; d < ndet_; ++d)
      for (long iv = 0; iv < ninterval_; ++iv) {
        const int ipsd = psd_index_det(dets_[d], btime_[kstart_pp_[iv]]);
        if (ipsd < 0) continue;
        detw_iv_[d * ninterval_ + iv] = dets_[d].weights[ipsd];
      }
    DevBuf<double> dw;
    dw.alloc(detw_iv_.size());
    MADAM_CUDA(cudaMemcpyAsync(dw.get(), detw_iv_.data(), detw_iv_.size() * sizeof(double),
                               cudaMemcpyHostToDevice, st_));
    const long long nb = (long long)ndet_ * noba_short_;
    bw_.alloc(nb);
    MADAM_LAUNCH(k_baseline_weights, grid_for(nb), 256, 0, st_, bw_.get(), nb, noba_short_,
                 kstart_d_.get(), (int)ninterval_, dw.get());
    MADAM_CUDA(cudaStreamSynchronize(st_));
  }
  // flag_bad_baselines (read_data.f90:30-74)
  // flag_bad_baselines counts only samples whose pixel the input mask keeps,
  // but it runs before the mask is read (smadam.F90:309, 337-345), when the
  // mask table is still zero: with file_inmask it flags nothing
  if (par_.kfirst && par_.good_baseline_fraction != 0 && !par_.kfilter &&
      par_.file_inmask.empty()) {
    const long long nb = (long long)ndet_ * noba_short_;
    const unsigned grid = (unsigned)((nb * 32 + 255) / 256);
    if (nmap_ == 3)
      MADAM_LAUNCH(k_bad_baselines<3>, grid, 256, 0, st_, pix_.get(), point4_.get(), nullptr, nb,
                   noba_short_, nsamp_, bstart_d_.get(), (int)dummy_global_,
                   par_.good_baseline_fraction);
    else
      MADAM_LAUNCH(k_bad_baselines<1>, grid, 256, 0, st_, pix_.get(), nullptr, pixc_.get(), nb,
                   noba_short_, nsamp_, bstart_d_.get(), (int)dummy_global_,
                   par_.good_baseline_fraction);
  }
}

void Engine::trace(const char *what) {
  if (!trace_on_) return;
  // host time since the last point, and the stream's own time between
  // events recorded at the two points
  if (!trace_ev_[0]) {
    MADAM_CUDA(cudaEventCreate(&trace_ev_[0]));
    MADAM_CUDA(cudaEventCreate(&trace_ev_[1]));
    MADAM_CUDA(cudaEventRecord(trace_ev_[0], st_));
  }
  MADAM_CUDA(cudaEventRecord(trace_ev_[1], st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  float dev_ms = 0;
  MADAM_CUDA(cudaEventElapsedTime(&dev_ms, trace_ev_[0], trace_ev_[1]));
  std::swap(trace_ev_[0], trace_ev_[1]);
  const double t = now_ms();
  int dev = 0;
  cudaMemPool_t pool;
  uint64_t reserved = 0, used = 0;
  if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
  }
  std::fprintf(stderr,
               "madam_b200 trace: %-28s %9.3f ms (stream %9.3f ms)  pool %.2f GB reserved, "
               "%.2f GB used\n",
               what, t - trace_t_, dev_ms, reserved / 1e9, used / 1e9);
  trace_t_ = t;
}

void Engine::build_runs() {
  const long long n = (long long)ndet_ * nsamp_;
  const SampleMap sm = sample_map(istart_d_.get(), kstart_d_.get(), (int)ninterval_, nsamp_,
                                  noba_short_, fdn_);
  nruns_ = 0;
  nwork_ = 0;
  item_begin_.alloc(1);
  item_begin_.zero(st_);
  if (n == 0) return;
  DevBuf<uint8_t> sflag, eflag;
  sflag.alloc(n);
  eflag.alloc(n);
  const float4 *p4 = point4_.get();
  const int32_t *pc = pixc_.get();
  if (nmap_ == 3)
    MADAM_LAUNCH(k_run_flags<3>, grid_for(n), 256, 0, st_, p4, pc, n, sm, bw_.get(), (int)nloc_,
                 tile_shift_, sflag.get(), eflag.get());
  else
    MADAM_LAUNCH(k_run_flags<1>, grid_for(n), 256, 0, st_, p4, pc, n, sm, bw_.get(), (int)nloc_,
                 tile_shift_, sflag.get(), eflag.get());
  // select run starts / ends
  DevBuf<long long> starts, ends, nsel;
  starts.alloc(n);
  ends.alloc(n);
  nsel.alloc(2);
  cub::CountingInputIterator<long long> it(0);
  size_t tmpb = 0;
  MADAM_CUDA(cub::DeviceSelect::Flagged(nullptr, tmpb, it, sflag.get(), starts.get(), nsel.get(),
                                        n, st_));
  DevBuf<uint8_t> tmp;
  tmp.alloc(tmpb);
  MADAM_CUDA(cub::DeviceSelect::Flagged(tmp.get(), tmpb, it, sflag.get(), starts.get(),
                                        nsel.get(), n, st_));
  MADAM_CUDA(cub::DeviceSelect::Flagged(tmp.get(), tmpb, it, eflag.get(), ends.get(),
                                        nsel.get() + 1, n, st_));
  long long cnt[2];
  MADAM_CUDA(cudaMemcpyAsync(cnt, nsel.get(), sizeof cnt, cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  sflag.reset();
  eflag.reset();
  trace("runs: flags+select");
  if (cnt[0] != cnt[1]) fail("internal: unpaired run boundaries");
  const long long nr0 = cnt[0];
  if (nr0 == 0) return;
  // split long runs
  DevBuf<long long> pieces, poff;
  pieces.alloc(nr0);
  poff.alloc(nr0 + 1);
  MADAM_LAUNCH(k_run_pieces, grid_for(nr0), 256, 0, st_, starts.get(), ends.get(), nr0,
               pieces.get());
  tmpb = 0;
  MADAM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmpb, pieces.get(), poff.get(), nr0, st_));
  tmp.alloc(std::max<size_t>(tmpb, tmp.n));
  MADAM_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tmpb, pieces.get(), poff.get(), nr0, st_));
  long long lastoff, lastp;
  MADAM_CUDA(cudaMemcpyAsync(&lastoff, poff.get() + nr0 - 1, sizeof(long long),
                             cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaMemcpyAsync(&lastp, pieces.get() + nr0 - 1, sizeof(long long),
                             cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  const long long nr = lastoff + lastp;
  if (nr >= (1LL << 31)) fail("too many runs");
  DevBuf<Run> runs0;
  DevBuf<int> keys, lens, keys_sorted, idx, idx_sorted, lens_sorted;
  runs0.alloc(nr);
  keys.alloc(nr);
  lens.alloc(nr);
  if (nmap_ == 3)
    MADAM_LAUNCH(k_run_emit<3>, grid_for(nr0), 256, 0, st_, starts.get(), ends.get(), poff.get(),
                 nr0, sm, p4, pc, tile_shift_, runs0.get(), keys.get(), lens.get());
  else
    MADAM_LAUNCH(k_run_emit<1>, grid_for(nr0), 256, 0, st_, starts.get(), ends.get(), poff.get(),
                 nr0, sm, p4, pc, tile_shift_, runs0.get(), keys.get(), lens.get());
  starts.reset();
  ends.reset();
  trace("runs: split+emit");
  // bucket runs by tile (stable radix sort keeps time order inside a tile)
  idx.alloc(nr);
  idx_sorted.alloc(nr);
  keys_sorted.alloc(nr);
  MADAM_LAUNCH(k_iota, grid_for(nr), 256, 0, st_, idx.get(), nr);
  int endbit = 1;
  while ((1L << endbit) <= ntiles_) ++endbit;
  tmpb = 0;
  MADAM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmpb, keys.get(), keys_sorted.get(),
                                             idx.get(), idx_sorted.get(), (int)nr, 0, endbit, st_));
  tmp.alloc(std::max<size_t>(tmpb, tmp.n));
  MADAM_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmpb, keys.get(), keys_sorted.get(),
                                             idx.get(), idx_sorted.get(), (int)nr, 0, endbit, st_));
  trace("runs: iota+sort");
  runs_.alloc(nr);
  lens_sorted.alloc(nr);
  MADAM_LAUNCH(k_gather_runs, grid_for(nr), 256, 0, st_, idx_sorted.get(), runs0.get(),
               lens.get(), nr, runs_.get(), lens_sorted.get());
  runs0.reset();
  // work items: <= kItemSamples samples of one tile
  DevBuf<long long> lens64, pref;
  lens64.alloc(nr);
  pref.alloc(nr);
  tmpb = 0;
  cub::TransformInputIterator<long long, cub::CastOp<long long>, const int *> wide(
      lens_sorted.get(), cub::CastOp<long long>());
  MADAM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmpb, wide, pref.get(), nr, st_));
  tmp.alloc(std::max<size_t>(tmpb, tmp.n));
  MADAM_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tmpb, wide, pref.get(), nr, st_));
  DevBuf<uint8_t> iflag;
  iflag.alloc(nr);
  MADAM_LAUNCH(k_item_flags, grid_for(nr), 256, 0, st_, keys_sorted.get(), pref.get(), nr,
               iflag.get());
  DevBuf<long long> ibeg, nitem;
  ibeg.alloc(nr);
  nitem.alloc(1);
  cub::CountingInputIterator<long long> it2(0);
  tmpb = 0;
  MADAM_CUDA(cub::DeviceSelect::Flagged(nullptr, tmpb, it2, iflag.get(), ibeg.get(), nitem.get(),
                                        nr, st_));
  tmp.alloc(std::max<size_t>(tmpb, tmp.n));
  MADAM_CUDA(cub::DeviceSelect::Flagged(tmp.get(), tmpb, it2, iflag.get(), ibeg.get(),
                                        nitem.get(), nr, st_));
  long long ni;
  MADAM_CUDA(cudaMemcpyAsync(&ni, nitem.get(), sizeof ni, cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  item_begin_.alloc(ni + 1);
  item_tile_.alloc(ni);
  MADAM_LAUNCH(k_item_tiles, grid_for(ni), 256, 0, st_, ibeg.get(), ni, keys_sorted.get(),
               item_begin_.get(), item_tile_.get());
  const int nrr = (int)nr;
  MADAM_CUDA(cudaMemcpyAsync(item_begin_.get() + ni, &nrr, sizeof(int), cudaMemcpyHostToDevice,
                             st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  nruns_ = nr;
  nwork_ = ni;
}

void Engine::build_csr() {
  // pixel-sorted copy of the pointing for the PCG scatter (k_scatter_csr)
  const long long n = (long long)ndet_ * nsamp_;
  csr_nvalid_ = 0;
  nscatter_chunks_ = 0;
  nscatter_multi_ = 0;
  csr_off_.alloc((size_t)nloc_cross_ + 1);
  if (n == 0 || nloc_cross_ == 0) {
    csr_off_.zero(st_);
    return;
  }
  if (n >= (1LL << 31)) fail("too many samples for the pixel-sorted pointing");
  use_pairs_ = false;
  npairs_ = 0;
  gp4_.reset();
  poff_.reset();
  pair_chunks_.reset();
  npair_chunks_ = 0;
  have_xcsr_ = false;
  build_sample_csr();
  trace("csr: sample csr");
  if (fp32_ && nmap_ == 3) {
    // FP32-TOD form: the scatter runs over pointing pairs; the sample CSR
    // stays for the reliable updates' exact scatter (apply_A_exact)
    swap_csr();
    csr_off_.alloc((size_t)nloc_cross_ + 1);
    if (build_pairs()) {
      trace("csr: pairs");
      build_scatter_chunks();
      trace("csr: pair scatter chunks");
      have_xcsr_ = true;
      return;
    }
    swap_csr();  // no pairs: the samples serve both
  }
}

// The pixel-sorted samples and their scatter chunks trade places with the
// exact-scatter copy (x*).
void Engine::swap_csr() {
  auto sw = [](auto &a, auto &b) {
    std::swap(a.p, b.p);
    std::swap(a.n, b.n);
  };
  sw(sp4_, xsp4_);
  sw(sp2_, xsp2_);
  sw(csr_off_, xcsr_off_);
  sw(scatter_chunks_, xscatter_chunks_);
  sw(scatter_multi_, xscatter_multi_);
  sw(scatter_partial_, xscatter_partial_);
  std::swap(nscatter_chunks_, xnscatter_chunks_);
  std::swap(nscatter_multi_, xnscatter_multi_);
  std::swap(csr_nvalid_, xcsr_nvalid_);
}

void Engine::build_sample_csr() {
  const long long n = (long long)ndet_ * nsamp_;
  const SampleMap sm = sample_map(istart_d_.get(), kstart_d_.get(), (int)ninterval_, nsamp_,
                                  noba_short_, fdn_);
  DevBuf<int> keys, keys_s;
  DevBuf<uint32_t> vals, vals_s;
  DevBuf<unsigned long long> cnt;
  keys.alloc(n);
  vals.alloc(n);
  cnt.alloc(1);
  cnt.zero(st_);
  const int sentinel = (int)nloc_cross_;
  if (nmap_ == 3)
    MADAM_LAUNCH(k_csr_keys<3>, grid_for(n), 256, 0, st_, point4_.get(), pixc_.get(), n, sm,
                 bw_.get(), (int)nloc_, (int)ndeg_shift_, sentinel, keys.get(), vals.get(),
                 cnt.get());
  else
    MADAM_LAUNCH(k_csr_keys<1>, grid_for(n), 256, 0, st_, point4_.get(), pixc_.get(), n, sm,
                 bw_.get(), (int)nloc_, (int)ndeg_shift_, sentinel, keys.get(), vals.get(),
                 cnt.get());
  unsigned long long nv = 0;
  MADAM_CUDA(cudaMemcpyAsync(&nv, cnt.get(), sizeof nv, cudaMemcpyDeviceToHost, st_));
  keys_s.alloc(n);
  vals_s.alloc(n);
  int endbit = 1;
  while ((1L << endbit) <= sentinel) ++endbit;
  size_t tmpb = 0;
  MADAM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmpb, keys.get(), keys_s.get(), vals.get(),
                                             vals_s.get(), (int)n, 0, endbit, st_));
  DevBuf<uint8_t> tmp;
  tmp.alloc(tmpb);
  MADAM_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmpb, keys.get(), keys_s.get(),
                                             vals.get(), vals_s.get(), (int)n, 0, endbit, st_));
  tmp.reset();
  keys.reset();
  vals.reset();
  MADAM_CUDA(cudaStreamSynchronize(st_));
  trace("csr: keys+sort");
  csr_nvalid_ = (long long)nv;
  MADAM_LAUNCH(k_fill_int, grid_for(nloc_cross_ + 1), 256, 0, st_, csr_off_.get(),
               (long long)nloc_cross_ + 1, (int)csr_nvalid_);
  if (nmap_ == 3) {
    sp4_.alloc(std::max<long long>(1, csr_nvalid_));
    if (csr_nvalid_)
      MADAM_LAUNCH(k_csr_fill<3>, grid_for(csr_nvalid_), 256, 0, st_, keys_s.get(), vals_s.get(),
                   csr_nvalid_, point4_.get(), sm, sp4_.get(), (int2 *)nullptr, csr_off_.get());
  } else {
    sp2_.alloc(std::max<long long>(1, csr_nvalid_));
    if (csr_nvalid_)
      MADAM_LAUNCH(k_csr_fill<1>, grid_for(csr_nvalid_), 256, 0, st_, keys_s.get(), vals_s.get(),
                   csr_nvalid_, point4_.get(), sm, (float4 *)nullptr, sp2_.get(), csr_off_.get());
  }
  MADAM_CUDA(cudaStreamSynchronize(st_));
  trace("csr: fill");
  build_scatter_chunks();
}

void Engine::build_scatter_chunks() {
  // scatter chunks: every pixel's entries cut into chunks of at most
  // kScatterChunk; pixels of several chunks combine their partial sums
  // (built on the device: counts, three prefix sums, then the fill)
  const int np = (int)nloc_cross_;
  nscatter_chunks_ = 0;
  nscatter_multi_ = 0;
  if (np <= 0) {
    scatter_chunks_.alloc(1);
    scatter_multi_.alloc(1);
    scatter_partial_.alloc((size_t)nmap_);
    return;
  }
  DevBuf<int> cnt, off;
  cnt.alloc((size_t)3 * np);
  off.alloc((size_t)3 * (np + 1));
  int *nck = cnt.get(), *nslot = nck + np, *nmulti = nslot + np;
  int *ock = off.get(), *oslot = ock + (np + 1), *omulti = oslot + (np + 1);
  MADAM_LAUNCH(k_scatter_chunk_count, grid_for(np), 256, 0, st_, csr_off_.get(), np,
               kScatterChunk, nck, nslot, nmulti);
  size_t tmpb = 0;
  MADAM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmpb, nck, ock, np, st_));
  DevBuf<uint8_t> tmp;
  tmp.alloc(tmpb);
  // each total is the last prefix plus the last count
  for (int q = 0; q < 3; ++q)
    MADAM_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tmpb, cnt.get() + (size_t)q * np,
                                             off.get() + (size_t)q * (np + 1), np, st_));
  int last[6];
  for (int q = 0; q < 3; ++q) {
    MADAM_CUDA(cudaMemcpyAsync(&last[2 * q], off.get() + (size_t)q * (np + 1) + (np - 1),
                               sizeof(int), cudaMemcpyDeviceToHost, st_));
    MADAM_CUDA(cudaMemcpyAsync(&last[2 * q + 1], cnt.get() + (size_t)q * np + (np - 1),
                               sizeof(int), cudaMemcpyDeviceToHost, st_));
  }
  MADAM_CUDA(cudaStreamSynchronize(st_));
  const long long nck_tot = (long long)last[0] + last[1];
  const int nslot_tot = last[2] + last[3];
  const int nmulti_tot = last[4] + last[5];
  nscatter_chunks_ = nck_tot;
  nscatter_multi_ = nmulti_tot;
  scatter_chunks_.alloc(std::max<long long>(1, nck_tot));
  scatter_multi_.alloc(std::max(1, nmulti_tot));
  scatter_partial_.alloc((size_t)std::max(1, nslot_tot) * nmap_);
  MADAM_LAUNCH(k_scatter_chunk_fill, grid_for(np), 256, 0, st_, csr_off_.get(), np,
               kScatterChunk, ock, oslot, omulti, scatter_chunks_.get(), scatter_multi_.get());
  MADAM_CUDA(cudaStreamSynchronize(st_));
}

// Pointing pairs of the FP32-TOD form (pair_kernels.inl): time-ordered pairs
// with per-baseline offsets and gather chunks, and the pixel-sorted pairs in
// sp4_ / csr_off_ for the scatter.  false (nothing built) when a baseline
// holds more than kGatherChunk pairs.
bool Engine::build_pairs() {
  const long long n = (long long)ndet_ * nsamp_;
  const long long nb = (long long)ndet_ * noba_short_;
  const SampleMap sm = sample_map(istart_d_.get(), kstart_d_.get(), (int)ninterval_, nsamp_,
                                  noba_short_, fdn_);
  DevBuf<int> head, pidx;
  head.alloc(n);
  pidx.alloc(n);
  MADAM_LAUNCH(k_pair_heads, grid_for(n), 256, 0, st_, point4_.get(), n, sm, bw_.get(),
               (int)nloc_, (int)ndeg_shift_, head.get());
  {
    size_t tmpb = 0;
    MADAM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmpb, head.get(), pidx.get(), (int)n, st_));
    DevBuf<uint8_t> tmp;
    tmp.alloc(tmpb);
    MADAM_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tmpb, head.get(), pidx.get(), (int)n, st_));
  }
  int last[2] = {0, 0};
  MADAM_CUDA(cudaMemcpyAsync(&last[0], pidx.get() + (n - 1), sizeof(int), cudaMemcpyDeviceToHost,
                             st_));
  MADAM_CUDA(cudaMemcpyAsync(&last[1], head.get() + (n - 1), sizeof(int), cudaMemcpyDeviceToHost,
                             st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  const int np = last[0] + last[1];
  // per-baseline pair offsets, checked on the host before anything else
  poff_.alloc(nb + 1);
  MADAM_LAUNCH(k_pair_offsets, grid_for(nb + 1), 256, 0, st_, pidx.get(), bstart_d_.get(),
               (long long)nsamp_, noba_short_, nb, n, np, poff_.get());
  std::vector<int> offh((size_t)nb + 1);
  MADAM_CUDA(cudaMemcpyAsync(offh.data(), poff_.get(), offh.size() * sizeof(int),
                             cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  std::vector<int4> ck;
  for (long long d = 0; d < ndet_; ++d) {
    long long b = d * noba_short_;
    const long long b1 = b + noba_short_;
    while (b < b1) {
      if (offh[b + 1] - offh[b] > kGatherChunk) {
        poff_.reset();
        return false;
      }
      long long e = b + 1;
      while (e < b1 && e - b < 32 && offh[e + 1] - offh[b] <= kGatherChunk) ++e;
      ck.push_back(make_int4((int)b, (int)(e - b), offh[b], offh[e] - offh[b]));
      b = e;
    }
  }
  trace("pairs: heads+offsets+chunks");
  npairs_ = np;
  gp4_.alloc(std::max(1, np));
  DevBuf<int> pbase;
  pbase.alloc(std::max(1, np));
  MADAM_LAUNCH(k_pair_fill, grid_for(n), 256, 0, st_, point4_.get(), n, sm, bstart_d_.get(),
               (int)nloc_, (int)ndeg_shift_, head.get(), pidx.get(), gp4_.get(), pbase.get());
  head.reset();
  pidx.reset();
  npair_chunks_ = (long long)ck.size();
  pair_chunks_.alloc(std::max<size_t>(1, ck.size()));
  if (!ck.empty())
    MADAM_CUDA(cudaMemcpyAsync(pair_chunks_.get(), ck.data(), ck.size() * sizeof(int4),
                               cudaMemcpyHostToDevice, st_));
  trace("pairs: fill");
  // pixel-sorted pairs (stable radix sort: time order inside a pixel)
  csr_nvalid_ = np;
  MADAM_LAUNCH(k_fill_int, grid_for(nloc_cross_ + 1), 256, 0, st_, csr_off_.get(),
               (long long)nloc_cross_ + 1, np);
  sp4_.alloc(std::max(1, np));
  if (np > 0) {
    DevBuf<int> keys, keys_s;
    DevBuf<uint32_t> vals, vals_s;
    keys.alloc(np);
    vals.alloc(np);
    keys_s.alloc(np);
    vals_s.alloc(np);
    MADAM_LAUNCH(k_pair_keys, grid_for(np), 256, 0, st_, gp4_.get(), np, keys.get(), vals.get());
    int endbit = 1;
    while ((1L << endbit) <= nloc_cross_) ++endbit;
    size_t tmpb = 0;
    MADAM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmpb, keys.get(), keys_s.get(),
                                               vals.get(), vals_s.get(), np, 0, endbit, st_));
    DevBuf<uint8_t> tmp;
    tmp.alloc(tmpb);
    MADAM_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tmpb, keys.get(), keys_s.get(),
                                               vals.get(), vals_s.get(), np, 0, endbit, st_));
    MADAM_LAUNCH(k_pair_csr_fill, grid_for(np), 256, 0, st_, keys_s.get(), vals_s.get(), np,
                 gp4_.get(), pbase.get(), sp4_.get(), csr_off_.get());
  }
  use_pairs_ = true;
  MADAM_CUDA(cudaStreamSynchronize(st_));
  return true;
}

void Engine::bin_tod(bool accumulate_wamap) {
  wait_tod();
  // pixel_matrix + count_hits + bin_tod (smadam_routines.f90:111-422)
  const int ncc = nmap_ == 3 ? 6 : 1;
  const int T = 1 << tile_shift_;
  const size_t smem = (size_t)(ncc + nmap_) * T * sizeof(double) + T * sizeof(int);
  static bool attr = false;
  if (!attr) {
    MADAM_CUDA(cudaFuncSetAttribute(k_setup_scatter<3>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    MADAM_CUDA(cudaFuncSetAttribute(k_setup_scatter<1>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024));
    attr = true;
  }
  DevBuf<double> ccacc, bin;
  DevBuf<int> hits;
  ccacc.alloc((size_t)nloc_ * ncc);
  ccacc.zero(st_);
  bin.alloc((size_t)nloc_ * nmap_);
  bin.zero(st_);
  hits.alloc(nloc_);
  hits.zero(st_);
  if (nwork_ > 0) {
    if (nmap_ == 3)
      MADAM_LAUNCH(k_setup_scatter<3>, (unsigned)nwork_, 256, smem, st_, item_begin_.get(),
                   item_tile_.get(), runs_.get(), point4_.get(), pixc_.get(), d_tod_, bw_.get(),
                   fdn_, tile_shift_, ccacc.get(), bin.get(), hits.get());
    else
      MADAM_LAUNCH(k_setup_scatter<1>, (unsigned)nwork_, 256, smem, st_, item_begin_.get(),
                   item_tile_.get(), runs_.get(), point4_.get(), pixc_.get(), d_tod_, bw_.get(),
                   fdn_, tile_shift_, ccacc.get(), bin.get(), hits.get());
  }
  // collect_cc / collect_hits / collect_map across the ranks
  ar_sum(ccacc.get(), ccacc.n);
  ar_sum(bin.get(), bin.n);
  ar_sum(hits.get(), hits.n);
  const long long nv = (long long)nloc_ * nmap_;
  if (!accumulate_wamap) {
    // first call: cc, cca, hits, map, binmap, wamap from scratch
    cc_.alloc((size_t)nloc_ * ncc);
    MADAM_CUDA(cudaMemcpyAsync(cc_.get(), ccacc.get(), cc_.n * sizeof(double),
                               cudaMemcpyDeviceToDevice, st_));
    hits_.alloc(nloc_);
    MADAM_CUDA(cudaMemcpyAsync(hits_.get(), hits.get(), nloc_ * sizeof(int),
                               cudaMemcpyDeviceToDevice, st_));
    cca_.alloc((size_t)nloc_cross_ * ncc);
    wamap_.alloc((size_t)nloc_cross_ * nmap_);
    wamap_.zero(st_);
    if (ndeg_cross_ == 1) {
      MADAM_CUDA(cudaMemcpyAsync(cca_.get(), ccacc.get(), cca_.n * sizeof(double),
                                 cudaMemcpyDeviceToDevice, st_));
    } else {
      MADAM_LAUNCH(k_degrade, grid_for(nloc_cross_ * ncc), 256, 0, st_, ccacc.get(), cca_.get(),
                   (long long)nloc_cross_, ncc, (int)ndeg_cross_);
    }
  }
  map_.alloc(nv);
  binmap_.alloc(nv);
  if (par_.kfirst) {
    MADAM_CUDA(cudaMemcpyAsync(map_.get(), bin.get(), nv * sizeof(double),
                               cudaMemcpyDeviceToDevice, st_));
  } else {
    map_.zero(st_);
  }
  MADAM_CUDA(cudaMemcpyAsync(binmap_.get(), bin.get(), nv * sizeof(double),
                             cudaMemcpyDeviceToDevice, st_));
  if (par_.kfirst) {
    // collect_map(wamap) adds to whatever wamap holds
    DevBuf<double> wc;
    wc.alloc((size_t)nloc_cross_ * nmap_);
    if (ndeg_cross_ == 1)
      MADAM_CUDA(cudaMemcpyAsync(wc.get(), bin.get(), wc.n * sizeof(double),
                                 cudaMemcpyDeviceToDevice, st_));
    else
      MADAM_LAUNCH(k_degrade, grid_for(nloc_cross_ * nmap_), 256, 0, st_, bin.get(), wc.get(),
                   (long long)nloc_cross_, nmap_, (int)ndeg_cross_);
    MADAM_LAUNCH(k_add, grid_for(wc.n), 256, 0, st_, wamap_.get(), wc.get(), (long long)wc.n);
    MADAM_CUDA(cudaStreamSynchronize(st_));
  }
  MADAM_CUDA(cudaStreamSynchronize(st_));
}

void Engine::setup_scatter() { bin_tod(false); }

void Engine::apply_inmask() {
  // read_inmask (read_data.f90:90-190) up- or downgraded to nside_cross, and
  // the zeroing of the masked pixel matrices in invert_pixelmatrix_cross
  // (map_routines.f90:100-104); zeroing after the inversion gives the same
  // zero matrix, which the inversion leaves alone
  long ns = 0;
  std::string ord;
  const std::vector<float> col = read_mask_column(par_.file_inmask, ns, ord);
  if (ord == "RING") fail("Error in subroutine Read_inmask. Input mask should be in NESTED ordering.");
  if (ord != "NESTED")
    fail("Error in subroutine Read_inmask. Cannot determine the ordering (nested or ring).");
  const long nsc = par_.nside_cross;
  if (ns < par_.nside_submap || (ns & (ns - 1))) fail("file_inmask: invalid NSIDE");
  const long nin = (ns / par_.nside_submap) * (ns / par_.nside_submap);
  const long n = nsc >= ns ? (nsc / ns) * (nsc / ns) : (ns / nsc) * (ns / nsc);
  if ((long)col.size() < nosubmaps_tot_ * nin) fail("file_inmask: too few pixels");
  std::vector<uint8_t> m((size_t)nloc_cross_, 1);
  for (long j = 0; j < nolocmaps_; ++j) {
    const float *fb = col.data() + (size_t)(j + subtable2_[j]) * nin;
    uint8_t *mj = m.data() + (size_t)j * nosubpix_cross_;
    if (nsc >= ns) {
      for (long i = 0; i < nin; ++i)
        for (long q = 0; q < n; ++q) mj[i * n + q] = fb[i] < 0.5f ? 0 : 1;
    } else {
      for (long i = 0; i < nosubpix_cross_; ++i) {
        bool any = false;
        for (long q = 0; q < n; ++q) any = any || fb[i * n + q] < 0.5f;
        mj[i] = any ? 0 : 1;
      }
    }
  }
  DevBuf<uint8_t> dm;
  dm.alloc(m.size());
  MADAM_CUDA(cudaMemcpyAsync(dm.get(), m.data(), m.size(), cudaMemcpyHostToDevice, st_));
  MADAM_LAUNCH(k_apply_inmask, grid_for(nloc_cross_), 256, 0, st_, cca_.get(),
               (long long)nloc_cross_, nmap_ == 3 ? 6 : 1, dm.get());
  MADAM_CUDA(cudaStreamSynchronize(st_));
}

void Engine::map_side_setup() {
  // invert_pixelmatrix_cross (map_routines.f90:83-212)
  MatrixRules mr{(int)par_.pixmode_cross, par_.pixlim_cross, par_.allow_decoupling ? 1 : 0,
                 par_.incomplete_matrices ? 1 : 0};
  if (nloc_cross_ == 0) return;
  if (nmap_ == 3)
    MADAM_LAUNCH(k_invert_cross<3>, grid_for(nloc_cross_), 128, 0, st_, cca_.get(),
                 (long long)nloc_cross_, mr);
  else
    MADAM_LAUNCH(k_invert_cross<1>, grid_for(nloc_cross_), 128, 0, st_, cca_.get(),
                 (long long)nloc_cross_, mr);
  if (!par_.file_inmask.empty()) apply_inmask();
}

void Engine::initialize_a() {
  // initialize_a (smadam_routines.f90:428-671)
  const long long nb = (long long)ndet_ * noba_short_;
  if (nloc_cross_ > 0) {
    if (nmap_ == 3)
      MADAM_LAUNCH(k_ccmult<3>, grid_for(nloc_cross_), 256, 0, st_, cca_.get(), wamap_.get(),
                   (long long)nloc_cross_);
    else
      MADAM_LAUNCH(k_ccmult<1>, grid_for(nloc_cross_), 256, 0, st_, cca_.get(), wamap_.get(),
                   (long long)nloc_cross_);
  }
  if (nbasis_ > 1) return initialize_a_basis();
  yba_.alloc(nb);
  nna_.alloc(nb);
  aa_.alloc(nb);
  yba_.zero(st_);
  nna_.zero(st_);
  aa_.zero(st_);
  const unsigned grid = (unsigned)((nb * 32 + 255) / 256);
  if (nb > 0) {
    if (nmap_ == 3)
      MADAM_LAUNCH(k_init_a<3>, grid, 256, 0, st_, point4_.get(), pixc_.get(), d_tod_,
                   bstart_d_.get(), nb, noba_short_, nsamp_, bw_.get(), wamap_.get(),
                   (int)ndeg_shift_, (int)nloc_, yba_.get(), nna_.get());
    else
      MADAM_LAUNCH(k_init_a<1>, grid, 256, 0, st_, point4_.get(), pixc_.get(), d_tod_,
                   bstart_d_.get(), nb, noba_short_, nsamp_, bw_.get(), wamap_.get(),
                   (int)ndeg_shift_, (int)nloc_, yba_.get(), nna_.get());
  }
  nna_host_.resize(nb);
  MADAM_CUDA(cudaMemcpyAsync(nna_host_.data(), nna_.get(), nb * sizeof(double),
                             cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
}

namespace {
// psd_index (noise_routines.f90:193-208)
int psd_index_global(const std::vector<int> &psddet, const std::vector<double> &start,
                     const std::vector<double> &stop, long det, double t) {
  for (size_t i = 0; i < psddet.size(); ++i)
    if (psddet[i] == det && start[i] <= t && stop[i] >= t) return (int)i;
  return -1;
}
}  // namespace

void Engine::build_segments() {
  // trim_interval (noise_routines.f90:764-813) over every (det, period)
  segs_.clear();
  const long gapmin = (long)(60 * par_.fsample / dnshort_ + 1);
  const long long nb = (long long)ndet_ * noba_short_;
  std::vector<uint8_t> rm(nb, 0);
  for (long d = 0; d < ndet_; ++d) {
    const double *nna = nna_host_.data() + d * noba_short_;
    for (long iv = 0; iv < ninterval_; ++iv) {
      long ks = kstart_pp_[iv], kstop = ks + noba_pp_[iv];
      const int pf = par_.kfilter ? psd_index_global(psddet_, psdstart_, psdstop_, d, btime_[ks])
                                  : -1;
      int isub = 0;
      for (;;) {
        long noba = 0;
        bool allz = true;
        for (long k = ks; k < kstop; ++k)
          if (nna[k] != 0) { allz = false; break; }
        if (!allz) {
          while (ks < kstop && nna[ks] == 0) ++ks;
          while (kstop > ks && nna[kstop - 1] == 0) --kstop;
          noba = kstop - ks;
          long gap = 0;
          for (long i = ks; i < kstop; ++i) {
            if (nna[i] != 0) gap = 0;
            else if (++gap == gapmin) {
              noba = (i + 1) - gap - ks;
              break;
            }
          }
        }
        if (noba == 0) break;
        Segment s;
        s.det = (int)d;
        s.iv = (int)iv;
        s.isub = isub++;
        s.k0 = d * noba_short_ + ks;
        s.noba = noba;
        s.psd_filter = pf;
        s.psd_prec = par_.kfilter ? psd_index_global(psddet_, psdstart_, psdstop_, d, btime_[ks])
                                  : -1;
        const int ipd = psd_index_det(dets_[d], btime_[ks]);
        s.prec_ok = (ipd >= 0 && dets_[d].weights[ipd] != 0) ? 1 : 0;
        segs_.push_back(s);
        for (long k = 0; k < noba; ++k) rm[s.k0 + k] = 1;
        ks += noba;
      }
    }
  }
  rmask_.alloc(nb);
  MADAM_CUDA(cudaMemcpyAsync(rmask_.get(), rm.data(), nb, cudaMemcpyHostToDevice, st_));
  // convolve_interval segments (noise_routines.f90:816-857)
  filt_segs_.clear();
  for (const Segment &s : segs_) {
    if (s.psd_filter < 0) continue;
    if (s.noba > 2147483647L) fail("segment too long");
    ConvSeg c;
    c.x_off = s.k0;
    c.y_off = s.k0;
    c.n_in = (int)s.noba;
    c.n_out = (int)s.noba;
    c.spec = s.psd_filter;
    c.flags = 3;
    filt_segs_.push_back(c);
  }
  filt_segs_d_.alloc(std::max<size_t>(1, filt_segs_.size()));
  if (!filt_segs_.empty())
    MADAM_CUDA(cudaMemcpyAsync(filt_segs_d_.get(), filt_segs_.data(),
                               filt_segs_.size() * sizeof(ConvSeg), cudaMemcpyHostToDevice, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
}

void Engine::build_filter() {
  // init_filter (noise_routines.f90:242-292) + build_filter (367-739).  The
  // plateau of each PSD is found on the host; the spectra are computed on
  // the device (k_filter_spectra) and checked in build_filter_finish().  A
  // PSD table the device form does not cover (frequencies not ascending past
  // the first nonzero one, fewer than two of them) or a spectrum that is not
  // positive somewhere (which the reference fills from its neighbours) takes
  // the host's computation (filter_spectra, OpenMP over the PSDs) instead.
  filter_err_.clear();
  fcov_host_valid_ = false;
  filter_dev_ = false;
  if (fft_) fft_->forget_spectra();  // fcov is rewritten
  if (!par_.kfilter) return;
  long nof_min = 2 * noba_pp_max_;
  if (par_.precond_width_max > nof_min - 1) nof_min = par_.precond_width_max + 1;
  long nof = 1;
  while (nof < nof_min) nof *= 2;
  nof_ = std::max(4L, nof);
  npsdtot_ = 0;
  for (auto &d : dets_) npsdtot_ += d.npsd;
  const long nh = nof_ / 2 + 1;
  psddet_.assign(npsdtot_, 0);
  psdstart_.assign(npsdtot_, 0.0);
  psdstop_.assign(npsdtot_, 0.0);
  std::vector<std::pair<long, int>> tasks;
  for (long d = 0; d < ndet_; ++d) {
    if (!dets_[d].has_psd) fail("All detectors must have at least one PSD to build the filter");
    for (int ip = 0; ip < dets_[d].npsd; ++ip) tasks.push_back({d, ip});
  }
  for (long it = 0; it < (long)tasks.size(); ++it) {
    const long d = tasks[it].first;
    const int ip = tasks[it].second;
    psddet_[it] = (int)d;
    psdstart_[it] = dets_[d].psdstarts[ip];
    psdstop_[it] = (ip < dets_[d].npsd - 1) ? dets_[d].psdstarts[ip + 1] : fsp(1e30f);
  }
  filter_tasks_ = tasks;
  spectrum_file_.reset();
  if (!par_.file_spectrum.empty()) {
    // read_spectrum (noise_routines.f90:505-596): the file's sigmas replace
    // the detectors' (and their weights), and its table the PSDs; the
    // spectra are computed on the host from it (no plateau subtraction, as
    // get_spectrum_file returns the table's values)
    try {
      spectrum_file_.reset(new SpectrumFile(read_spectrum_file(par_.file_spectrum, dets_)));
    } catch (const std::exception &e) {
      filter_err_ = e.what();
      return;
    }
    for (long d = 0; d < ndet_; ++d) {
      Detector &det = dets_[d];
      const double sg = spectrum_file_->sigma[d];
      for (int ip = 0; ip < det.npsd; ++ip) {
        det.sigmas[ip] = sg;
        det.weights[ip] = 1 / (sg * sg);
      }
      if (rank() == 0) std::printf(" %s, SIGMA == %.15g\n", det.name.c_str(), sg);
    }
    std::fflush(stdout);
    filter_job_ =
        std::async(std::launch::async, [this, tasks, nh]() { filter_spectra(tasks, nh); });
    return;
  }
  // the device form: plateaus and tables on the host, spectra on the device
  const double fa = par_.fsample / (double)nshort_;
  const double margin = par_.radiometers ? fsp(1e-6f) : fsp(1e-3f);
  std::vector<FiltTask> ft(tasks.size());
  std::vector<double> tfr, tps, tlf, tlp;
  bool dev_ok = true;
  filter_sigma0_.assign(tasks.size(), 0.0);
  try {
    for (size_t it = 0; it < tasks.size() && dev_ok; ++it) {
      const long d = tasks[it].first;
      const int ip = tasks[it].second;
      const Detector &det = dets_[d];
      const std::vector<double> &fq = det.psdfreqs, &pv = det.psds[ip];
      const long nin = (long)fq.size();
      if ((long)pv.size() != nin) fail("freq and psd do not have the same shape");
      long first = 0;
      while (first < nin && fq[first] == 0) ++first;
      if (first == nin) fail("input freqs are all zero.");
      if (nin - first < 2) dev_ok = false;
      for (long i = first + 1; i < nin && dev_ok; ++i)
        if (!(fq[i] >= fq[i - 1])) dev_ok = false;
      if (!dev_ok) break;
      double plateau;
      if (par_.noise_weights_from_psd) {
        plateau = det.plateaus[ip];
      } else if (par_.radiometers) {
        const double ff = par_.fsample / 2;
        interpolate_psd(fq, pv, &ff, &plateau, 1);
      } else {
        std::vector<double> fr(1000), dt(1000);
        for (int i = 0; i < 1000; ++i) fr[i] = 1 + (double)(i * 10) / 1000;
        interpolate_psd(fq, pv, fr.data(), dt.data(), 1000);
        plateau = *std::min_element(dt.begin(), dt.end());
      }
      ft[it] = FiltTask{(int)tfr.size(), (int)nin, (int)first, plateau, det.sigmas[ip]};
      for (long i = 0; i < nin; ++i) {
        tfr.push_back(fq[i]);
        tps.push_back(pv[i]);
        tlf.push_back(std::log(fq[i]));
        tlp.push_back(std::log(pv[i]));
      }
    }
  } catch (const std::exception &e) {
    filter_err_ = e.what();  // raised where the host's spectra raise it
    return;
  }
  if (!dev_ok || tasks.empty() || tasks.size() > 65535) {  // (a grid dimension per PSD)
    filter_job_ =
        std::async(std::launch::async, [this, tasks, nh]() { filter_spectra(tasks, nh); });
    return;
  }
  for (size_t it = 0; it < tasks.size(); ++it) {
    Detector &det = dets_[tasks[it].first];
    filter_sigma0_[it] = det.sigmas[tasks[it].second];
    if (!par_.noise_weights_from_psd)
      det.sigmas[tasks[it].second] = std::sqrt(ft[it].plateau * par_.fsample);
  }
  filter_dev_ = true;
  DevBuf<FiltTask> dft;
  DevBuf<double> tab;
  const size_t nt = tfr.size();
  dft.alloc(ft.size());
  tab.alloc(4 * nt);
  MADAM_CUDA(cudaMemcpyAsync(dft.get(), ft.data(), ft.size() * sizeof(FiltTask),
                             cudaMemcpyHostToDevice, st_));
  const std::vector<double> *parts[4] = {&tfr, &tps, &tlf, &tlp};
  for (int q = 0; q < 4; ++q)
    MADAM_CUDA(cudaMemcpyAsync(tab.get() + q * nt, parts[q]->data(), nt * sizeof(double),
                               cudaMemcpyHostToDevice, st_));
  fcov_.alloc((size_t)nh * npsdtot_);
  filter_flag_.alloc(1);
  filter_flag_.zero(st_);
  const unsigned gx = (unsigned)std::min<long>((nh + 255) / 256, 4096);
  MADAM_LAUNCH(k_filter_spectra, dim3(gx, (unsigned)tasks.size()), 256, 0, st_, dft.get(),
               tab.get(), tab.get() + nt, tab.get() + 2 * nt, tab.get() + 3 * nt, nof_, nh, fa,
               margin, fcov_.get(), filter_flag_.get());
}

// The host copy of the filter's spectra (the covariance output and the
// "fcov" result read it).
const std::vector<double> &Engine::fcov_host() {
  if (!fcov_host_valid_ && filter_dev_ && fcov_.n) {
    fcov_host_.resize(fcov_.n);
    MADAM_CUDA(cudaMemcpyAsync(fcov_host_.data(), fcov_.get(), fcov_.n * sizeof(double),
                               cudaMemcpyDeviceToHost, st_));
    MADAM_CUDA(cudaStreamSynchronize(st_));
  }
  fcov_host_valid_ = true;
  return fcov_host_;
}

const std::vector<double> &Engine::invcov_host() {
  if (invcov_valid_ && invcov_host_.empty() && invcov_.n) {
    invcov_host_.resize((size_t)nof_ * npsdtot_);
    MADAM_CUDA(cudaMemcpyAsync(invcov_host_.data(), invcov_.get(),
                               invcov_host_.size() * sizeof(double), cudaMemcpyDeviceToHost, st_));
    MADAM_CUDA(cudaStreamSynchronize(st_));
  }
  return invcov_host_;
}

void Engine::filter_spectra(const std::vector<std::pair<long, int>> &tasks, long nh) {
  const double fa = par_.fsample / (double)nshort_;
  const double kPi = 3.141592653589793238462643383279502884197;
  std::string err;
  fcov_host_.assign((size_t)nh * npsdtot_, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
  for (long it = 0; it < (long)tasks.size(); ++it) {
    try {
      const long d = tasks[it].first;
      const int ip = tasks[it].second;
      Detector &det = dets_[d];  // this task's entries only
      const double sigma = det.sigmas[ip];
      std::vector<double> aspec(nh, 0.0), f(nof_), g(nof_), spec(nof_);
      for (int k = 0; k <= 2; ++k) {
        for (long i = 0; i < nof_; ++i) f[i] = k * fa + (double)i * fa / (double)nof_;
        if (spectrum_file_) {
          // get_spectrum_file (noise_routines.f90:600-634): the table's
          // spectrum as it stands
          spectrum_from_file(*spectrum_file_, (int)d, f.data(), spec.data(), nof_);
          for (long i = 0; i < nof_; ++i) {
            const double x = kPi * f[i] / fa;
            g[i] = (x < fsp(1e-30f)) ? 1.0 : std::sin(x) * std::sin(x) / (x * x);
          }
          if (k == 0) aspec[0] = spec[0];
          else aspec[0] = aspec[0] + 2 * spec[0] * g[0];
          for (long i = 1; i < nh; ++i)
            aspec[i] = aspec[i] + spec[i] * g[i] + spec[nof_ - i] * g[nof_ - i];
          continue;
        }
        // get_spectrum_interp (noise_routines.f90:638-737)
        interpolate_psd(det.psdfreqs, det.psds[ip], f.data(), spec.data(), nof_);
        double plateau;
        if (par_.noise_weights_from_psd) {
          plateau = det.plateaus[ip];
        } else {
          if (par_.radiometers) {
            const double ff = par_.fsample / 2;
            interpolate_psd(det.psdfreqs, det.psds[ip], &ff, &plateau, 1);
          } else {
            std::vector<double> fr(1000), dt(1000);
            for (int i = 0; i < 1000; ++i) fr[i] = 1 + (double)(i * 10) / 1000;
            interpolate_psd(det.psdfreqs, det.psds[ip], fr.data(), dt.data(), 1000);
            plateau = *std::min_element(dt.begin(), dt.end());
          }
          det.sigmas[ip] = std::sqrt(plateau * par_.fsample);
        }
        const double margin = par_.radiometers ? fsp(1e-6f) : fsp(1e-3f);
        bool anyneg = false;
        for (long i = 0; i < nof_; ++i) {
          spec[i] = (spec[i] > plateau * (1 + margin)) ? spec[i] - plateau : spec[i] * margin;
          if (spec[i] <= 0) anyneg = true;
        }
        if (anyneg) {
          for (long i = 0; i < nof_; ++i) {
            if (spec[i] <= 0) {
              bool found = false;
              for (long j = i + 1; j < nof_; ++j)
                if (spec[j] > 0) { spec[i] = spec[j]; found = true; break; }
              if (found) continue;
            }
            if (spec[i] <= 0)
              for (long j = i - 1; j >= 0; --j)
                if (spec[j] > 0) { spec[i] = spec[j]; break; }
          }
        }
        if (f[0] == 0) spec[0] = 0;
        for (long i = 0; i < nof_; ++i) {
          const double x = kPi * f[i] / fa;
          g[i] = (x < fsp(1e-30f)) ? 1.0 : std::sin(x) * std::sin(x) / (x * x);
        }
        if (k == 0) aspec[0] = spec[0];
        else aspec[0] = aspec[0] + 2 * spec[0] * g[0];
        for (long i = 1; i < nh; ++i)
          aspec[i] = aspec[i] + spec[i] * g[i] + spec[nof_ - i] * g[nof_ - i];
      }
      for (long i = 0; i < nh; ++i)
        aspec[i] = (std::fabs(aspec[i]) > sigma * fsp(1e-30f)) ? 1.0 / (fa * aspec[i]) : 0.0;
      aspec[0] = 0;
      for (long i = 0; i < nh; ++i) {
        if (std::isnan(aspec[i])) fail("NaN in fcov. Check input PSD and sigma.");
        fcov_host_[(size_t)it * nh + i] = aspec[i];
      }
    } catch (const std::exception &e) {
#pragma omp critical
      err = e.what();
    }
  }
  filter_err_ = err;
}

void Engine::build_filter_finish() {
  if (!par_.kfilter) return;
  if (filter_dev_) {
    int flag = 0;
    MADAM_CUDA(cudaMemcpyAsync(&flag, filter_flag_.get(), sizeof flag, cudaMemcpyDeviceToHost,
                               st_));
    MADAM_CUDA(cudaStreamSynchronize(st_));
    if (flag & 1) {
      // a spectrum that is not positive somewhere: the host's computation
      // with the reference's fill (from the sigmas the filter started from)
      for (size_t it = 0; it < filter_tasks_.size(); ++it)
        dets_[filter_tasks_[it].first].sigmas[filter_tasks_[it].second] = filter_sigma0_[it];
      filter_dev_ = false;
      filter_spectra(filter_tasks_, nof_ / 2 + 1);
    } else if (flag & 2) {
      fail("NaN in fcov. Check input PSD and sigma.");
    }
  } else if (filter_job_.valid()) {
    filter_job_.get();
  }
  if (!filter_err_.empty()) fail(filter_err_);
  if (!filter_dev_) {
    fcov_.alloc(fcov_host_.size());
    MADAM_CUDA(cudaMemcpyAsync(fcov_.get(), fcov_host_.data(),
                               fcov_host_.size() * sizeof(double), cudaMemcpyHostToDevice, st_));
    fcov_host_valid_ = true;
  }
  fft_.reset(new FFTPlan(nof_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
}

void Engine::construct_preconditioner() {
  // construct_preconditioner (noise_routines.f90:920-1153)
  invcov_valid_ = false;
  invcov_host_.clear();
  band_segs_.clear();
  cg_prec_segs_.clear();
  band_widths_.clear();
  n_band_fail_ = 0;
  use_diagonal_ = false;
  if (nbasis_ > 1) return;  // the F^T F inverses precondition (initialize_a_basis)
  const long long nb = (long long)ndet_ * noba_short_;
  if (par_.precond_width_max < 1) return;
  if (!par_.kfilter || par_.precond_width_max == 1) {
    use_diagonal_ = true;
    std::vector<double> pd(nb, 0.0);
    for (long d = 0; d < ndet_; ++d)
      for (long iv = 0; iv < ninterval_; ++iv) {
        const long ks = kstart_pp_[iv];
        const int ipd = psd_index_det(dets_[d], btime_[ks]);
        for (long k = ks; k < ks + noba_pp_[iv]; ++k) {
          const size_t o = d * noba_short_ + k;
          if (ipd < 0) pd[o] = 1.;
          else if (nna_host_[o] == 0) pd[o] = 1. / dets_[d].weights[ipd];
          else pd[o] = 1. / nna_host_[o];
        }
      }
    prec_diag_.alloc(nb);
    MADAM_CUDA(cudaMemcpyAsync(prec_diag_.get(), pd.data(), nb * sizeof(double),
                               cudaMemcpyHostToDevice, st_));
    MADAM_CUDA(cudaStreamSynchronize(st_));
    return;
  }
  const long nh = nof_ / 2 + 1;
  {
    std::vector<double> w(npsdtot_);
    long ip = 0;
    for (long d = 0; d < ndet_; ++d)
      for (int k = 0; k < dets_[d].npsd; ++k, ++ip) w[ip] = dets_[d].weights[k];
    DevBuf<double> wd;
    wd.alloc(std::max<long>(1, npsdtot_));
    MADAM_CUDA(cudaMemcpyAsync(wd.get(), w.data(), npsdtot_ * sizeof(double),
                               cudaMemcpyHostToDevice, st_));
    if (fft_) fft_->forget_spectra();  // fprec is rewritten
    fprec_.alloc((size_t)nh * npsdtot_);
    MADAM_LAUNCH(k_fprec, grid_for((long long)nh * npsdtot_), 256, 0, st_, fcov_.get(), wd.get(),
                 nh, (long)npsdtot_, (double)nshort_, fprec_.get());
    MADAM_CUDA(cudaStreamSynchronize(st_));
  }
  if (par_.use_fprecond) {
    MADAM_CUDA(cudaStreamSynchronize(st_));
    return;
  }
  // invcov = c2r(fcov): convolution of a unit impulse without mean removal
  invcov_.alloc((size_t)nof_ * npsdtot_);
  delta_.alloc(1);
  const double one = 1.0;
  MADAM_CUDA(cudaMemcpyAsync(delta_.get(), &one, sizeof one, cudaMemcpyHostToDevice, st_));
  std::vector<ConvSeg> ic(npsdtot_);
  for (long ip = 0; ip < npsdtot_; ++ip) {
    ic[ip].x_off = 0;
    ic[ip].y_off = ip * nof_;
    ic[ip].n_in = 1;
    ic[ip].n_out = (int)nof_;
    ic[ip].spec = (int)ip;
    ic[ip].flags = 0;
  }
  convolve(delta_.get(), invcov_.get(), ic, fcov_.get(), tmp_segs_d_);
  invcov_host_.clear();  // copied to the host only when asked for (result "invcov")
  invcov_valid_ = true;
  // the kernels' power sums, in the host's order of summation
  const long pw_w = std::max<long>(1, std::min<long>(nof_, par_.precond_width_max));
  std::vector<double> ptot(npsdtot_), ppre((size_t)npsdtot_ * pw_w);
  {
    DevBuf<double> dpt, dpre;
    dpt.alloc(std::max<long>(1, npsdtot_));
    dpre.alloc(std::max<size_t>(1, ppre.size()));
    if (npsdtot_ > 0)
      MADAM_LAUNCH(k_invcov_power, (unsigned)npsdtot_, 256, 0, st_, invcov_.get(), nof_, pw_w,
                   dpt.get(), dpre.get());
    MADAM_CUDA(cudaMemcpyAsync(ptot.data(), dpt.get(), npsdtot_ * sizeof(double),
                               cudaMemcpyDeviceToHost, st_));
    MADAM_CUDA(cudaMemcpyAsync(ppre.data(), dpre.get(), ppre.size() * sizeof(double),
                               cudaMemcpyDeviceToHost, st_));
    MADAM_CUDA(cudaStreamSynchronize(st_));
  }
  trace("precond: fprec+invcov");
  // candidate segments
  std::vector<int> cand;
  for (int i = 0; i < (int)segs_.size(); ++i) {
    const Segment &s = segs_[i];
    if (s.psd_prec == -1) continue;  // nothing is built (preconditioning falls back to CG)
    cand.push_back(i);
  }
  if (par_.use_cgprecond) {
    for (int i : cand) cg_prec_segs_.push_back(i);
    return;
  }
  const double plim = (double)(1.0f - 1e-5f);
  struct Try { int seg; long nband; int tr; };
  std::vector<Try> todo;
  for (int i : cand) {
    const Segment &s = segs_[i];
    const double p_tot = ptot[s.psd_prec];
    const double *pre = ppre.data() + (size_t)s.psd_prec * pw_w;
    long tr = 1, nband = 0;
    bool ok = false;
    for (;;) {
      nband = std::min(s.noba, tr * par_.precond_width_min);
      nband = std::min(nband, par_.precond_width_max);
      const double pp = nband > 0 ? pre[nband - 1] : 0.0;
      if (pp > plim * p_tot) { ok = true; break; }
      if (nband == s.noba || nband == par_.precond_width_max) break;
      if (tr == 1000) break;
      ++tr;
    }
    if (ok) todo.push_back({i, nband, (int)tr});
    else {
      cg_prec_segs_.push_back(i);
      ++n_band_fail_;
    }
  }
  // factor; segments that are not positive definite get a wider band
  // (noise_routines.f90:1092-1120).  Band widths up to kBand2MaxWidth use the
  // deduplicated factor (band2.cu), wider ones the plain column store.
  struct Done2 { int seg; PSeg ps; size_t round; int nu, nr; };
  struct Done1 { int seg; BandSeg bs; size_t round; };
  std::vector<std::unique_ptr<DevBuf<double>>> rows_r;
  std::vector<std::unique_ptr<DevBuf<PRun>>> runs_r;
  std::vector<std::unique_ptr<DevBuf<double>>> band_r;
  std::vector<Done2> done2;
  std::vector<Done1> done1;
  while (!todo.empty()) {
    std::vector<Try> t2, t1, next;
    for (const Try &t : todo) (t.nband <= kBand2MaxWidth ? t2 : t1).push_back(t);
    std::vector<int> stat2, stat1, nu2, nr2;
    std::vector<PSeg> ps(t2.size());
    std::vector<BandSeg> bs(t1.size());
    if (!t2.empty()) {
      std::vector<int> spec(t2.size());
      long long roff = 0;
      int runoff = 0;
      for (size_t t = 0; t < t2.size(); ++t) {
        const Segment &sg = segs_[t2[t].seg];
        ps[t] = PSeg{sg.k0, roff, (int)sg.noba, (int)t2[t].nband, runoff, 0, 0, 0, 0, 0};
        spec[t] = sg.psd_prec;
        roff += (long long)sg.noba * (t2[t].nband + 1);
        runoff += (int)sg.noba;
      }
      DevBuf<PSeg> dps;
      DevBuf<int> dspec, dstat, dnu, dnr;
      rows_r.emplace_back(new DevBuf<double>());
      runs_r.emplace_back(new DevBuf<PRun>());
      rows_r.back()->alloc(std::max<long long>(1, roff));
      runs_r.back()->alloc(std::max(1, runoff));
      dps.alloc(ps.size());
      dspec.alloc(ps.size());
      dstat.alloc(ps.size());
      dnu.alloc(ps.size());
      dnr.alloc(ps.size());
      MADAM_CUDA(cudaMemcpyAsync(dps.get(), ps.data(), ps.size() * sizeof(PSeg),
                                 cudaMemcpyHostToDevice, st_));
      MADAM_CUDA(cudaMemcpyAsync(dspec.get(), spec.data(), spec.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, st_));
      band2_factor(st_, dps.get(), (int)ps.size(), dspec.get(), invcov_.get(), nof_, nna_.get(),
                   rows_r.back()->get(), runs_r.back()->get(), dstat.get(), dnu.get(), dnr.get());
      stat2.resize(ps.size());
      nu2.resize(ps.size());
      nr2.resize(ps.size());
      MADAM_CUDA(cudaMemcpyAsync(stat2.data(), dstat.get(), ps.size() * sizeof(int),
                                 cudaMemcpyDeviceToHost, st_));
      MADAM_CUDA(cudaMemcpyAsync(nu2.data(), dnu.get(), ps.size() * sizeof(int),
                                 cudaMemcpyDeviceToHost, st_));
      MADAM_CUDA(cudaMemcpyAsync(nr2.data(), dnr.get(), ps.size() * sizeof(int),
                                 cudaMemcpyDeviceToHost, st_));
      MADAM_CUDA(cudaStreamSynchronize(st_));
    }
    if (!t1.empty()) {
      std::vector<int> spec(t1.size());
      long long off = 0;
      for (size_t t = 0; t < t1.size(); ++t) {
        const Segment &sg = segs_[t1[t].seg];
        bs[t] = BandSeg{sg.k0, off, (int)sg.noba, (int)t1[t].nband};
        spec[t] = sg.psd_prec;
        off += (long long)sg.noba * t1[t].nband;
      }
      DevBuf<BandSeg> dbs;
      DevBuf<int> dspec, dstat;
      band_r.emplace_back(new DevBuf<double>());
      band_r.back()->alloc(off);
      dbs.alloc(bs.size());
      dspec.alloc(bs.size());
      dstat.alloc(bs.size());
      MADAM_CUDA(cudaMemcpyAsync(dbs.get(), bs.data(), bs.size() * sizeof(BandSeg),
                                 cudaMemcpyHostToDevice, st_));
      MADAM_CUDA(cudaMemcpyAsync(dspec.get(), spec.data(), spec.size() * sizeof(int),
                                 cudaMemcpyHostToDevice, st_));
      band_factor(st_, dbs.get(), (int)bs.size(), dspec.get(), invcov_.get(), nof_, nna_.get(),
                  band_r.back()->get(), dstat.get());
      stat1.resize(bs.size());
      MADAM_CUDA(cudaMemcpyAsync(stat1.data(), dstat.get(), stat1.size() * sizeof(int),
                                 cudaMemcpyDeviceToHost, st_));
      MADAM_CUDA(cudaStreamSynchronize(st_));
    }
    auto retry = [&](Try nt) {
      const Segment &sg = segs_[nt.seg];
      if (nt.tr == 1000 || nt.nband == sg.noba || nt.nband == par_.precond_width_max) {
        cg_prec_segs_.push_back(nt.seg);
        ++n_band_fail_;
      } else {
        ++nt.tr;
        nt.nband = std::min(nt.nband + par_.precond_width_min, par_.precond_width_max);
        next.push_back(nt);
      }
    };
    for (size_t t = 0; t < t2.size(); ++t) {
      if (stat2[t] == 0) {
        done2.push_back({t2[t].seg, ps[t], rows_r.size() - 1, nu2[t], nr2[t]});
        band_widths_.push_back(t2[t].nband);
      } else {
        retry(t2[t]);
      }
    }
    for (size_t t = 0; t < t1.size(); ++t) {
      if (stat1[t] == 0) {
        done1.push_back({t1[t].seg, bs[t], band_r.size() - 1});
        band_widths_.push_back(t1[t].nband);
      } else {
        retry(t1[t]);
      }
    }
    todo.swap(next);
  }
  trace("precond: factor");
  // pack the deduplicated factors the apply step uses (prec_ok segments),
  // ordered by register width class so that each class's chunks are contiguous
  struct Pack { const Done2 *dn; std::vector<PRun> rl; int W; };
  std::vector<Pack> packs;
  long nmax = 0;
  for (const Done2 &dn : done2) {
    if (!segs_[dn.seg].prec_ok) continue;
    Pack pk{&dn, std::vector<PRun>(dn.nr), band2_class_width(dn.ps.nb - 1)};
    MADAM_CUDA(cudaMemcpy(pk.rl.data(), runs_r[dn.round]->get() + dn.ps.run_off,
                          dn.nr * sizeof(PRun), cudaMemcpyDeviceToHost));
    nmax = std::max<long>(nmax, dn.ps.n);
    packs.push_back(std::move(pk));
  }
  auto cls_key = [](int W) { return W == 0 ? INT_MAX : W; };
  std::stable_sort(packs.begin(), packs.end(),
                   [&](const Pack &a, const Pack &b) { return cls_key(a.W) < cls_key(b.W); });
  // chunk length ~ sqrt(n / 4): balances the chunk passes (latency-bound
  // recurrences, ~85 ns per position) against the state scan (~90 ns per
  // chunk)
  int C = 64;
  while (C < 4096 && (long)C * C * 4 < nmax) C *= 2;
  std::vector<PSeg> pseg;
  std::vector<PRun> pruns, cruns;
  std::vector<PChunk> chunks;
  std::vector<PTrans> trans;
  long long tab_end = 0, nunique = 0;
  for (const Pack &pk : packs) {
    PSeg q = pk.dn->ps;
    q.row_off = tab_end;
    tab_end += (long long)pk.dn->nu * (q.nb + 1);
    nunique += pk.dn->nu;
    pseg.push_back(q);
  }
  band2_cls_w_.clear();
  band2_cls_begin_.clear();
  band2_cls_seg_.clear();
  std::vector<int> tcls_begin;
  int max_ncrun = 0;
  std::map<std::pair<long long, int>, long long> tcache;
  long long toff = 0;
  for (size_t si = 0; si < packs.size(); ++si) {
    const Pack &pk = packs[si];
    PSeg &q = pseg[si];
    const int n = q.n, w = q.nb - 1, S = q.nb + 1;
    if (band2_cls_w_.empty() || band2_cls_w_.back() != pk.W) {
      band2_cls_w_.push_back(pk.W);
      band2_cls_begin_.push_back((int)chunks.size());
      band2_cls_seg_.push_back((int)si);
      tcls_begin.push_back((int)trans.size());
    }
    q.run_off = (int)pruns.size();
    q.nrun = pk.dn->nr;
    for (PRun r : pk.rl) {
      r.off = r.off - pk.dn->ps.row_off + q.row_off;
      r.fill = 0;
      pruns.push_back(r);
    }
    // backward runs (p = n - 1 - j ascending): column j is row j's entry
    // while rows j..j+w are one run; the w columns before each run's end
    // (and the segment end) are assembled
    q.crun_off = (int)cruns.size();
    for (int ri = q.nrun - 1; ri >= 0; --ri) {
      const int s0 = pruns[q.run_off + ri].start;
      const int e0 = ri + 1 < q.nrun ? pruns[q.run_off + ri + 1].start : n;
      for (int j = e0 - 1; j >= std::max(s0, e0 - w); --j) {
        cruns.push_back({n - 1 - j, 1, tab_end});
        tab_end += S;
      }
      if (e0 - w - 1 >= s0) cruns.push_back({n - 1 - (e0 - w - 1), 0, pruns[q.run_off + ri].off});
    }
    q.ncrun = (int)cruns.size() - q.crun_off;
    max_ncrun = std::max(max_ncrun, q.ncrun);
    auto find = [](const std::vector<PRun> &v, int lo, int hi, int pos) {
      while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (v[mid].start <= pos) lo = mid;
        else hi = mid - 1;
      }
      return lo;
    };
    q.nch = (n + C - 1) / C;
    q.ch_off = (int)chunks.size();
    for (int c = 0; c < q.nch; ++c) {
      PChunk k;
      k.seg = (int)si;
      k.a = c * C;
      k.b = std::min(n, k.a + C);
      k.run_f = find(pruns, q.run_off, q.run_off + q.nrun - 1, k.a);
      k.run_b = find(cruns, q.crun_off, q.crun_off + q.ncrun - 1, n - k.b);
      k.first = c == 0;
      k.last = c == q.nch - 1;
      k.tf = k.tb = 0;
      if (!k.first && !k.last && w > 0) {
        const int ci = (int)chunks.size();
        // a chunk inside one run has the transfer matrix of that entry and
        // length, whichever direction
        const bool steady_f =
            find(pruns, q.run_off, q.run_off + q.nrun - 1, k.b - 1) == k.run_f && k.b - k.a == C;
        const bool steady_b =
            find(cruns, q.crun_off, q.crun_off + q.ncrun - 1, n - k.a - 1) == k.run_b &&
            k.b - k.a == C;
        for (int dir = 0; dir < 2; ++dir) {
          const bool steady = dir == 0 ? steady_f : steady_b;
          const long long eoff = dir == 0 ? pruns[k.run_f].off : cruns[k.run_b].off;
          long long off = -1;
          if (steady) {
            auto it = tcache.find({eoff, q.nb});
            if (it != tcache.end()) off = it->second;
          }
          if (off < 0) {
            off = toff;
            toff += (long long)w * w;
            trans.push_back({ci, dir, off});
            if (steady) tcache[{eoff, q.nb}] = off;
          }
          (dir == 0 ? k.tf : k.tb) = (int)off;
        }
      }
      chunks.push_back(k);
    }
  }
  band2_cls_begin_.push_back((int)chunks.size());
  band2_cls_seg_.push_back((int)pseg.size());
  tcls_begin.push_back((int)trans.size());
  if (toff >= (1LL << 31)) fail("too many band transfer matrices");
  p2nseg_ = (int)pseg.size();
  p2nch_ = (int)chunks.size();
  p2segs_.alloc(std::max<size_t>(1, pseg.size()));
  p2runs_.alloc(std::max<size_t>(1, pruns.size()));
  p2cruns_.alloc(std::max<size_t>(1, cruns.size()));
  p2ch_.alloc(std::max<size_t>(1, chunks.size()));
  p2rows_.alloc(std::max<long long>(1, tab_end));
  p2T_.alloc(std::max<long long>(1, toff));
  p2wp_.alloc((size_t)std::max(1, p2nch_) * kBand2State);
  p2ws_.alloc((size_t)std::max(1, p2nch_) * kBand2State);
  if (!pseg.empty()) {
    for (size_t si = 0; si < packs.size(); ++si) {
      const Done2 &dn = *packs[si].dn;
      MADAM_CUDA(cudaMemcpyAsync(p2rows_.get() + pseg[si].row_off,
                                 rows_r[dn.round]->get() + dn.ps.row_off,
                                 (size_t)dn.nu * (dn.ps.nb + 1) * sizeof(double),
                                 cudaMemcpyDeviceToDevice, st_));
    }
    MADAM_CUDA(cudaMemcpyAsync(p2segs_.get(), pseg.data(), pseg.size() * sizeof(PSeg),
                               cudaMemcpyHostToDevice, st_));
    MADAM_CUDA(cudaMemcpyAsync(p2runs_.get(), pruns.data(), pruns.size() * sizeof(PRun),
                               cudaMemcpyHostToDevice, st_));
    MADAM_CUDA(cudaMemcpyAsync(p2cruns_.get(), cruns.data(), cruns.size() * sizeof(PRun),
                               cudaMemcpyHostToDevice, st_));
    MADAM_CUDA(cudaMemcpyAsync(p2ch_.get(), chunks.data(), chunks.size() * sizeof(PChunk),
                               cudaMemcpyHostToDevice, st_));
    std::vector<int> tf(chunks.size()), tb(chunks.size());
    for (size_t c = 0; c < chunks.size(); ++c) {
      tf[c] = chunks[c].tf;
      tb[c] = chunks[c].tb;
    }
    p2tf_.alloc(tf.size());
    p2tb_.alloc(tb.size());
    MADAM_CUDA(cudaMemcpyAsync(p2tf_.get(), tf.data(), tf.size() * sizeof(int),
                               cudaMemcpyHostToDevice, st_));
    MADAM_CUDA(cudaMemcpyAsync(p2tb_.get(), tb.data(), tb.size() * sizeof(int),
                               cudaMemcpyHostToDevice, st_));
    band2_columns(st_, p2segs_.get(), p2nseg_, max_ncrun, p2runs_.get(), p2cruns_.get(),
                  p2rows_.get());
    DevBuf<PTrans> dtr;
    dtr.alloc(std::max<size_t>(1, trans.size()));
    if (!trans.empty()) {
      MADAM_CUDA(cudaMemcpyAsync(dtr.get(), trans.data(), trans.size() * sizeof(PTrans),
                                 cudaMemcpyHostToDevice, st_));
      band2_transfer(st_, p2segs_.get(), p2ch_.get(), dtr.get(), band2_cls_w_.data(),
                     tcls_begin.data(), (int)band2_cls_w_.size(), p2runs_.get(), p2cruns_.get(),
                     p2rows_.get(), p2T_.get());
    }
    MADAM_CUDA(cudaStreamSynchronize(st_));
  }
  band2_pseg_h_ = pseg;
  band2_ch_h_ = chunks;
  batch_tables_r_ = 0;
  band2_rows_ = nunique;
  band2_ntrans_ = (long)trans.size();
  band2_chunk_ = C;
  trace("precond: scan tables");
  build_guarded_chunks(pruns, cruns);
  trace("precond: guarded chunks");
  // plain column store for the wide bands
  long long total = 0;
  band_segs_.clear();
  std::vector<const Done1 *> keep;
  for (const Done1 &dn : done1) {
    if (!segs_[dn.seg].prec_ok) continue;
    BandSeg b = dn.bs;
    b.l_off = total;
    total += (long long)b.n * b.nband;
    band_segs_.push_back(b);
    keep.push_back(&dn);
  }
  band_.alloc(std::max<long long>(1, total));
  for (size_t j = 0; j < keep.size(); ++j)
    MADAM_CUDA(cudaMemcpyAsync(band_.get() + band_segs_[j].l_off,
                               band_r[keep[j]->round]->get() + keep[j]->bs.l_off,
                               (size_t)band_segs_[j].n * band_segs_[j].nband * sizeof(double),
                               cudaMemcpyDeviceToDevice, st_));
  band_segs_d_.alloc(std::max<size_t>(1, band_segs_.size()));
  if (!band_segs_.empty())
    MADAM_CUDA(cudaMemcpyAsync(band_segs_d_.get(), band_segs_.data(),
                               band_segs_.size() * sizeof(BandSeg), cudaMemcpyHostToDevice, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  // segments without a factor that the apply step reaches use the CG fallback
  std::vector<int> cgk;
  for (int i : cg_prec_segs_)
    if (segs_[i].prec_ok) cgk.push_back(i);
  cg_prec_segs_ = cgk;
}

void Engine::finish_dots(int nd, int mode, int slot0, int nblk, bool global) {
  if (!global || !sharded()) {
    MADAM_LAUNCH(k_finish, 1, 1024, 0, st_, part_.get(), nblk, nd, scal_.get(), mode, slot0);
    return;
  }
  // the rank's partial sums, summed over the ranks, then the CG scalars
  // (sum_mpi of the inner products, smadam_routines.f90:865-901)
  const int dst = mode == 0 ? slot0 : S_SHARD;
  MADAM_LAUNCH(k_finish, 1, 1024, 0, st_, part_.get(), nblk, nd, scal_.get(), 0, dst);
  ar_sum(scal_.get() + dst, nd);
  if (mode != 0) MADAM_LAUNCH(k_finish_apply, 1, 32, 0, st_, scal_.get(), mode, S_SHARD);
}

double Engine::ar_sum_host(double v) {
  if (!sharded()) return v;
  DevBuf<double> t;
  t.alloc(1);
  MADAM_CUDA(cudaMemcpyAsync(t.get(), &v, sizeof v, cudaMemcpyHostToDevice, st_));
  ar_sum(t.get(), 1);
  MADAM_CUDA(cudaMemcpyAsync(&v, t.get(), sizeof v, cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  return v;
}

void Engine::scatter_baselines(const double *pw, double *target, bool fine) {
  if (nwork_ == 0) return;
  const int T = 1 << tile_shift_;
  const int deg = fine ? 0 : (int)ndeg_shift_;
  const int tilec = std::max(1, T >> deg);
  const size_t smem = (size_t)tilec * nmap_ * sizeof(double);
  if (nmap_ == 3)
    MADAM_LAUNCH(k_scatter<3>, (unsigned)nwork_, 256, smem, st_, item_begin_.get(),
                 item_tile_.get(), runs_.get(), point4_.get(), pixc_.get(), pw, fdn_, tile_shift_,
                 deg, tilec, target);
  else
    MADAM_LAUNCH(k_scatter<1>, (unsigned)nwork_, 256, smem, st_, item_begin_.get(),
                 item_tile_.get(), runs_.get(), point4_.get(), pixc_.get(), pw, fdn_, tile_shift_,
                 deg, tilec, target);
}

void Engine::convolve(const double *x, double *y, const std::vector<ConvSeg> &segs,
                      const double *spectra, DevBuf<ConvSeg> &dsegs) {
  if (segs.empty()) return;
  if (dsegs.n < segs.size()) dsegs.alloc(segs.size());
  MADAM_CUDA(cudaMemcpyAsync(dsegs.get(), segs.data(), segs.size() * sizeof(ConvSeg),
                             cudaMemcpyHostToDevice, st_));
  fft_->convolve(st_, dsegs.get(), (long)segs.size(), spectra, npsdtot_, x, y);
}

void Engine::apply_A(const double *p, const double *pw, double *ap, bool timed) {
  if (nbasis_ > 1) return apply_A_basis(p, ap, timed);
  const long long nb = (long long)ndet_ * noba_short_;
  // 1) baseline -> map, collect, ccmultiply, scatter back (iterate_a 798-827)
  if (timed) MADAM_CUDA(cudaEventRecord(ev_[0], st_));
  if (nscatter_chunks_ == 0 && nloc_cross_ > 0) lmap_.zero(st_);  // a rank with no samples
  if (nloc_cross_ > 0 && nscatter_chunks_ > 0) {
    // the grid from the launch-shape tuner (tuned_grid; the chunks' sums do
    // not depend on it)
    if (nmap_ == 3) {
      tuned_grid((const void *)k_scatter_chunks<3>, 10, nscatter_chunks_, 1, [&](unsigned g) {
        MADAM_LAUNCH(k_scatter_chunks<3>, g, 256, 0, st_, scatter_chunks_.get(),
                     nscatter_chunks_, sp4_.get(), sp2_.get(), pw, lmap_.get(),
                     scatter_partial_.get());
      });
      if (nscatter_multi_ > 0)
        MADAM_LAUNCH(k_scatter_combine<3>, grid_for(nscatter_multi_), 256, 0, st_,
                     scatter_multi_.get(), nscatter_multi_, scatter_partial_.get(), lmap_.get());
    } else {
      tuned_grid((const void *)k_scatter_chunks<1>, 11, nscatter_chunks_, 1, [&](unsigned g) {
        MADAM_LAUNCH(k_scatter_chunks<1>, g, 256, 0, st_, scatter_chunks_.get(),
                     nscatter_chunks_, sp4_.get(), sp2_.get(), pw, lmap_.get(),
                     scatter_partial_.get());
      });
      if (nscatter_multi_ > 0)
        MADAM_LAUNCH(k_scatter_combine<1>, grid_for(nscatter_multi_), 256, 0, st_,
                     scatter_multi_.get(), nscatter_multi_, scatter_partial_.get(), lmap_.get());
    }
  }
  ar_sum(lmap_.get(), (size_t)nloc_cross_ * nmap_);  // collect_map across the ranks
  if (timed) MADAM_CUDA(cudaEventRecord(ev_[1], st_));
  if (nloc_cross_ > 0) {
    if (nmap_ == 3 && fp32_)
      MADAM_LAUNCH(k_ccmult_copy<true>, grid_for(nloc_cross_), 256, 0, st_, cca_.get(),
                   lmap_.get(), (long long)nloc_cross_, (double2 *)nullptr, lmapf_.get());
    else if (nmap_ == 3)
      MADAM_LAUNCH(k_ccmult_copy<false>, grid_for(nloc_cross_), 256, 0, st_, cca_.get(),
                   lmap_.get(), (long long)nloc_cross_, lmapg_.get(), (float4 *)nullptr);
    else
      MADAM_LAUNCH(k_ccmult<1>, grid_for(nloc_cross_), 256, 0, st_, cca_.get(), lmap_.get(),
                   (long long)nloc_cross_);
  }
  // 2) noise prior: ap = C_a^-1 p (cinvmul, 829-845)
  if (timed) MADAM_CUDA(cudaEventRecord(ev_[2], st_));
  if (par_.kfilter) {
    MADAM_CUDA(cudaMemcpyAsync(ap, p, nb * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    if (!filt_segs_.empty())
      fft_->convolve(st_, filt_segs_d_.get(), (long)filt_segs_.size(), fcov_.get(), npsdtot_, p,
                     ap);
  } else if (par_.diagfilter != 0) {
    MADAM_LAUNCH(k_diagfilter, grid_for(nb), 256, 0, st_, ap, nna_.get(), p, par_.diagfilter, nb);
  } else {
    MADAM_CUDA(cudaMemsetAsync(ap, 0, nb * sizeof(double), st_));
  }
  if (timed) MADAM_CUDA(cudaEventRecord(ev_[3], st_));
  // 3) map -> baseline and p.ap (849-878)
  if (use_pairs_) {
    MADAM_LAUNCH(k_gather_pairs, kRedBlocks, 256, 0, st_, pair_chunks_.get(), npair_chunks_,
                 gp4_.get(), poff_.get(), bw_.get(), p, nna_.get(), lmapf_.get(), rmask_.get(),
                 ap, part_.get());
  } else if (ngather_chunks_ > 0) {
    if (nmap_ == 3 && fp32_)
      MADAM_LAUNCH((k_gather_chunks<3, float4>), kGatherChunkBlocks, 256, 0, st_, gather_chunks_.get(),
                   ngather_chunks_, point4_.get(), pixc_.get(), bstart_d_.get(), noba_short_,
                   nsamp_, bw_.get(), p, nna_.get(), lmap_.get(), lmapf_.get(),
                   (int)ndeg_shift_, (int)nloc_, rmask_.get(), ap, part_.get());
    else if (nmap_ == 3)
      MADAM_LAUNCH((k_gather_chunks<3, double2>), kGatherChunkBlocks, 256, 0, st_, gather_chunks_.get(),
                   ngather_chunks_, point4_.get(), pixc_.get(), bstart_d_.get(), noba_short_,
                   nsamp_, bw_.get(), p, nna_.get(), lmap_.get(), lmapg_.get(),
                   (int)ndeg_shift_, (int)nloc_, rmask_.get(), ap, part_.get());
    else
      MADAM_LAUNCH((k_gather_chunks<1, double2>), kGatherChunkBlocks, 256, 0, st_, gather_chunks_.get(),
                   ngather_chunks_, point4_.get(), pixc_.get(), bstart_d_.get(), noba_short_,
                   nsamp_, bw_.get(), p, nna_.get(), lmap_.get(), (const double2 *)nullptr,
                   (int)ndeg_shift_, (int)nloc_, rmask_.get(), ap, part_.get());
  } else if (gather_kb_ > 0) {
    if (nmap_ == 3)
      MADAM_LAUNCH(k_gather_tiled<3>, kRedBlocks, 256, 0, st_, point4_.get(), pixc_.get(),
                   bstart_d_.get(), noba_short_, nsamp_, gather_kb_, gather_tiles_det_,
                   (int)ndet_, bw_.get(), p, nna_.get(), lmap_.get(), (int)ndeg_shift_,
                   (int)nloc_, rmask_.get(), ap, part_.get());
    else
      MADAM_LAUNCH(k_gather_tiled<1>, kRedBlocks, 256, 0, st_, point4_.get(), pixc_.get(),
                   bstart_d_.get(), noba_short_, nsamp_, gather_kb_, gather_tiles_det_,
                   (int)ndet_, bw_.get(), p, nna_.get(), lmap_.get(), (int)ndeg_shift_,
                   (int)nloc_, rmask_.get(), ap, part_.get());
  } else if (nmap_ == 3) {
    MADAM_LAUNCH(k_gather<3>, kRedBlocks, 256, 0, st_, point4_.get(), pixc_.get(),
                 bstart_d_.get(), nb, noba_short_, nsamp_, bw_.get(), p, nna_.get(), lmap_.get(),
                 (int)ndeg_shift_, (int)nloc_, rmask_.get(), ap, part_.get());
  } else {
    MADAM_LAUNCH(k_gather<1>, kRedBlocks, 256, 0, st_, point4_.get(), pixc_.get(),
                 bstart_d_.get(), nb, noba_short_, nsamp_, bw_.get(), p, nna_.get(), lmap_.get(),
                 (int)ndeg_shift_, (int)nloc_, rmask_.get(), ap, part_.get());
  }
  finish_dots(1, 1, 0, (!use_pairs_ && ngather_chunks_ > 0) ? kGatherChunkBlocks : kRedBlocks,
              true);
  if (timed) MADAM_CUDA(cudaEventRecord(ev_[4], st_));
}

// A x with float64 projections over the exact sample pointing (the caller's
// float32 weights, float64 map and baseline values): the operator of the
// float64 path, for the true residual of the FP32-TOD forms' reliable
// updates.  Works in its own buffers, so the PCG's vectors and its last
// A p map (wamap) are left alone.
void Engine::apply_A_exact(const double *x, double *ax) {
  const long long nb = (long long)ndet_ * noba_short_;
  const long ncross = std::max<long>(1, nloc_cross_);
  pwx_.alloc(std::max<long long>(1, nb));
  lmapx_.alloc((size_t)ncross * nmap_);
  partx_.alloc(3 * kRedBlocks);
  if (nmap_ == 3) lmapgx_.alloc((size_t)ncross * 2);
  MADAM_LAUNCH(k_mul, grid_for(nb), 256, 0, st_, pwx_.get(), x, bw_.get(), nb);
  // 1) baseline -> map over the samples: the pixel-sorted samples when the
  // scatter has them, else the time-ordered runs (pairs round the weights)
  if (nloc_cross_ > 0) {
    if (have_xcsr_ || (!use_pairs_ && nscatter_chunks_ > 0)) {
      // the pixel-sorted samples (kept beside the pairs in the FP32-TOD form)
      DevBuf<int4> &ck = have_xcsr_ ? xscatter_chunks_ : scatter_chunks_;
      DevBuf<int4> &mu = have_xcsr_ ? xscatter_multi_ : scatter_multi_;
      DevBuf<double> &pa = have_xcsr_ ? xscatter_partial_ : scatter_partial_;
      const float4 *q4 = have_xcsr_ ? xsp4_.get() : sp4_.get();
      const int2 *q2 = have_xcsr_ ? xsp2_.get() : sp2_.get();
      const long long nck = have_xcsr_ ? xnscatter_chunks_ : nscatter_chunks_;
      const int nmu = have_xcsr_ ? xnscatter_multi_ : nscatter_multi_;
      if (nmap_ == 3) {
        if (nck > 0)
          MADAM_LAUNCH(k_scatter_chunks<3>, kRedBlocks, 256, 0, st_, ck.get(), nck, q4, q2,
                       pwx_.get(), lmapx_.get(), pa.get());
        if (nmu > 0)
          MADAM_LAUNCH(k_scatter_combine<3>, grid_for(nmu), 256, 0, st_, mu.get(), nmu,
                       pa.get(), lmapx_.get());
      } else {
        if (nck > 0)
          MADAM_LAUNCH(k_scatter_chunks<1>, kRedBlocks, 256, 0, st_, ck.get(), nck, q4, q2,
                       pwx_.get(), lmapx_.get(), pa.get());
        if (nmu > 0)
          MADAM_LAUNCH(k_scatter_combine<1>, grid_for(nmu), 256, 0, st_, mu.get(), nmu,
                       pa.get(), lmapx_.get());
      }
    } else {
      lmapx_.zero(st_);
      scatter_baselines(pwx_.get(), lmapx_.get(), false);
    }
  }
  ar_sum(lmapx_.get(), (size_t)nloc_cross_ * nmap_);
  if (nloc_cross_ > 0) {
    if (nmap_ == 3)
      MADAM_LAUNCH(k_ccmult_copy<false>, grid_for(nloc_cross_), 256, 0, st_, cca_.get(),
                   lmapx_.get(), (long long)nloc_cross_, lmapgx_.get(), (float4 *)nullptr);
    else
      MADAM_LAUNCH(k_ccmult<1>, grid_for(nloc_cross_), 256, 0, st_, cca_.get(), lmapx_.get(),
                   (long long)nloc_cross_);
  }
  // 2) noise prior
  if (par_.kfilter) {
    MADAM_CUDA(cudaMemcpyAsync(ax, x, nb * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    if (!filt_segs_.empty())
      fft_->convolve(st_, filt_segs_d_.get(), (long)filt_segs_.size(), fcov_.get(), npsdtot_, x,
                     ax);
  } else if (par_.diagfilter != 0) {
    MADAM_LAUNCH(k_diagfilter, grid_for(nb), 256, 0, st_, ax, nna_.get(), x, par_.diagfilter, nb);
  } else {
    MADAM_CUDA(cudaMemsetAsync(ax, 0, nb * sizeof(double), st_));
  }
  // 3) map -> baseline over the samples (the partial x.Ax sums are not used)
  if (ngather_chunks_ > 0) {
    if (nmap_ == 3)
      MADAM_LAUNCH((k_gather_chunks<3, double2>), kGatherChunkBlocks, 256, 0, st_,
                   gather_chunks_.get(), ngather_chunks_, point4_.get(), pixc_.get(),
                   bstart_d_.get(), noba_short_, nsamp_, bw_.get(), x, nna_.get(), lmapx_.get(),
                   lmapgx_.get(), (int)ndeg_shift_, (int)nloc_, rmask_.get(), ax, partx_.get());
    else
      MADAM_LAUNCH((k_gather_chunks<1, double2>), kGatherChunkBlocks, 256, 0, st_,
                   gather_chunks_.get(), ngather_chunks_, point4_.get(), pixc_.get(),
                   bstart_d_.get(), noba_short_, nsamp_, bw_.get(), x, nna_.get(), lmapx_.get(),
                   (const double2 *)nullptr, (int)ndeg_shift_, (int)nloc_, rmask_.get(), ax,
                   partx_.get());
  } else if (gather_kb_ > 0) {
    if (nmap_ == 3)
      MADAM_LAUNCH(k_gather_tiled<3>, kRedBlocks, 256, 0, st_, point4_.get(), pixc_.get(),
                   bstart_d_.get(), noba_short_, nsamp_, gather_kb_, gather_tiles_det_,
                   (int)ndet_, bw_.get(), x, nna_.get(), lmapx_.get(), (int)ndeg_shift_,
                   (int)nloc_, rmask_.get(), ax, partx_.get());
    else
      MADAM_LAUNCH(k_gather_tiled<1>, kRedBlocks, 256, 0, st_, point4_.get(), pixc_.get(),
                   bstart_d_.get(), noba_short_, nsamp_, gather_kb_, gather_tiles_det_,
                   (int)ndet_, bw_.get(), x, nna_.get(), lmapx_.get(), (int)ndeg_shift_,
                   (int)nloc_, rmask_.get(), ax, partx_.get());
  } else if (nmap_ == 3) {
    MADAM_LAUNCH(k_gather<3>, kRedBlocks, 256, 0, st_, point4_.get(), pixc_.get(),
                 bstart_d_.get(), nb, noba_short_, nsamp_, bw_.get(), x, nna_.get(),
                 lmapx_.get(), (int)ndeg_shift_, (int)nloc_, rmask_.get(), ax, partx_.get());
  } else {
    MADAM_LAUNCH(k_gather<1>, kRedBlocks, 256, 0, st_, point4_.get(), pixc_.get(),
                 bstart_d_.get(), nb, noba_short_, nsamp_, bw_.get(), x, nna_.get(),
                 lmapx_.get(), (int)ndeg_shift_, (int)nloc_, rmask_.get(), ax, partx_.get());
  }
}

// r = b - A x with the float64 operator (apply_A_exact)
void Engine::true_residual(const double *x, const double *b, double *r) {
  const long long nb = (long long)ndet_ * noba_short_;
  apx_.alloc(std::max<long long>(1, nb));
  apply_A_exact(x, apx_.get());
  MADAM_LAUNCH(k_residual, grid_for(nb), 256, 0, st_, r, b, apx_.get(), nb);
  ++n_reliable_;
}

// Chunks of the guarded band solve.  The factor's rows settle to a fixed
// point whose recurrence forgets its state geometrically (at the 1/f priors
// of the benchmarked workloads by 1e-17 within about 200 positions), so a
// chunk can start its recurrence a guard of G positions early from a zero
// state instead of waiting for the true state: every chunk is independent
// and the solve is two launches, forward and backward, without transfer
// matrices or state scans.  The guard is checked at set-up for every chunk
// start a multiple of kGuardGrain rows (and every backward end the same
// distance from the segment end), so that chunks of any multiple of
// kGuardGrain rows are covered: the state a unit state at the guard start
// leaves at the chunk's first written position stays below kBand2GuardTol.
// G = 256, 512, 1024 are tried; if none passes everywhere (or a band is
// wider than the register classes) the state-scan solve stays in use.
// MADAM_B200_BAND_SOLVE=scan selects the state-scan solve.
namespace {
constexpr int kGuardGrain = 128;
}  // namespace

std::vector<GChunk> Engine::make_gchunks(int Cg, int G, std::vector<int> &cls_begin,
                                         std::vector<int> &seg_off) const {
  auto find = [](const std::vector<PRun> &v, int lo, int hi, int pos) {
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (v[mid].start <= pos) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  };
  const std::vector<PSeg> &pseg = band2_pseg_h_;
  const std::vector<PRun> &pr = band2_pruns_h_, &cr = band2_cruns_h_;
  std::vector<GChunk> gcs;
  cls_begin.clear();
  seg_off.clear();
  for (size_t ci = 0; ci + 1 < band2_cls_seg_.size(); ++ci) {
    cls_begin.push_back((int)gcs.size());
    for (int si = band2_cls_seg_[ci]; si < band2_cls_seg_[ci + 1]; ++si) {
      const PSeg &q = pseg[si];
      const int n = q.n;
      seg_off.push_back((int)gcs.size());
      for (int a = 0; a < n; a += Cg) {
        GChunk k;
        k.seg = si;
        k.a = a;
        k.b = std::min(n, a + Cg);
        k.ga = std::max(0, a - G);
        k.run_fg = find(pr, q.run_off, q.run_off + q.nrun - 1, k.ga);
        k.run_fa = find(pr, q.run_off, q.run_off + q.nrun - 1, k.a);
        k.gp = std::max(0, n - k.b - G);
        k.run_bg = find(cr, q.crun_off, q.crun_off + q.ncrun - 1, k.gp);
        k.run_bb = find(cr, q.crun_off, q.crun_off + q.ncrun - 1, n - k.b);
        gcs.push_back(k);
      }
    }
  }
  cls_begin.push_back((int)gcs.size());
  seg_off.push_back((int)gcs.size());
  return gcs;
}

// chunk length for npos positions in all: a multiple of kGuardGrain rows
// giving at most one resident wave of the guarded kernel (a warp of 32
// chunks per block, about 8 blocks per SM at its shared-memory size), so
// that no second wave's tail idles the SMs; up to 4096 rows
int Engine::guard_chunk_len(long long npos) const {
  const long long maxchains = 148LL * 8 * 32;
  const long long units = (npos + kGuardGrain * maxchains - 1) / (kGuardGrain * maxchains);
  return (int)std::min<long long>(4096, kGuardGrain * std::max<long long>(1, units));
}

void Engine::build_guarded_chunks(const std::vector<PRun> &pruns,
                                  const std::vector<PRun> &cruns) {
  band2_guarded_ = false;
  band2_gch_h_.clear();
  band2_gcls_begin_.clear();
  band2_gseg_off_.clear();
  p2gc_.reset();
  const std::vector<PSeg> &pseg = band2_pseg_h_;
  if (pseg.empty()) return;
  const char *mode = std::getenv("MADAM_B200_BAND_SOLVE");
  if (mode && std::string(mode) == "scan") return;
  for (int W : band2_cls_w_)
    if (W == 0) return;
  band2_pruns_h_ = pruns;
  band2_cruns_h_ = cruns;
  DevBuf<double> worst;
  DevBuf<GChunk> dgc;
  for (int G = 256; G <= 1024; G *= 2) {
    std::vector<int> gb, soff;
    std::vector<GChunk> gcs = make_gchunks(kGuardGrain, G, gb, soff);
    if (gcs.empty()) return;
    dgc.alloc(gcs.size());
    MADAM_CUDA(cudaMemcpyAsync(dgc.get(), gcs.data(), gcs.size() * sizeof(GChunk),
                               cudaMemcpyHostToDevice, st_));
    worst.alloc(gcs.size());
    band2_guard_check(st_, p2segs_.get(), dgc.get(), band2_cls_w_.data(), gb.data(),
                      (int)band2_cls_w_.size(), p2runs_.get(), p2cruns_.get(), p2rows_.get(),
                      worst.get());
    std::vector<double> wh(gcs.size());
    MADAM_CUDA(cudaMemcpyAsync(wh.data(), worst.get(), wh.size() * sizeof(double),
                               cudaMemcpyDeviceToHost, st_));
    MADAM_CUDA(cudaStreamSynchronize(st_));
    bool ok = true;
    for (double v : wh) ok = ok && v < kBand2GuardTol;
    if (!ok) continue;
    long long npos = 0;
    for (const PSeg &q : pseg) npos += q.n;
    band2_guarded_ = true;
    band2_guard_ = G;
    band2_err_.alloc(1);
    band2_err_.zero(st_);
    band2_gchunk_ = guard_chunk_len(npos);
    band2_gch_h_ = make_gchunks(band2_gchunk_, G, band2_gcls_begin_, band2_gseg_off_);
    p2gc_.alloc(band2_gch_h_.size());
    MADAM_CUDA(cudaMemcpyAsync(p2gc_.get(), band2_gch_h_.data(),
                               band2_gch_h_.size() * sizeof(GChunk), cudaMemcpyHostToDevice,
                               st_));
    MADAM_CUDA(cudaStreamSynchronize(st_));
    return;
  }
}

// The guarded band solve's staging waits are bounded; one that ran out
// leaves a flag (never seen in practice), checked once per solve.
void Engine::check_band_err() {
  if (!band2_guarded_ || !band2_err_.get()) return;
  int e = 0;
  MADAM_CUDA(cudaMemcpyAsync(&e, band2_err_.get(), sizeof e, cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  if (e) {
    band2_err_.zero(st_);
    fail("band preconditioner: a staging wait of the guarded solve ran out");
  }
}

// checknan (parameter_control.f90:321-330, smadam_routines.f90:456-502,
// 740 / 978-1033): NaN counts of the detector parameters, of the right-hand
// side, the binned map and the pointing weights after initialize_a, and of
// the first CG vectors, reported as the reference reports them (a message
// per kind on standard output; the solve goes on) and kept as "nan_checks".
unsigned long long Engine::count_nan(const double *v, long long n) {
  if (n <= 0 || !v) return 0;
  DevBuf<unsigned long long> c;
  c.alloc(1);
  c.zero(st_);
  MADAM_LAUNCH(k_count_nan<double>, grid_for(n), 256, 0, st_, v, n, c.get());
  unsigned long long h = 0;
  MADAM_CUDA(cudaMemcpyAsync(&h, c.get(), sizeof h, cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  return h;
}

unsigned long long Engine::count_nan(const float *v, long long n) {
  if (n <= 0 || !v) return 0;
  DevBuf<unsigned long long> c;
  c.alloc(1);
  c.zero(st_);
  MADAM_LAUNCH(k_count_nan<float>, grid_for(n), 256, 0, st_, v, n, c.get());
  unsigned long long h = 0;
  MADAM_CUDA(cudaMemcpyAsync(&h, c.get(), sizeof h, cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  return h;
}

void Engine::check_nan_setup() {
  nan_checks_.assign(kNanChecks, 0.0);
  if (!par_.checknan) return;
  for (const Detector &d : dets_) {
    bool bad = false;
    for (double w : d.weights) bad = bad || std::isnan(w);
    for (double s : d.sigmas) bad = bad || std::isnan(s);
    if (bad) {
      std::printf("%d : Bad detector params (NaN in sigmas or weights) : %s\n", rank(),
                  d.name.c_str());
      nan_checks_[0] += 1;
    }
  }
  const long long nb = (long long)ndet_ * noba_short_ * nbasis_;
  nan_checks_[1] = (double)count_nan(yba_.get(), nb);
  nan_checks_[2] = (double)count_nan(wamap_.get(), (long long)wamap_.n);
  if (nmap_ != 1) nan_checks_[3] = (double)count_nan(d_w_, (long long)ndet_ * nsamp_ * nnz_);
  if (nan_checks_[1] > 0) std::printf("%d : NaN in uninitialized yba\n", rank());
  if (nan_checks_[2] > 0) std::printf("%d : NaN in locmap\n", rank());
  if (nan_checks_[3] > 0) std::printf("%d : NaN in weights\n", rank());
  std::fflush(stdout);
}

void Engine::check_nan_iterate(double rz, long long nb) {
  if (!par_.checknan) return;
  if (std::isnan(rz)) std::printf("%d : ERROR: rz is nan\n", rank());
  nan_checks_[4] = (double)count_nan(r_.get(), nb);
  nan_checks_[5] = (double)count_nan(z_.get(), nb);
  nan_checks_[6] = (double)count_nan(p_.get(), nb);
  if (nan_checks_[1] > 0) std::printf("%d : yba has NaN(s)\n", rank());
  if (nan_checks_[4] > 0) std::printf("%d : r has NaN(s)\n", rank());
  if (nan_checks_[5] > 0) std::printf("%d : z has NaN(s)\n", rank());
  if (nan_checks_[6] > 0) std::printf("%d : p has NaN(s)\n", rank());
  std::fflush(stdout);
}

void Engine::cg_preconditioner_segments(const double *r, double *z) {
  if (cg_prec_segs_.empty()) return;
  const long long nb = (long long)ndet_ * noba_short_;
  if (!cgp_) cgp_.reset(new CgpWork());
  CgpWork &w = *cgp_;
  if (w.nseg != (long)cg_prec_segs_.size()) {
    std::vector<CgpSeg> hs;
    w.hcsegs.clear();
    for (int i : cg_prec_segs_) {
      const Segment &s = segs_[i];
      hs.push_back({s.k0, (int)s.noba, s.psd_prec});
      ConvSeg c;
      c.x_off = s.k0;
      c.y_off = s.k0;
      c.n_in = (int)s.noba;
      c.n_out = (int)s.noba;
      c.spec = s.psd_prec;
      c.flags = 3;
      w.hcsegs.push_back(c);
    }
    w.nseg = (long)hs.size();
    w.segs.alloc(hs.size());
    MADAM_CUDA(cudaMemcpyAsync(w.segs.get(), hs.data(), hs.size() * sizeof(CgpSeg),
                               cudaMemcpyHostToDevice, st_));
    w.csegs.alloc(w.hcsegs.size());
    MADAM_CUDA(cudaMemcpyAsync(w.csegs.get(), w.hcsegs.data(), w.hcsegs.size() * sizeof(ConvSeg),
                               cudaMemcpyHostToDevice, st_));
    for (auto *b : {&w.x, &w.resid, &w.prop, &w.aprop, &w.zres, &w.prec}) b->alloc(nb);
    w.st.alloc(4 * w.nseg);
    w.done.alloc(w.nseg);
    w.active.alloc(1);
  }
  const unsigned ns = (unsigned)w.nseg;
  MADAM_LAUNCH(k_cgp_init, ns, 256, 0, st_, w.segs.get(), r, w.x.get(), w.resid.get(),
               w.prop.get(), w.zres.get(), w.prec.get(), nna_.get(), invcov_.get(),
               (long long)nof_, w.st.get(), w.done.get());
  for (int iter = 1; iter <= 100; ++iter) {
    fft_->convolve(st_, w.csegs.get(), w.nseg, fcov_.get(), npsdtot_, w.prop.get(),
                   w.aprop.get());
    MADAM_CUDA(cudaMemsetAsync(w.active.get(), 0, sizeof(int), st_));
    MADAM_LAUNCH(k_cgp_step, ns, 256, 0, st_, w.segs.get(), w.x.get(), w.resid.get(),
                 w.prop.get(), w.aprop.get(), w.zres.get(), w.prec.get(), nna_.get(), w.st.get(),
                 w.done.get(), iter, w.active.get());
    int active = 0;
    MADAM_CUDA(cudaMemcpyAsync(&active, w.active.get(), sizeof(int), cudaMemcpyDeviceToHost, st_));
    MADAM_CUDA(cudaStreamSynchronize(st_));
    if (active == 0) break;
  }
  MADAM_LAUNCH(k_copy_seg, ns, 256, 0, st_, w.segs.get(), w.x.get(), z);
}

void Engine::apply_preconditioner(const double *r, double *z) {
  // preconditioning_band (noise_routines.f90:1159-1256)
  if (nbasis_ > 1) return precondition_basis(r, z);
  const long long nb = (long long)ndet_ * noba_short_;
  if (par_.precond_width_max < 1) {
    MADAM_CUDA(cudaMemcpyAsync(z, r, nb * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    return;
  }
  if (use_diagonal_) {
    MADAM_LAUNCH(k_mul, grid_for(nb), 256, 0, st_, z, r, prec_diag_.get(), nb);
    return;
  }
  MADAM_CUDA(cudaMemcpyAsync(z, r, nb * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  if (par_.use_fprecond) {
    if (!filt_segs_.empty())
      fft_->convolve(st_, filt_segs_d_.get(), (long)filt_segs_.size(), fprec_.get(), npsdtot_, r,
                     z);
    return;
  }
  if (band2_guarded_) {
    p2y_.alloc(std::max<long long>(1, nb));
    band2_solve_guarded(st_, p2segs_.get(), p2gc_.get(), band2_cls_w_.data(),
                        band2_gcls_begin_.data(), (int)band2_cls_w_.size(), p2runs_.get(),
                        p2cruns_.get(), p2rows_.get(), r, p2y_.get(), z, band2_err_.get());
  } else {
    band2_solve(st_, p2segs_.get(), p2nseg_, p2ch_.get(), p2nch_, p2tf_.get(), p2tb_.get(),
                band2_cls_w_.data(),
                band2_cls_begin_.data(), band2_cls_seg_.data(), (int)band2_cls_w_.size(),
                p2runs_.get(), p2cruns_.get(), p2rows_.get(), p2T_.get(), r, z, p2wp_.get(),
                p2ws_.get());
  }
  band_solve(st_, band_segs_d_.get(), (int)band_segs_.size(), band_.get(), r, z);
  cg_preconditioner_segments(r, z);
}

void Engine::iterate() {
  // iterate_a (smadam_routines.f90:677-983); nb counts the CG vectors'
  // amplitudes (basis_order + 1 per baseline)
  double t0 = now_ms();
  const long long nb = (long long)ndet_ * noba_short_ * nbasis_;
  const double *bwv = bw_.get();
  const uint8_t *rmv = rmask_.get();
  if (nbasis_ > 1) {
    basis_vectors();
    bwv = bwn_.get();
    rmv = rmaskn_.get();
  }
  for (auto *b : {&r_, &p_, &z_, &ap_, &ro_, &pw_}) b->alloc(std::max<long long>(1, nb));
  part_.alloc(3 * kRedBlocks);
  scal_.alloc(S_NSCAL);
  scal_.zero(st_);
  lmap_.alloc((size_t)std::max<long>(1, nloc_cross_) * nmap_);
  if (nmap_ == 3) {
    if (fp32_) lmapf_.alloc((size_t)std::max<long>(1, nloc_cross_));
    else lmapg_.alloc((size_t)std::max<long>(1, nloc_cross_) * 2);
  }
  MADAM_CUDA(cudaMemcpyAsync(r_.get(), yba_.get(), nb * sizeof(double), cudaMemcpyDeviceToDevice,
                             st_));
  aa_.zero(st_);
  apply_preconditioner(r_.get(), z_.get());
  MADAM_LAUNCH(k_update_p, grid_for(nb), 256, 0, st_, p_.get(), z_.get(), pw_.get(), bwv,
               nb, scal_.get(), 1);
  MADAM_LAUNCH(k_dots, kRedBlocks, 256, 0, st_, r_.get(), z_.get(), r_.get(), r_.get(), nullptr,
               nullptr, 2, rmv, nb, part_.get());
  finish_dots(2, 0, S_RZ, kRedBlocks, true);
  scal_host_.assign(S_NSCAL, 0.0);
  MADAM_CUDA(cudaMemcpyAsync(scal_host_.data(), scal_.get(), S_NSCAL * sizeof(double),
                             cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  const double rzinit = scal_host_[S_RZ];
  rrinit = scal_host_[S_RR];
  rr_final = 1.0;
  noiter = 0;
  check_nan_iterate(rzinit, nb);
  if (rzinit < fsp(1e-30f) || std::isnan(rzinit)) {
    timings.iterate_ms = now_ms() - t0;
    return;
  }
  long istep = 0;
  float tm[4];
  pcg_reset();
  if (nloc_cross_ > 0 && nscatter_chunks_ > 0 && !sharded() &&
      !tuned(nmap_ == 3 ? 10 : 11, nscatter_chunks_, 1)) {
    // the scatter's launch shape, tuned once per shape (a pass of A p whose
    // outputs the first iteration overwrites); counted in the setup time
    const double tt = now_ms();
    tune_batch_ = true;
    try {
      apply_A(p_.get(), pw_.get(), ap_.get(), false);
    } catch (...) {
      tune_batch_ = false;
      throw;
    }
    tune_batch_ = false;
    MADAM_CUDA(cudaStreamSynchronize(st_));
    timings.setup_ms += now_ms() - tt;
    t0 += now_ms() - tt;
  }
  while (istep < par_.iter_max) {
    ++istep;
    apply_A(p_.get(), pw_.get(), ap_.get(), true);
    MADAM_LAUNCH(k_update_ar, grid_for(nb), 256, 0, st_, aa_.get(), r_.get(), ro_.get(), p_.get(),
                 ap_.get(), nb, scal_.get());
    MADAM_CUDA(cudaEventRecord(ev_[5], st_));
    apply_preconditioner(r_.get(), z_.get());
    MADAM_CUDA(cudaEventRecord(ev_[6], st_));
    MADAM_LAUNCH(k_dots, kRedBlocks, 256, 0, st_, r_.get(), z_.get(), ro_.get(), z_.get(),
                 r_.get(), r_.get(), 3, rmv, nb, part_.get());
    finish_dots(3, 2, 0, kRedBlocks, true);
    MADAM_CUDA(cudaMemcpyAsync(scal_host_.data(), scal_.get(), S_NSCAL * sizeof(double),
                               cudaMemcpyDeviceToHost, st_));
    MADAM_CUDA(cudaStreamSynchronize(st_));
    MADAM_CUDA(cudaEventElapsedTime(&tm[0], ev_[0], ev_[1]));
    MADAM_CUDA(cudaEventElapsedTime(&tm[1], ev_[2], ev_[3]));
    MADAM_CUDA(cudaEventElapsedTime(&tm[2], ev_[3], ev_[4]));
    MADAM_CUDA(cudaEventElapsedTime(&tm[3], ev_[5], ev_[6]));
    timings.scatter_ms += tm[0];
    timings.filter_ms += tm[1];
    timings.gather_ms += tm[2];
    timings.precond_ms += tm[3];
    if (pcg_stop_test(istep, scal_host_[S_RZ], scal_host_[S_RR])) break;
    MADAM_LAUNCH(k_update_p, grid_for(nb), 256, 0, st_, p_.get(), z_.get(), pw_.get(), bwv,
                 nb, scal_.get(), 0);
  }
  check_band_err();
  // iterate_a leaves wamap holding the last A.p map (collect_map + ccmultiply
  // on wamap, smadam_routines.f90:818-822); destripe_with_cache adds the new
  // binned map onto it (smadam.F90:719-732)
  if (istep > 0)
    MADAM_CUDA(cudaMemcpyAsync(wamap_.get(), lmap_.get(), wamap_.n * sizeof(double),
                               cudaMemcpyDeviceToDevice, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  timings.iterate_ms = now_ms() - t0;
}

// The step after a PCG iteration's inner products (iterate_a 890-924):
// reliable update of the FP32-TOD form, history, divergence and convergence
// tests.  Returns true when the iteration stops.
void Engine::pcg_reset() {
  // FP32-TOD form: reliable updates each time the carried residual norm has
  // dropped by kReliableDrop (squared) since the last true one, and before
  // convergence is accepted
  pcg_reliable_ = refine() && nbasis_ == 1;
  pcg_rr_true_ = rrinit;
  n_reliable_ = 0;
}

bool Engine::pcg_stop_test(long istep, double rz, double rr) {
  if (pcg_reliable_ && ((rr / rrinit < par_.cglimit && istep > par_.iter_min) ||
                        rr < kReliableDrop * pcg_rr_true_)) {
    // reliable update: the residual the float32 projections carried is
    // replaced by the true one, so that convergence is tested, and the
    // iteration continues, on the float64 system
    const long long nb = (long long)ndet_ * noba_short_ * nbasis_;
    true_residual(aa_.get(), yba_.get(), r_.get());
    apply_preconditioner(r_.get(), z_.get());
    MADAM_LAUNCH(k_dots, kRedBlocks, 256, 0, st_, r_.get(), z_.get(), ro_.get(), z_.get(),
                 r_.get(), r_.get(), 3, rmask_.get(), nb, part_.get());
    finish_dots(3, 3, 0, kRedBlocks, true);
    MADAM_CUDA(cudaMemcpyAsync(scal_host_.data(), scal_.get(), S_NSCAL * sizeof(double),
                               cudaMemcpyDeviceToHost, st_));
    MADAM_CUDA(cudaStreamSynchronize(st_));
    rz = scal_host_[S_RZ];
    rr = scal_host_[S_RR];
    pcg_rr_true_ = rr;
  }
  rr_history.push_back(rr / rrinit);
  rr_final = rr / rrinit;
  noiter = istep;
  if (rr / rrinit > 1e3) fail("CG is diverging");
  if (rr / rrinit < par_.cglimit && istep > par_.iter_min) return true;
  return rz == 0;
}

// ---------------------------------------------------------- stepwise PCG --
// The serving stepper advances the PCG of several engines in rounds: per
// round every engine's A p (pcg_apply) and preconditioner (pcg_precond) on a
// stream the stepper picks, the vector algebra of all of them in shared
// launches (pcg_shared), one host synchronisation, then pcg_after for each.
// The arithmetic is that of iterate(): the same kernels, grids and reduction
// order, so a job's products do not depend on the others in its rounds.
bool Engine::stepwise_ok() const {
  return par_.kfirst && par_.file_covmat.empty() && !sharded();
}

bool Engine::pcg_begin() {
  const double t0 = now_ms();
  pcg_t0_ = t0;
  const long long nb = (long long)ndet_ * noba_short_ * nbasis_;
  pcg_bw_ = bw_.get();
  pcg_rmask_ = rmask_.get();
  if (nbasis_ > 1) {
    basis_vectors();
    pcg_bw_ = bwn_.get();
    pcg_rmask_ = rmaskn_.get();
  }
  for (auto *b : {&r_, &p_, &z_, &ap_, &ro_, &pw_}) b->alloc(std::max<long long>(1, nb));
  part_.alloc(3 * kRedBlocks);
  scal_.alloc(S_NSCAL);
  scal_.zero(st_);
  lmap_.alloc((size_t)std::max<long>(1, nloc_cross_) * nmap_);
  if (nmap_ == 3) {
    if (fp32_) lmapf_.alloc((size_t)std::max<long>(1, nloc_cross_));
    else lmapg_.alloc((size_t)std::max<long>(1, nloc_cross_) * 2);
  }
  MADAM_CUDA(cudaMemcpyAsync(r_.get(), yba_.get(), nb * sizeof(double), cudaMemcpyDeviceToDevice,
                             st_));
  aa_.zero(st_);
  apply_preconditioner(r_.get(), z_.get());
  MADAM_LAUNCH(k_update_p, grid_for(nb), 256, 0, st_, p_.get(), z_.get(), pw_.get(), pcg_bw_,
               nb, scal_.get(), 1);
  MADAM_LAUNCH(k_dots, kRedBlocks, 256, 0, st_, r_.get(), z_.get(), r_.get(), r_.get(), nullptr,
               nullptr, 2, pcg_rmask_, nb, part_.get());
  finish_dots(2, 0, S_RZ, kRedBlocks, true);
  scal_host_.assign(S_NSCAL, 0.0);
  MADAM_CUDA(cudaMemcpyAsync(scal_host_.data(), scal_.get(), S_NSCAL * sizeof(double),
                             cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  const double rzinit = scal_host_[S_RZ];
  rrinit = scal_host_[S_RR];
  rr_final = 1.0;
  noiter = 0;
  pcg_istep_ = 0;
  check_nan_iterate(rzinit, nb);
  pcg_reset();
  return !(rzinit < fsp(1e-30f) || std::isnan(rzinit)) && par_.iter_max > 0;
}

void Engine::pcg_use_stream(cudaStream_t s) {
  if (!pcg_own_st_) pcg_own_st_ = st_;
  st_ = s ? s : pcg_own_st_;
  g_alloc_stream = st_;
}

void Engine::pcg_apply() {
  ++pcg_istep_;
  apply_A(p_.get(), pw_.get(), ap_.get(), false);
}

void Engine::pcg_precond() { apply_preconditioner(r_.get(), z_.get()); }

PcgJob Engine::pcg_job() {
  PcgJob j{};
  j.aa = aa_.get();
  j.r = r_.get();
  j.ro = ro_.get();
  j.p = p_.get();
  j.ap = ap_.get();
  j.z = z_.get();
  j.pw = pw_.get();
  j.bw = pcg_bw_;
  j.rmask = pcg_rmask_;
  j.part = part_.get();
  j.scal = scal_.get();
  j.nb = (long long)ndet_ * noba_short_ * nbasis_;
  j.active = 1;
  return j;
}

bool Engine::pcg_after(double rz, double rr) {
  return pcg_stop_test(pcg_istep_, rz, rr) || pcg_istep_ >= par_.iter_max;
}

void Engine::pcg_end() {
  check_band_err();
  if (pcg_istep_ > 0)
    MADAM_CUDA(cudaMemcpyAsync(wamap_.get(), lmap_.get(), wamap_.n * sizeof(double),
                               cudaMemcpyDeviceToDevice, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  pcg_use_stream(nullptr);
  pcg_own_st_ = nullptr;
  timings.iterate_ms = now_ms() - pcg_t0_;
}

void pcg_shared(cudaStream_t st, const PcgJob *tab, int n, long long nbmax, int step,
                double *out) {
  if (n <= 0) return;
  if (n > 65535) fail("too many jobs in one stepper round");
  if (step == 0) {
    MADAM_LAUNCH(k_pcg_update_ar_j, dim3(grid_for(nbmax), (unsigned)n), 256, 0, st, tab);
  } else if (step == 1) {
    MADAM_LAUNCH(k_pcg_dots_j, dim3(kRedBlocks, (unsigned)n), 256, 0, st, tab);
    MADAM_LAUNCH(k_pcg_finish_j, (unsigned)n, 1024, 0, st, tab, kRedBlocks, out);
  } else {
    MADAM_LAUNCH(k_pcg_update_p_j, dim3(grid_for(nbmax), (unsigned)n), 256, 0, st, tab);
  }
}

void Engine::subtract_baselines() {
  // subtract_baselines_a (smadam_routines.f90:1489-1539)
  const long long nb = (long long)ndet_ * noba_short_;
  lmap_fine_.alloc((size_t)std::max<long>(1, nloc_) * nmap_);
  lmap_fine_.zero(st_);
  if (nbasis_ > 1) {
    scatter_basis(aa_.get(), -1.0, lmap_fine_.get(), true);
  } else {
    tmpv_.alloc(nb);
    MADAM_LAUNCH(k_scale_neg, grid_for(nb), 256, 0, st_, aa_.get(), bw_.get(), tmpv_.get(), nb);
    scatter_baselines(tmpv_.get(), lmap_fine_.get(), true);
  }
  const long long nv = (long long)nloc_ * nmap_;
  ar_sum(lmap_fine_.get(), (size_t)nv);
  if (nv > 0) MADAM_LAUNCH(k_add, grid_for(nv), 256, 0, st_, map_.get(), lmap_fine_.get(), nv);
}

void Engine::clean_tod() {
  // clean_tod (smadam_routines.f90:1545-1585)
  if (!par_.write_tod && par_.ndetset == 0 && par_.nsurvey == 0) return;
  if (!par_.kfirst || tod_cleaned_) return;
  if (isubchunk_ > 0) return;  // only the full-data pass cleans (smadam.F90:432)
  tod_cleaned_ = true;
  if (nbasis_ > 1) return clean_tod_basis();
  const long long n = (long long)ndet_ * nsamp_;
  const SampleMap sm = sample_map(istart_d_.get(), kstart_d_.get(), (int)ninterval_, nsamp_,
                                  noba_short_, fdn_);
  if (n > 0) MADAM_LAUNCH(k_clean_tod, grid_for(n), 256, 0, st_, d_tod_, n, sm, aa_.get());
}

void Engine::finalize(bool first_call) {
  if (par_.kfirst) subtract_baselines();
  const long long nm = nloc_;
  if (first_call && par_.do_matrix) {
    // the pixel matrices before inversion (write_matrix(cc), smadam.F90:389)
    cc_raw_host_.assign((size_t)12 * par_.nside_map * par_.nside_map * nmap_ * nmap_, 0.0);
    result_copy("cc", cc_raw_host_.data(), (long)(cc_raw_host_.size() * sizeof(double)));
  }
  if (first_call) {
    // invert_pixelmatrix_map (map_routines.f90:218-321)
    mask_.alloc(std::max<long long>(1, nm));
    mask_.zero(st_);
    crit_.alloc(std::max<long long>(1, nm));
    crit_.zero(st_);
    MatrixRules mr{(int)par_.pixmode_map, par_.pixlim_map, par_.allow_decoupling ? 1 : 0,
                   par_.incomplete_matrices ? 1 : 0};
    if (nm > 0) {
      if (nmap_ == 3)
        MADAM_LAUNCH(k_invert_map<3>, grid_for(nm), 128, 0, st_, cc_.get(), nm, mr, mask_.get(),
                     crit_.get());
      else
        MADAM_LAUNCH(k_invert_map<1>, grid_for(nm), 128, 0, st_, cc_.get(), nm, mr, mask_.get(),
                     crit_.get());
    }
  }
  // makemaps (map_routines.f90:327-357)
  if (nm > 0) {
    for (double *m : {binmap_.get(), map_.get()}) {
      if (nmap_ == 3) MADAM_LAUNCH(k_ccmult<3>, grid_for(nm), 256, 0, st_, cc_.get(), m, nm);
      else MADAM_LAUNCH(k_ccmult<1>, grid_for(nm), 256, 0, st_, cc_.get(), m, nm);
      if (par_.rm_monopole) {
        part_.alloc(std::max<size_t>(part_.n, 3 * kRedBlocks));
        scal_.alloc(std::max<size_t>(scal_.n, S_NSCAL));
        MADAM_LAUNCH(k_monopole, kRedBlocks, 256, 0, st_, m, mask_.get(), nm, nmap_, part_.get());
        finish_dots(2, 0, 8);
        MADAM_LAUNCH(k_sub_monopole, grid_for(nm), 256, 0, st_, m, mask_.get(), nm, nmap_,
                     scal_.get() + 8);
      }
    }
  }
  // leakage matrices and subsets (smadam.F90:405-408, 430), binned from the
  // TOD before clean_tod
  extra_d_.clear();
  extra_i_.clear();
  if (!suppress_fits_) {
    if (first_call && par_.do_leakmatrix) leak_matrices();
    run_subsets();
  }
  clean_tod();
  writeback_host();
  MADAM_CUDA(cudaStreamSynchronize(st_));
  write_fits(first_call);
}

void Engine::write_fits(bool first_call) {
  if (suppress_fits_ || !writes_files()) return;
  // write_map / write_binmap / write_mask / write_hits / write_matrix
  // (smadam.F90:401-422, 756-764)
  const bool any = par_.do_map || par_.do_binmap ||
                   (first_call && (par_.do_hits || par_.do_mask || par_.do_matrix || par_.do_wcov ||
                                   par_.do_leakmatrix));
  if (!any) return;
  const long npix = 12 * par_.nside_map * par_.nside_map;
  std::vector<double> map((size_t)npix * nmap_), bin((size_t)npix * nmap_), ccinv;
  std::vector<int> hits(npix), mask(npix);
  std::vector<float> crit(npix);
  result_copy("mask", mask.data(), (long)(mask.size() * sizeof(int)));
  if (par_.do_map) result_copy("map", map.data(), (long)(map.size() * sizeof(double)));
  if (par_.do_binmap) result_copy("binmap", bin.data(), (long)(bin.size() * sizeof(double)));
  if (first_call) {
    result_copy("hits", hits.data(), (long)(hits.size() * sizeof(int)));
    result_copy("crit", crit.data(), (long)(crit.size() * sizeof(float)));
    if (par_.do_wcov) {
      ccinv.resize((size_t)npix * nmap_ * nmap_);
      result_copy("cc", ccinv.data(), (long)(ccinv.size() * sizeof(double)));
    }
  }
  FitsInput in;
  in.par = &par_;
  in.nosubpix_map = nosubpix_map_;
  in.nosubmaps_tot = nosubmaps_tot_;
  in.ndet = ndet_;
  in.nmap = nmap_;
  in.first_call = first_call;
  in.isubchunk = isubchunk_;
  in.nsubchunk = nsubchunk_;
  in.map = par_.do_map ? map.data() : nullptr;
  in.binmap = par_.do_binmap ? bin.data() : nullptr;
  in.hits = hits.data();
  in.mask = mask.data();
  in.crit = crit.data();
  in.cc_raw = cc_raw_host_.empty() ? nullptr : cc_raw_host_.data();
  in.cc_inv = ccinv.empty() ? nullptr : ccinv.data();
  for (long d = 0; d < ndet_; ++d) {
    auto it = extra_d_.find("leakmatrix:" + std::to_string(d));
    if (it != extra_d_.end()) in.leak.push_back({dets_[d].name, it->second.data()});
  }
  write_products(in);
  cc_raw_host_.clear();
}

void Engine::writeback_host() {
  // restore_pixels (pointing.f90:168-191): the caller's pixel buffer shows the
  // reference's edits (flagged samples become 12 nside_max^2); a subchunk pass
  // leaves the caller's buffers to the full-data pass that follows it
  const long long n = (long long)ndet_ * nsamp_;
  if (n == 0 || isubchunk_ > 0) return;
  DevBuf<int> sub2;
  sub2.alloc(nosubmaps_tot_ + 1);
  std::vector<int> s2(subtable2_.begin(), subtable2_.end());
  MADAM_CUDA(cudaMemcpyAsync(sub2.get(), s2.data(), s2.size() * sizeof(int),
                             cudaMemcpyHostToDevice, st_));
  const long long cap = std::max<long long>(1024, n / 16);
  DevBuf<long long> idx;
  DevBuf<int32_t> val;
  DevBuf<unsigned long long> cnt;
  idx.alloc(cap);
  val.alloc(cap);
  cnt.alloc(1);
  cnt.zero(st_);
  MADAM_LAUNCH(k_restore, grid_for(n), 256, 0, st_, pix_.get(), pix_orig_.get(), n, sub2.get(),
               (int)nosubpix_max_, in_device_ ? d_pix_caller_ : (int32_t *)nullptr, idx.get(),
               val.get(), cnt.get(), cap);
  if (!in_device_) {
    unsigned long long c = 0;
    MADAM_CUDA(cudaMemcpyAsync(&c, cnt.get(), sizeof c, cudaMemcpyDeviceToHost, st_));
    MADAM_CUDA(cudaStreamSynchronize(st_));
    if ((long long)c <= cap) {
      std::vector<long long> hi(c);
      std::vector<int32_t> hv(c);
      if (c) {
        MADAM_CUDA(cudaMemcpyAsync(hi.data(), idx.get(), c * sizeof(long long),
                                   cudaMemcpyDeviceToHost, st_));
        MADAM_CUDA(cudaMemcpyAsync(hv.data(), val.get(), c * sizeof(int32_t),
                                   cudaMemcpyDeviceToHost, st_));
        MADAM_CUDA(cudaStreamSynchronize(st_));
      }
      for (size_t i = 0; i < c; ++i) h_pix_[hi[i]] = hv[i];
    } else {
      DevBuf<int32_t> fin;
      fin.alloc(n);
      MADAM_LAUNCH(k_restore, grid_for(n), 256, 0, st_, pix_.get(), (const int32_t *)nullptr, n,
                   sub2.get(), (int)nosubpix_max_, fin.get(), idx.get(), val.get(), cnt.get(), 0LL);
      MADAM_CUDA(cudaMemcpyAsync(h_pix_, fin.get(), n * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                 st_));
    }
    if (tod_cleaned_ && !fp32_)
      MADAM_CUDA(cudaMemcpyAsync(h_signal_, d_tod_, n * sizeof(double), cudaMemcpyDeviceToHost,
                                 st_));
  }
  if (tod_cleaned_ && fp32_) {
    // the cleaned float32 TOD goes back into the caller's signal buffer
    if (in_device_) {
      MADAM_LAUNCH(k_f64_to_f32, grid_for(n), 256, 0, st_, d_tod_, sig32_caller_, n);
    } else {
      DevBuf<float> t32;
      t32.alloc(n);
      MADAM_LAUNCH(k_f64_to_f32, grid_for(n), 256, 0, st_, d_tod_, t32.get(), n);
      MADAM_CUDA(cudaMemcpyAsync(sig32_caller_, t32.get(), n * sizeof(float),
                                 cudaMemcpyDeviceToHost, st_));
      MADAM_CUDA(cudaStreamSynchronize(st_));
    }
  }
  MADAM_CUDA(cudaStreamSynchronize(st_));
}

// destripe() up to the PCG: inputs, layout, filter, flagging, pointing
// tables, binning, right-hand side, preconditioner (smadam.F90:64-362)
void Engine::run_setup(const Params &par, std::vector<Detector> dets, long ndet, long nsamp,
                       long nnz, double *timestamps, int32_t *pix, float *pixweights,
                       double *signal, long nperiod, const long *periods, bool is_device) {
  g_alloc_stream = st_;
  const double t0 = now_ms();
  timings = Timings();
  rr_history.clear();
  noiter = 0;
  rrinit = 0;
  rr_final = 0;
  par_ = par;
  fp32_ = fp32_next_;
  fp32_next_ = false;
  dets_ = std::move(dets);
  ndet_ = ndet;
  nsamp_ = nsamp;
  nnz_ = nnz;
  nmap_ = (int)nnz;
  cached_ = false;
  tod_cleaned_ = false;
  cgp_.reset();
  d_pix_caller_ = is_device ? pix : nullptr;
  times_in_ = timestamps;
  times_dev_ = is_device;
  const long long n = (long long)ndet * nsamp;
  auto mark = [&](int i) {
    MADAM_CUDA(cudaStreamSynchronize(st_));
    setup_marks_[i] = now_ms() - t0;
  };
  trace_on_ = std::getenv("MADAM_B200_TRACE") != nullptr;
  trace_t_ = t0;
  if (trace_on_ && trace_ev_[0]) MADAM_CUDA(cudaEventRecord(trace_ev_[0], st_));
  bind_inputs(timestamps, pix, pixweights, signal, is_device, true);
  trace("bind_inputs");
  struct TodGuard {
    Engine &e;
    ~TodGuard() { e.sync_tod(); }
  } tod_guard{*this};
  mark(0);
  // pixel range check (smadam.F90:156-171)
  {
    DevBuf<int> mm;
    mm.alloc(2);
    const int init[2] = {INT_MAX, INT_MIN};
    MADAM_CUDA(cudaMemcpyAsync(mm.get(), init, sizeof init, cudaMemcpyHostToDevice, st_));
    if (n > 0) MADAM_LAUNCH(k_minmax, grid_for(n), 256, 0, st_, pix_.get(), n, mm.get());
    int out[2];
    MADAM_CUDA(cudaMemcpyAsync(out, mm.get(), sizeof out, cudaMemcpyDeviceToHost, st_));
    MADAM_CUDA(cudaStreamSynchronize(st_));
    const long nside_max = std::max(par_.nside_map, par_.nside_cross);
    std::string err;
    if (n > 0 && out[0] < -1) err = "Too small pixel number";
    if (n > 0 && (long)out[1] > 12 * nside_max * nside_max - 1) err = "Too large pixel number";
    // every rank of a sharded run learns of a failed check before the first
    // reduction that would otherwise wait for it
    if (ar_sum_host(err.empty() ? 0.0 : 1.0) > 0)
      fail(err.empty() ? "another rank failed its input checks" : err);
  }
  trace("pixel_check");
  init_layout(nperiod, periods);
  trace("init_layout");
  // baseline start times (baseline_times, parameter_control.f90:956-977)
  btime_.assign(noba_short_, 0.0);
  if (is_device) {
    if (noba_short_ > 0) {
      DevBuf<double> bt;
      bt.alloc(noba_short_);
      MADAM_LAUNCH(k_take, grid_for(noba_short_), 256, 0, st_, timestamps, bstart_d_.get(),
                   (long long)noba_short_, bt.get());
      MADAM_CUDA(cudaMemcpyAsync(btime_.data(), bt.get(), noba_short_ * sizeof(double),
                                 cudaMemcpyDeviceToHost, st_));
      MADAM_CUDA(cudaStreamSynchronize(st_));
    }
  } else {
    for (long k = 0; k < noba_short_; ++k) btime_[k] = timestamps[bstart_[k]];
  }
  mark(1);
  struct FilterJobGuard {
    std::future<void> &f;
    ~FilterJobGuard() {
      if (f.valid()) f.wait();
    }
  } filter_guard{filter_job_};
  trace("baseline_times");
  build_filter();
  mark(2);
  trace("build_filter");
  flag_and_compact(true);
  mark(3);
  trace("flag_and_compact");
  build_runs();
  mark(4);
  trace("build_runs");
  setup_scatter();
  mark(5);
  trace("setup_scatter");
  if (par_.kfirst) build_csr();
  mark(6);
  trace("build_csr");
  if (par_.kfirst) {
    map_side_setup();
    trace("map_side_setup");
    initialize_a();
    trace("initialize_a");
    check_nan_setup();
    mark(7);
    build_segments();
    trace("build_segments");
    build_filter_finish();
    mark(8);
    trace("build_filter_finish");
    construct_preconditioner();
    mark(9);
    trace("construct_preconditioner");
  }
  MADAM_CUDA(cudaStreamSynchronize(st_));
  timings.setup_ms = now_ms() - t0;
  run_t0_ = t0;
}

void Engine::run(const Params &par, std::vector<Detector> dets, long ndet, long nsamp, long nnz,
                 double *timestamps, int32_t *pix, float *pixweights, double *signal,
                 long nperiod, const long *periods, bool is_device) {
  run_setup(par, std::move(dets), ndet, nsamp, nnz, timestamps, pix, pixweights, signal, nperiod,
            periods, is_device);
  run_solve();
  run_finish();
}

void Engine::run_solve() {
  if (!par_.kfirst) return;
  // write_covmat in place of the solve (smadam.F90:364-377)
  if (par_.file_covmat.empty()) iterate();
  else write_covmat();
}

void Engine::run_finish() {
  const double tf = now_ms();
  finalize(true);
  timings.finalize_ms = now_ms() - tf;
  if (par_.mcmode) cached_ = true;
  timings.total_ms = now_ms() - run_t0_;
}

void Engine::run_cached(long ndet, long nsamp, long nnz, double *timestamps, int32_t *pix,
                        float *pixweights, double *signal, bool is_device) {
  g_alloc_stream = st_;
  // destripe_with_cache (smadam.F90:593-918)
  if (!cached_) fail("destripe_with_cache called with empty caches.");
  if (par_.temperature_only && nnz != 1)
    fail("temperature_only=T but pointing weights are polarized");
  if (ndet != ndet_ || nsamp != nsamp_ || nnz != nnz_)
    fail("destripe_with_cache: data shape differs from the cached call");
  const double t0 = now_ms();
  timings = Timings();
  rr_history.clear();
  noiter = 0;
  tod_cleaned_ = false;
  d_pix_caller_ = is_device ? pix : nullptr;
  times_in_ = timestamps;
  times_dev_ = is_device;
  fp32_ = false;  // destripe_with_cache takes float64 signals
  fp32_next_ = false;
  bind_inputs(timestamps, pix, pixweights, signal, is_device, false);
  struct TodGuard {
    Engine &e;
    ~TodGuard() { e.sync_tod(); }
  } tod_guard{*this};
  flag_and_compact(false);
  build_runs();
  bin_tod(true);
  if (par_.kfirst) build_csr();
  if (par_.kfirst) {
    std::vector<Segment> old = segs_;
    initialize_a();
    build_segments();
    bool same = old.size() == segs_.size();
    for (size_t i = 0; same && i < old.size(); ++i)
      same = old[i].k0 == segs_[i].k0 && old[i].noba == segs_[i].noba;
    if (!same) fail("destripe_with_cache: flagging differs from the cached call");
    MADAM_CUDA(cudaStreamSynchronize(st_));
    timings.setup_ms = now_ms() - t0;
    iterate();
  }
  const double tf = now_ms();
  finalize(false);
  timings.finalize_ms = now_ms() - tf;
  timings.total_ms = now_ms() - t0;
}

// --------------------------------------------------------------- results --
namespace {
enum RKind { RK_DOUBLE, RK_INT, RK_FLOAT, RK_LONG };
}

// compacted per-pixel arrays (hit submaps only) -> the full sky
void Engine::expand_host(const void *host, size_t elem, long per_pix, long nosubpix, void *out) {
  const long total = nosubmaps_tot_ * nosubpix;
  std::memset(out, 0, (size_t)total * per_pix * elem);
  for (long j = 0; j < nolocmaps_; ++j) {
    const long g = j + subtable2_[j];
    std::memcpy((char *)out + (size_t)g * nosubpix * per_pix * elem,
                (const char *)host + (size_t)j * nosubpix * per_pix * elem,
                (size_t)nosubpix * per_pix * elem);
  }
}

void Engine::expand_to_sky(const void *dev, size_t elem, long per_pix, long nosubpix,
                           void *out) {
  const long nloc_pix = nolocmaps_ * nosubpix;
  std::vector<char> h((size_t)nloc_pix * per_pix * elem);
  MADAM_CUDA(cudaStreamSynchronize(st_));  // the engine's stream does not order cudaMemcpy
  if (nloc_pix) MADAM_CUDA(cudaMemcpy(h.data(), dev, h.size(), cudaMemcpyDeviceToHost));
  expand_host(h.data(), elem, per_pix, nosubpix, out);
}

long Engine::result_size(const std::string &name) {
  const long npm = 12 * par_.nside_map * par_.nside_map;
  const long npc = 12 * par_.nside_cross * par_.nside_cross;
  const long nb = ndet_ * noba_short_;
  if (name == "map" || name == "binmap") return npm * nmap_;
  if (name == "hits" || name == "mask" || name == "crit") return npm;
  if (name == "cc") return npm * nmap_ * nmap_;
  if (name == "cca") return npc * nmap_ * nmap_;
  if (name == "aa" || name == "yba") return nb * nbasis_;
  if (name == "nna") return nb * nbasis_ * nbasis_;
  if (name == "fcov") return (long)fcov_host().size();
  if (name == "invcov") return (long)invcov_host().size();
  if (name == "rr_history") return (long)rr_history.size();
  if (name == "band_widths") return (long)band_widths_.size();
  if (name == "scalars") return 24;
  if (name == "timings") return 9;
  if (name == "nan_checks") return (long)nan_checks_.size();
  if (name == "setup_marks") return kSetupMarks;
  if (name == "map_batch" || name == "binmap_batch") return nrhs_ * npm * nmap_;
  if (name == "aa_batch") return nrhs_ * nb;
  if (name == "noiter_batch" || name == "rrinit_batch" || name == "rr_final_batch")
    return (long)noiter_b_.size();
  auto ed = extra_d_.find(name);
  if (ed != extra_d_.end()) return (long)ed->second.size();
  auto ei = extra_i_.find(name);
  if (ei != extra_i_.end()) return (long)ei->second.size();
  auto sd = subchunk_d_.find(name);
  if (sd != subchunk_d_.end()) return (long)sd->second.size();
  auto si = subchunk_i_.find(name);
  if (si != subchunk_i_.end()) return (long)si->second.size();
  return -1;
}

void Engine::keep_subchunk_results(int isub) {
  // the products of subchunk pass isub, kept beside the full-data pass's
  const std::string k = ":" + std::to_string(isub);
  for (const char *nm : {"map", "binmap"}) {
    std::vector<double> &v = subchunk_d_[std::string("subchunk_") + nm + k];
    v.resize(result_size(nm));
    result_copy(nm, v.data(), (long)(v.size() * sizeof(double)));
  }
  for (const char *nm : {"hits", "mask"}) {
    std::vector<int> &v = subchunk_i_[std::string("subchunk_") + nm + k];
    v.resize(result_size(nm));
    result_copy(nm, v.data(), (long)(v.size() * sizeof(int)));
  }
  for (auto &e : extra_d_) subchunk_d_["subchunk" + k + "/" + e.first] = e.second;
  for (auto &e : extra_i_) subchunk_i_["subchunk" + k + "/" + e.first] = e.second;
}

void Engine::result_copy(const std::string &name, void *dst, long nbytes) {
  g_alloc_stream = st_;
  const long sz = result_size(name);
  if (sz < 0) fail("unknown result: " + name);
  auto need = [&](size_t elem) {
    if ((size_t)nbytes < (size_t)sz * elem) fail("result buffer too small for " + name);
  };
  MADAM_CUDA(cudaStreamSynchronize(st_));
  auto expand = [&](const void *dev, size_t elem, long per_pix, long nosubpix, void *out) {
    expand_to_sky(dev, elem, per_pix, nosubpix, out);
  };
  auto sym = [&](const std::vector<double> &s6, long npix, double *out) {
    for (long p = 0; p < npix; ++p) {
      double *o = out + p * nmap_ * nmap_;
      if (nmap_ == 1) {
        o[0] = s6[p];
        continue;
      }
      const double *c = &s6[p * 6];
      o[0] = c[0]; o[1] = c[1]; o[2] = c[2];
      o[3] = c[1]; o[4] = c[3]; o[5] = c[4];
      o[6] = c[2]; o[7] = c[4]; o[8] = c[5];
    }
  };
  const long ncc = nmap_ == 3 ? 6 : 1;
  {
    auto sd = subchunk_d_.find(name);
    if (sd != subchunk_d_.end()) {
      need(sizeof(double));
      std::memcpy(dst, sd->second.data(), sd->second.size() * sizeof(double));
      return;
    }
    auto si = subchunk_i_.find(name);
    if (si != subchunk_i_.end()) {
      need(sizeof(int));
      std::memcpy(dst, si->second.data(), si->second.size() * sizeof(int));
      return;
    }
    auto ed = extra_d_.find(name);
    if (ed != extra_d_.end()) {
      need(sizeof(double));
      std::memcpy(dst, ed->second.data(), ed->second.size() * sizeof(double));
      return;
    }
    auto ei = extra_i_.find(name);
    if (ei != extra_i_.end()) {
      need(sizeof(int));
      std::memcpy(dst, ei->second.data(), ei->second.size() * sizeof(int));
      return;
    }
  }
  if (name == "map_batch" || name == "binmap_batch") {
    need(sizeof(double));
    const long long nv = (long long)nloc_ * nmap_;
    const long long npm = 12LL * par_.nside_map * par_.nside_map * nmap_;
    const double *src = name == "map_batch" ? mapb_.get() : binmapb_.get();
    for (long k = 0; k < nrhs_; ++k)
      expand(src + k * nv, sizeof(double), nmap_, nosubpix_map_, (double *)dst + k * npm);
  } else if (name == "aa_batch") {
    need(sizeof(double));
    if (sz) MADAM_CUDA(cudaMemcpy(dst, aab_.get(), sz * sizeof(double), cudaMemcpyDeviceToHost));
  } else if (name == "noiter_batch" || name == "rrinit_batch" || name == "rr_final_batch") {
    need(sizeof(double));
    const std::vector<double> &v = name == "noiter_batch" ? noiter_b_
                                   : name == "rrinit_batch" ? rrinit_b_ : rrfinal_b_;
    std::memcpy(dst, v.data(), v.size() * sizeof(double));
  } else if (name == "map" || name == "binmap") {
    need(sizeof(double));
    expand(name == "map" ? map_.get() : binmap_.get(), sizeof(double), nmap_, nosubpix_map_, dst);
  } else if (name == "hits") {
    need(sizeof(int));
    expand(hits_.get(), sizeof(int), 1, nosubpix_map_, dst);
  } else if (name == "mask") {
    need(sizeof(int));
    expand(mask_.get(), sizeof(int), 1, nosubpix_map_, dst);
  } else if (name == "crit") {
    need(sizeof(float));
    expand(crit_.get(), sizeof(float), 1, nosubpix_map_, dst);
  } else if (name == "cc" || name == "cca") {
    need(sizeof(double));
    const bool cross = name == "cca";
    const long nsp = cross ? nosubpix_cross_ : nosubpix_map_;
    std::vector<double> s6((size_t)nosubmaps_tot_ * nsp * ncc);
    expand(cross ? cca_.get() : cc_.get(), sizeof(double), ncc, nsp, s6.data());
    sym(s6, nosubmaps_tot_ * nsp, (double *)dst);
  } else if (name == "aa" || name == "yba" || name == "nna") {
    need(sizeof(double));
    const double *src = name == "aa" ? aa_.get() : name == "yba" ? yba_.get() : nna_.get();
    if (sz) MADAM_CUDA(cudaMemcpy(dst, src, sz * sizeof(double), cudaMemcpyDeviceToHost));
  } else if (name == "fcov") {
    need(sizeof(double));
    std::memcpy(dst, fcov_host().data(), sz * sizeof(double));
  } else if (name == "invcov") {
    need(sizeof(double));
    std::memcpy(dst, invcov_host().data(), sz * sizeof(double));
  } else if (name == "rr_history") {
    need(sizeof(double));
    std::memcpy(dst, rr_history.data(), sz * sizeof(double));
  } else if (name == "band_widths") {
    need(sizeof(long));
    std::memcpy(dst, band_widths_.data(), sz * sizeof(long));
  } else if (name == "scalars") {
    need(sizeof(double));
    const double v[24] = {(double)noiter, rrinit, rr_final, (double)nof_,
                          (double)band_widths_.size(), (double)n_band_fail_, timings.iterate_ms,
                          timings.total_ms, (double)nmap_, (double)noba_short_,
                          (double)(12 * par_.nside_map * par_.nside_map), (double)nruns_,
                          (double)nwork_, (double)nloc_, (double)segs_.size(),
                          (double)cg_prec_segs_.size(), (double)band2_rows_,
                          (double)band2_ntrans_, (double)p2nch_, (double)csr_nvalid_,
                          (double)(use_pairs_ ? npairs_ : 0), fp32_ ? 1.0 : 0.0,
                          (double)n_reliable_, band2_guarded_ ? (double)band2_guard_ : 0.0};
    std::memcpy(dst, v, sizeof v);
  } else if (name == "setup_marks") {
    need(sizeof(double));
    std::memcpy(dst, setup_marks_, sizeof setup_marks_);
  } else if (name == "nan_checks") {
    need(sizeof(double));
    std::memcpy(dst, nan_checks_.data(), nan_checks_.size() * sizeof(double));
  } else if (name == "timings") {
    need(sizeof(double));
    const double v[9] = {timings.setup_ms, timings.iterate_ms, timings.finalize_ms,
                         timings.total_ms, timings.scatter_ms, timings.gather_ms,
                         timings.filter_ms, timings.precond_ms, timings.other_ms};
    std::memcpy(dst, v, sizeof v);
  }
}

// K timed PCG iterations restarted from the solve's right-hand side.  The
// solution of the last solve is kept.  out: [total_ms, ms_per_iter,
// launches_per_iter, scatter_ms, filter_ms, gather_ms, precond_ms, update_ms]
void Engine::bench_iterations(int warmup, int iters, std::vector<double> &out) {
  g_alloc_stream = st_;
  if (!par_.kfirst || noba_short_ == 0) fail("no solve state to benchmark");
  if (nbasis_ > 1) fail("the iteration benchmark takes basis_order 0");
  const long long nb = (long long)ndet_ * noba_short_;
  DevBuf<double> aa_keep;
  aa_keep.alloc(nb);
  MADAM_CUDA(cudaMemcpyAsync(aa_keep.get(), aa_.get(), nb * sizeof(double),
                             cudaMemcpyDeviceToDevice, st_));
  auto restart = [&]() {
    MADAM_CUDA(cudaMemcpyAsync(r_.get(), yba_.get(), nb * sizeof(double),
                               cudaMemcpyDeviceToDevice, st_));
    aa_.zero(st_);
    apply_preconditioner(r_.get(), z_.get());
    MADAM_LAUNCH(k_update_p, grid_for(nb), 256, 0, st_, p_.get(), z_.get(), pw_.get(), bw_.get(),
                 nb, scal_.get(), 1);
    MADAM_LAUNCH(k_dots, kRedBlocks, 256, 0, st_, r_.get(), z_.get(), r_.get(), r_.get(), nullptr,
                 nullptr, 2, rmask_.get(), nb, part_.get());
    finish_dots(2, 0, S_RZ, kRedBlocks, true);
  };
  auto one = [&](bool timed) {
    apply_A(p_.get(), pw_.get(), ap_.get(), timed);
    MADAM_LAUNCH(k_update_ar, grid_for(nb), 256, 0, st_, aa_.get(), r_.get(), ro_.get(), p_.get(),
                 ap_.get(), nb, scal_.get());
    if (timed) MADAM_CUDA(cudaEventRecord(ev_[5], st_));
    apply_preconditioner(r_.get(), z_.get());
    if (timed) MADAM_CUDA(cudaEventRecord(ev_[6], st_));
    MADAM_LAUNCH(k_dots, kRedBlocks, 256, 0, st_, r_.get(), z_.get(), ro_.get(), z_.get(),
                 r_.get(), r_.get(), 3, rmask_.get(), nb, part_.get());
    finish_dots(3, 2, 0, kRedBlocks, true);
    MADAM_LAUNCH(k_update_p, grid_for(nb), 256, 0, st_, p_.get(), z_.get(), pw_.get(), bw_.get(),
                 nb, scal_.get(), 0);
    if (timed) MADAM_CUDA(cudaEventRecord(ev_[7], st_));
  };
  restart();
  for (int i = 0; i < warmup; ++i) one(false);
  MADAM_CUDA(cudaStreamSynchronize(st_));
  cudaEvent_t a, b;
  MADAM_CUDA(cudaEventCreate(&a));
  MADAM_CUDA(cudaEventCreate(&b));
  const unsigned long long l0 = g_kernel_launches;
  MADAM_CUDA(cudaEventRecord(a, st_));
  for (int i = 0; i < iters; ++i) one(false);
  MADAM_CUDA(cudaEventRecord(b, st_));
  MADAM_CUDA(cudaEventSynchronize(b));
  const unsigned long long l1 = g_kernel_launches;
  float total = 0;
  MADAM_CUDA(cudaEventElapsedTime(&total, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  check_band_err();
  // per-phase breakdown on separate iterations
  double sc = 0, fi = 0, ga = 0, pr = 0, up = 0;
  const int nbrk = std::max(1, std::min(iters, 5));
  for (int i = 0; i < nbrk; ++i) {
    one(true);
    MADAM_CUDA(cudaStreamSynchronize(st_));
    float t[5];
    MADAM_CUDA(cudaEventElapsedTime(&t[0], ev_[0], ev_[1]));
    MADAM_CUDA(cudaEventElapsedTime(&t[1], ev_[2], ev_[3]));
    MADAM_CUDA(cudaEventElapsedTime(&t[2], ev_[3], ev_[4]));
    MADAM_CUDA(cudaEventElapsedTime(&t[3], ev_[5], ev_[6]));
    MADAM_CUDA(cudaEventElapsedTime(&t[4], ev_[6], ev_[7]));
    sc += t[0];
    fi += t[1];
    ga += t[2];
    pr += t[3];
    up += t[4];
  }
  MADAM_CUDA(cudaMemcpyAsync(aa_.get(), aa_keep.get(), nb * sizeof(double),
                             cudaMemcpyDeviceToDevice, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  out = {total, total / std::max(1, iters), (double)(l1 - l0) / std::max(1, iters), sc / nbrk,
         fi / nbrk, ga / nbrk, pr / nbrk, up / nbrk};
}
