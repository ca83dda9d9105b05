// Subset maps and leakage matrices: run_subsets (smadam.F90:954-1257) and
// leakmatrix (smadam_routines.f90:38-105).
//
// After the full-data maps, every (survey, detector set) pair but the full
// one is binned again: pixel matrix, hits (first pass), binned map,
// inversion with the map rules, leakage matrices of its detectors (first
// pass), makemaps.  The reference sets kfirst = F before these passes, so
// their clean_tod returns at once and the subsets are binned from the TOD as
// it stands; a second pass (binned and destriped maps both requested) repeats
// the binned map under the "_map" name.  A nopol set of polarised data is
// binned with nmap = 1, which, as in pixel_matrix / bin_tod, ignores the
// weights.  Products are kept as named host results and written as FITS
// files; the full-data products are untouched.

// pixel matrix, binned map and hits of the samples of the flagged detectors
// whose time lies in one of the spans (all samples when nspan = 0)
template <int NMAPS, int NNZ>
__global__ void k_subset_accum(const float4 *__restrict__ p4, const int32_t *__restrict__ pc,
                               const double *__restrict__ tod, long long n, SampleMap sm,
                               const double *__restrict__ bw, int nloc,
                               const uint8_t *__restrict__ detflags,
                               const double *__restrict__ times, const double2 *__restrict__ spans,
                               int nspan, double *__restrict__ cc, double *__restrict__ bin,
                               int *__restrict__ hits) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long det = i / sm.nsamp, s = i - det * sm.nsamp;
    if (!detflags[det]) continue;
    if (nspan > 0) {
      const double t = times[s];
      bool on = false;
      for (int j = 0; j < nspan; ++j)
        if (spans[j].x <= t && t <= spans[j].y) on = true;
      if (!on) continue;
    }
    const double detw = bw[baseline_of(sm, det, s)];
    if (detw == 0) continue;
    float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
    int px;
    if (NNZ == 3) {
      q = p4[i];
      px = point_pix(q);
    } else {
      px = pc[i];
    }
    if (px >= nloc) continue;
    if (hits) atomicAdd(hits + px, 1);
    if (NMAPS == 1) {
      if (cc) atomicAdd(cc + px, detw);
      if (bin) atomicAdd(bin + px, tod[i] * detw);
    } else {
      const double sq = sqrt(detw);
      const double w0 = (double)q.x * sq, w1 = (double)q.y * sq, w2 = (double)q.z * sq;
      if (cc) {
        double *c = cc + (long long)px * 6;
        atomicAdd(c + 0, w0 * w0);
        atomicAdd(c + 1, w0 * w1);
        atomicAdd(c + 2, w0 * w2);
        atomicAdd(c + 3, w1 * w1);
        atomicAdd(c + 4, w1 * w2);
        atomicAdd(c + 5, w2 * w2);
      }
      if (bin) {
        const double t = tod[i];
        double *m = bin + (long long)px * 3;
        atomicAdd(m + 0, (double)q.x * t * detw);
        atomicAdd(m + 1, (double)q.y * t * detw);
        atomicAdd(m + 2, (double)q.z * t * detw);
      }
    }
  }
}

namespace {
// packed upper triangle (1 or 6 values) -> full symmetric nmap x nmap
inline void unpack_sym(const double *c, int nmap, double *o) {
  if (nmap == 1) {
    o[0] = c[0];
    return;
  }
  o[0] = c[0]; o[1] = c[1]; o[2] = c[2];
  o[3] = c[1]; o[4] = c[3]; o[5] = c[4];
  o[6] = c[2]; o[7] = c[4]; o[8] = c[5];
}
}  // namespace

void Engine::subset_accumulate(const std::vector<uint8_t> &detflags,
                               const std::vector<double2> &spans, int nmaps, double *cc,
                               double *bin, int *hits) {
  const long long n = (long long)ndet_ * nsamp_;
  if (n == 0 || nloc_ == 0) return;
  DevBuf<uint8_t> df;
  df.alloc(detflags.size());
  MADAM_CUDA(cudaMemcpyAsync(df.get(), detflags.data(), detflags.size(), cudaMemcpyHostToDevice,
                             st_));
  DevBuf<double2> sp;
  sp.alloc(std::max<size_t>(1, spans.size()));
  if (!spans.empty())
    MADAM_CUDA(cudaMemcpyAsync(sp.get(), spans.data(), spans.size() * sizeof(double2),
                               cudaMemcpyHostToDevice, st_));

  const SampleMap sm = sample_map(istart_d_.get(), kstart_d_.get(), (int)ninterval_, nsamp_,
                                  noba_short_, fdn_);
  const double *times = spans.empty() ? nullptr : subset_times_;
  if (nnz_ == 3 && nmaps == 3)
    MADAM_LAUNCH((k_subset_accum<3, 3>), grid_for(n), 256, 0, st_, point4_.get(), pixc_.get(),
                 d_tod_, n, sm, bw_.get(), (int)nloc_, df.get(), times, sp.get(),
                 (int)spans.size(), cc, bin, hits);
  else if (nnz_ == 3)
    MADAM_LAUNCH((k_subset_accum<1, 3>), grid_for(n), 256, 0, st_, point4_.get(), pixc_.get(),
                 d_tod_, n, sm, bw_.get(), (int)nloc_, df.get(), times, sp.get(),
                 (int)spans.size(), cc, bin, hits);
  else
    MADAM_LAUNCH((k_subset_accum<1, 1>), grid_for(n), 256, 0, st_, point4_.get(), pixc_.get(),
                 d_tod_, n, sm, bw_.get(), (int)nloc_, df.get(), times, sp.get(),
                 (int)spans.size(), cc, bin, hits);
  // collect_cc / collect_hits / collect_map across the ranks of a sharded run
  if (cc) ar_sum(cc, (size_t)nloc_ * (nmaps == 3 ? 6 : 1));
  if (bin) ar_sum(bin, (size_t)nloc_ * nmaps);
  if (hits) ar_sum(hits, (size_t)nloc_);
  MADAM_CUDA(cudaStreamSynchronize(st_));
}

// gamma = C^-1 C_det per compacted pixel (both symmetric, packed), expanded
// to the full sky as [npix][nmap][nmap], row i column j
std::vector<double> Engine::leak_product(const std::vector<double> &cinv,
                                         const std::vector<double> &cdet, int nmaps) {
  const int ncc = nmaps == 3 ? 6 : 1, nn = nmaps * nmaps;
  const long nm = nloc_;
  std::vector<double> g((size_t)nm * nn, 0.0);
  double a[9], b[9];
  for (long p = 0; p < nm; ++p) {
    unpack_sym(&cinv[(size_t)p * ncc], nmaps, a);
    unpack_sym(&cdet[(size_t)p * ncc], nmaps, b);
    for (int i = 0; i < nmaps; ++i)
      for (int j = 0; j < nmaps; ++j) {
        double s = 0;
        for (int k = 0; k < nmaps; ++k) s += a[i * nmaps + k] * b[k * nmaps + j];
        g[(size_t)p * nn + i * nmaps + j] = s;
      }
  }
  std::vector<double> out((size_t)nosubmaps_tot_ * nosubpix_map_ * nn);
  expand_host(g.data(), sizeof(double), nn, nosubpix_map_, out.data());
  return out;
}

std::vector<double> Engine::detector_matrix(long det, int nmaps) {
  // pixel_matrix of one detector over all samples (leakmatrix)
  const int ncc = nmaps == 3 ? 6 : 1;
  DevBuf<double> c;
  c.alloc((size_t)std::max<long>(1, nloc_) * ncc);
  c.zero(st_);
  std::vector<uint8_t> f(ndet_, 0);
  f[det] = 1;
  subset_accumulate(f, subset_spans_, nmaps, c.get(), nullptr, nullptr);
  std::vector<double> h((size_t)nloc_ * ncc);
  if (!h.empty())
    MADAM_CUDA(cudaMemcpy(h.data(), c.get(), h.size() * sizeof(double), cudaMemcpyDeviceToHost));
  return h;
}

// In a sharded run the leakage matrices take one reduction per detector, so,
// as in the reference, every rank must hold the same detectors: compared
// through a hash of their names, on every rank alike.
void Engine::check_same_detectors() {
  if (!sharded()) return;
  uint64_t h = 1469598103934665603ull;
  for (const auto &d : dets_)
    for (char c : d.name + ";") h = (h ^ (unsigned char)c) * 1099511628211ull;
  DevBuf<int> v;
  v.alloc(4);
  const int hv[4] = {(int)(h & 0x3fffffff), (int)((h >> 30) & 0x3fffffff),
                     -(int)(h & 0x3fffffff), -(int)((h >> 30) & 0x3fffffff)};
  MADAM_CUDA(cudaMemcpyAsync(v.get(), hv, sizeof hv, cudaMemcpyHostToDevice, st_));
  ar_max(v.get(), 4);
  int r[4];
  MADAM_CUDA(cudaMemcpyAsync(r, v.get(), sizeof r, cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
  if (r[0] != -r[2] || r[1] != -r[3])
    fail("leakage matrices of a sharded run need the same detectors on every rank");
}

void Engine::leak_matrices() {
  // leakmatrix (smadam_routines.f90:38-105) for every detector of the
  // full-data run, from the inverted full-data matrices
  check_same_detectors();
  const int ncc = nmap_ == 3 ? 6 : 1;
  MADAM_CUDA(cudaStreamSynchronize(st_));
  std::vector<double> cinv((size_t)nloc_ * ncc);
  if (!cinv.empty())
    MADAM_CUDA(cudaMemcpy(cinv.data(), cc_.get(), cinv.size() * sizeof(double),
                          cudaMemcpyDeviceToHost));
  subset_spans_.clear();
  for (long d = 0; d < ndet_; ++d)
    extra_d_["leakmatrix:" + std::to_string(d)] = leak_product(cinv, detector_matrix(d, nmap_),
                                                               nmap_);
}

void Engine::run_subsets() {
  const Params &p = par_;
  if (!p.bin_subsets || (p.ndetset == 0 && p.nsurvey == 0)) return;
  const long nm = nloc_;
  const long npix = nosubmaps_tot_ * nosubpix_map_;
  // per-sample times for the surveys (sampletime, same for every detector)
  std::vector<double> htimes;
  if (p.nsurvey > 0) {
    htimes.resize(nsamp_);
    if (times_dev_) {
      MADAM_CUDA(cudaMemcpy(htimes.data(), times_in_, nsamp_ * sizeof(double),
                            cudaMemcpyDeviceToHost));
      subset_times_ = times_in_;
    } else {
      std::memcpy(htimes.data(), times_in_, nsamp_ * sizeof(double));
      times_own_.alloc(nsamp_);
      MADAM_CUDA(cudaMemcpyAsync(times_own_.get(), times_in_, nsamp_ * sizeof(double),
                                 cudaMemcpyHostToDevice, st_));
      subset_times_ = times_own_.get();
    }
  }
  const int npass = (p.do_binmap && p.do_map) ? 2 : 1;
  if (p.do_leakmatrix) check_same_detectors();
  std::vector<double> table;
  long k = 0;
  for (int pass = 1; pass <= npass; ++pass) {
    for (int isv = 0; isv <= p.nsurvey; ++isv) {
      subset_spans_.clear();
      long nhs = nsamp_;
      if (isv != 0) {
        const Params::Survey &sv = p.surveys[isv];
        for (size_t j = 0; j < sv.starts.size(); ++j)
          subset_spans_.push_back(make_double2(sv.starts[j], sv.stops[j]));
        nhs = 0;
        for (long i = 0; i < nsamp_; ++i)
          for (const double2 &s2 : subset_spans_)
            if (s2.x <= htimes[i] && htimes[i] <= s2.y) {
              ++nhs;
              break;
            }
      }
      nhs = (long)ar_sum_host((double)nhs);  // sum_mpi(nhit_survey)
      if (nhs == 0) continue;
      for (int ids = 0; ids <= p.ndetset; ++ids) {
        if (ids == 0 && isv == 0) continue;
        std::vector<uint8_t> df(ndet_, 1);
        bool tonly = p.temperature_only;
        if (ids != 0) {
          const Params::DetSet &ds = p.detsets[ids];
          for (long d = 0; d < ndet_; ++d) {
            df[d] = 0;
            for (const std::string &nme : ds.dets)
              if (dets_[d].name == nme) df[d] = 1;
          }
          tonly = ds.nopol && !p.force_pol;
        }
        long nhd = 0;
        for (long d = 0; d < ndet_; ++d) nhd += df[d];
        nhd = (long)ar_sum_host((double)nhd);  // sum_mpi(nhit_det)
        if (nhd == 0) continue;
        const int nms = tonly ? 1 : nmap_;
        const int ncc = nms == 3 ? 6 : 1;
        DevBuf<double> c, b;
        DevBuf<int> h, msk;
        DevBuf<float> cr;
        c.alloc((size_t)std::max<long>(1, nm) * ncc);
        c.zero(st_);
        b.alloc((size_t)std::max<long>(1, nm) * nms);
        b.zero(st_);
        h.alloc(std::max<long>(1, nm));
        h.zero(st_);
        msk.alloc(std::max<long>(1, nm));
        msk.zero(st_);
        cr.alloc(std::max<long>(1, nm));
        cr.zero(st_);
        subset_accumulate(df, subset_spans_, nms, c.get(), b.get(), pass == 1 ? h.get() : nullptr);
        std::vector<double> craw;  // (subset_accumulate has synchronised the stream)
        if (pass == 1 && p.do_matrix) {
          std::vector<double> packed((size_t)nm * ncc);
          if (nm)
            MADAM_CUDA(cudaMemcpy(packed.data(), c.get(), packed.size() * sizeof(double),
                                  cudaMemcpyDeviceToHost));
          craw = full_sym(packed, nms);
        }
        MatrixRules mr{(int)p.pixmode_map, p.pixlim_map, p.allow_decoupling ? 1 : 0,
                       p.incomplete_matrices ? 1 : 0};
        if (nm > 0) {
          if (nms == 3)
            MADAM_LAUNCH(k_invert_map<3>, grid_for(nm), 128, 0, st_, c.get(), (long long)nm, mr,
                         msk.get(), cr.get());
          else
            MADAM_LAUNCH(k_invert_map<1>, grid_for(nm), 128, 0, st_, c.get(), (long long)nm, mr,
                         msk.get(), cr.get());
        }
        MADAM_CUDA(cudaStreamSynchronize(st_));
        std::vector<double> cinv((size_t)nm * ncc);
        if (nm)
          MADAM_CUDA(cudaMemcpy(cinv.data(), c.get(), cinv.size() * sizeof(double),
                                cudaMemcpyDeviceToHost));
        const std::string key = std::to_string(k);
        std::vector<std::pair<std::string, const double *>> leaks;
        if (pass == 1 && p.do_leakmatrix) {
          for (long d = 0; d < ndet_; ++d) {
            if (!df[d]) continue;
            std::vector<double> cd((size_t)nm * ncc);
            {
              DevBuf<double> c1;
              c1.alloc((size_t)std::max<long>(1, nm) * ncc);
              c1.zero(st_);
              std::vector<uint8_t> f1(ndet_, 0);
              f1[d] = 1;
              subset_accumulate(f1, subset_spans_, nms, c1.get(), nullptr, nullptr);
              if (nm)
                MADAM_CUDA(cudaMemcpy(cd.data(), c1.get(), cd.size() * sizeof(double),
                                      cudaMemcpyDeviceToHost));
            }
            const std::string nme = "subset_leak:" + key + ":" + std::to_string(d);
            extra_d_[nme] = leak_product(cinv, cd, nms);
          }
          for (long d = 0; d < ndet_; ++d)
            if (df[d])
              leaks.push_back({dets_[d].name,
                               extra_d_["subset_leak:" + key + ":" + std::to_string(d)].data()});
        }
        // makemaps (map_routines.f90:327-357)
        if (nm > 0) {
          if (nms == 3)
            MADAM_LAUNCH(k_ccmult<3>, grid_for(nm), 256, 0, st_, c.get(), b.get(), (long long)nm);
          else
            MADAM_LAUNCH(k_ccmult<1>, grid_for(nm), 256, 0, st_, c.get(), b.get(), (long long)nm);
          if (p.rm_monopole) {
            part_.alloc(std::max<size_t>(part_.n, 3 * kRedBlocks));
            scal_.alloc(std::max<size_t>(scal_.n, S_NSCAL));
            MADAM_LAUNCH(k_monopole, kRedBlocks, 256, 0, st_, b.get(), msk.get(), (long long)nm,
                         nms, part_.get());
            finish_dots(2, 0, 8);
            MADAM_LAUNCH(k_sub_monopole, grid_for(nm), 256, 0, st_, b.get(), msk.get(),
                         (long long)nm, nms, scal_.get() + 8);
          }
        }
        MADAM_CUDA(cudaStreamSynchronize(st_));
        std::vector<double> &bm = extra_d_["subset_binmap:" + key];
        bm.resize((size_t)npix * nms);
        expand_to_sky(b.get(), sizeof(double), nms, nosubpix_map_, bm.data());
        std::vector<int> mv(npix);
        expand_to_sky(msk.get(), sizeof(int), 1, nosubpix_map_, mv.data());
        std::vector<float> cv;
        std::vector<double> crawfull;
        if (pass == 1) {
          std::vector<int> &hh = extra_i_["subset_hits:" + key];
          hh.resize(npix);
          expand_to_sky(h.get(), sizeof(int), 1, nosubpix_map_, hh.data());
          extra_i_["subset_mask:" + key] = mv;
          cv.resize(npix);
          expand_to_sky(cr.get(), sizeof(float), 1, nosubpix_map_, cv.data());
          std::vector<double> &cf = extra_d_["subset_cc:" + key];
          const std::vector<double> full = full_sym(cinv, nms);
          cf.resize((size_t)npix * nms * nms);
          expand_host(full.data(), sizeof(double), nms * nms, nosubpix_map_, cf.data());
          if (!craw.empty()) {
            crawfull.resize((size_t)npix * nms * nms);
            expand_host(craw.data(), sizeof(double), nms * nms, nosubpix_map_, crawfull.data());
          }
        }
        if (!suppress_fits_ && writes_files()) {
          SubsetFits sf;
          sf.par = &par_;
          sf.nosubpix_map = nosubpix_map_;
          sf.nosubmaps_tot = nosubmaps_tot_;
          sf.ndet = ndet_;
          sf.nmap = nms;
          sf.pass = pass;
          sf.npass = npass;
          sf.isubchunk = isubchunk_;
          sf.nsubchunk = nsubchunk_;
          sf.set = p.detsets[ids].name;
          sf.survey = p.surveys[isv].name;
          sf.binmap = bm.data();
          sf.mask = mv.data();
          if (pass == 1) {
            sf.hits = extra_i_["subset_hits:" + key].data();
            sf.crit = cv.data();
            sf.cc_inv = extra_d_["subset_cc:" + key].data();
            sf.cc_raw = crawfull.empty() ? nullptr : crawfull.data();
          }
          sf.leak = leaks;
          write_subset_products(sf);
        }
        table.insert(table.end(), {(double)pass, (double)isv, (double)ids, (double)nms});
        ++k;
      }
    }
  }
  extra_d_["subsets"] = table;
  subset_spans_.clear();
}

std::vector<double> Engine::full_sym(const std::vector<double> &packed, int nmaps) {
  const int ncc = nmaps == 3 ? 6 : 1, nn = nmaps * nmaps;
  const size_t np = packed.size() / ncc;
  std::vector<double> o(np * nn);
  for (size_t p = 0; p < np; ++p) unpack_sym(&packed[p * ncc], nmaps, &o[p * nn]);
  return o;
}
