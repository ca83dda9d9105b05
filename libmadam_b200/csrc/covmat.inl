// Inverse noise covariance of the map (file_covmat), one dense matrix per
// detector.  Follows write_covmat (covmat.F90:48-186) and its helpers
// get_ptf (434-470), get_hitmap (358-431), get_middlematrix (474-530),
// add_white (190-222), symmetrize (226-244) and save_matrix (248-354):
//
//   N^-1 = P^T C_w^-1 P - sum over pointing periods of A M A^T,
//   A = P^T C_w^-1 F (pixels x baselines), M = Toeplitz(irfft(1 / (fcov +
//   nshort / sigma^2))) of the period's baselines,
//
// written as N x N native doubles (N = 12 nside_map^2 nmap), column-major,
// to <file_covmat>_<detector>_inv_bin.dat, -1 on the diagonal of unobserved
// pixels.
//
// On the device: the non-zeros of A are the distinct (pixel, baseline)
// pairs of the period samples, found by one radix sort of (pixel, baseline)
// keys and run-length encoding (the weights of a run are summed in time
// order, as get_ptf sums them); M comes from the FFT convolution of a unit
// impulse with each period's spectrum; the products A M A^T run one CTA per
// hit pixel p1 and one thread per pixel p2 >= p1, each thread summing its
// 3x3 block over the pairs of entries in a common period (a binary search
// finds p1's entries of the period of each of p2's entries) and storing the
// block and its transpose, so the dense matrix needs no atomics except for
// the white-noise diagonal.  Ranks add their matrices; rank 0 writes.

// sample keys: (global pixel << 32 | baseline) for samples of a period,
// all ones otherwise
__global__ void k_covmat_keys(const int32_t *pix, long long n, SampleMap sm, const int *seg_of,
                              int dummy, const int *sub2, int nosubpix, unsigned long long *keys,
                              uint32_t *idx) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x) {
    const int c = pix[s];
    const long long b = baseline_of(sm, 0, s);
    unsigned long long key = ~0ull;
    if (c != dummy && seg_of[b] >= 0) {
      const unsigned long long gp =
          (unsigned long long)c + (unsigned long long)sub2[c / nosubpix] * nosubpix;
      key = (gp << 32) | (unsigned long long)b;
    }
    keys[s] = key;
    idx[s] = (uint32_t)s;
  }
}

// get_ptf: the entry's summed weights times the period's 1/sigma^2
template <int NMAP>
__global__ void k_covmat_ptf(const unsigned long long *ukeys, const int *counts,
                             const int *offs, long long nent, const uint32_t *idx,
                             const float *w, int nnz, const int *seg_of, const double *seg_w,
                             int *ent_k, int *ent_p, double *ptf) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nent;
       e += (long long)gridDim.x * blockDim.x) {
    const unsigned long long key = ukeys[e];
    const int b = (int)(key & 0xffffffffull);
    double acc[NMAP];
#pragma unroll
    for (int c = 0; c < NMAP; ++c) acc[c] = 0;
    for (int j = offs[e]; j < offs[e] + counts[e]; ++j) {
      const long long s = idx[j];
#pragma unroll
      for (int c = 0; c < NMAP; ++c) acc[c] += (double)w[s * nnz + c];
    }
    const double dw = seg_w[seg_of[b]];
#pragma unroll
    for (int c = 0; c < NMAP; ++c) ptf[e * NMAP + c] = acc[c] != 0 ? acc[c] * dw : 0.0;
    ent_k[e] = b;
    ent_p[e] = (int)(key >> 32);
  }
}

// first index in [lo, hi) of the sorted ent_k with ent_k >= v
__device__ __forceinline__ int lower_bound_k(const int *ent_k, int lo, int hi, int v) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ent_k[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// the A M A^T blocks: CTA per hit pixel q1, threads over q2 >= q1
template <int NMAP>
__global__ void __launch_bounds__(256) k_covmat_pairs(
    const int *__restrict__ ent_k, const double *__restrict__ ptf, const int *__restrict__ poff,
    const int *__restrict__ hp, int nhit, const int *__restrict__ seg_of,
    const int *__restrict__ seg_k0, const int *__restrict__ seg_n,
    const long long *__restrict__ seg_m, const double *__restrict__ mm, double *G, long long N) {
  const int q1 = blockIdx.x;
  const int a0 = poff[q1], a1 = poff[q1 + 1];
  const long long p1 = hp[q1];
  for (int q2 = q1 + threadIdx.x; q2 < nhit; q2 += blockDim.x) {
    double acc[NMAP * NMAP];
#pragma unroll
    for (int e = 0; e < NMAP * NMAP; ++e) acc[e] = 0;
    for (int e2 = poff[q2]; e2 < poff[q2 + 1]; ++e2) {
      const int b2 = ent_k[e2];
      const int s = seg_of[b2];
      const int k0 = seg_k0[s], k1 = k0 + seg_n[s];
      double v2[NMAP];
#pragma unroll
      for (int c = 0; c < NMAP; ++c) v2[c] = ptf[(long long)e2 * NMAP + c];
      for (int e1 = lower_bound_k(ent_k, a0, a1, k0); e1 < a1; ++e1) {
        const int b1 = ent_k[e1];
        if (b1 >= k1) break;
        const double m = -mm[seg_m[s] + (b2 > b1 ? b2 - b1 : b1 - b2)];
#pragma unroll
        for (int b = 0; b < NMAP; ++b) {
          const double t = m * ptf[(long long)e1 * NMAP + b];
#pragma unroll
          for (int a = 0; a < NMAP; ++a) acc[a + NMAP * b] += v2[a] * t;
        }
      }
    }
    const long long p2 = hp[q2];
    if (q2 == q1) {
#pragma unroll
      for (int b = 0; b < NMAP; ++b)
#pragma unroll
        for (int a = 0; a < NMAP; ++a)
          G[(p1 * NMAP + b) * N + p1 * NMAP + a] += acc[a + NMAP * b];
    } else if (acc[0] != 0) {
      // the block (p2, p1) and, by symmetrize, its transpose at (p1, p2)
#pragma unroll
      for (int b = 0; b < NMAP; ++b)
#pragma unroll
        for (int a = 0; a < NMAP; ++a) {
          G[(p1 * NMAP + b) * N + p2 * NMAP + a] = acc[a + NMAP * b];
          G[(p2 * NMAP + a) * N + p1 * NMAP + b] = acc[a + NMAP * b];
        }
    }
  }
}

// add_white: detweight w w^T onto the diagonal blocks, every sample
template <int NMAP>
__global__ void k_covmat_white(const int32_t *pix, long long n, const float *w, int nnz,
                               int dummy, const int *sub2, int nosubpix, double detw, double *G,
                               long long N) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < n;
       s += (long long)gridDim.x * blockDim.x) {
    const int c = pix[s];
    if (c == dummy) continue;
    const long long p = c + (long long)sub2[c / nosubpix] * nosubpix;
#pragma unroll
    for (int b = 0; b < NMAP; ++b) {
      const double t = detw * (double)w[s * nnz + b];
#pragma unroll
      for (int a = 0; a < NMAP; ++a)
        atomicAdd(G + (p * NMAP + b) * N + p * NMAP + a, (double)w[s * nnz + a] * t);
    }
  }
}

// save_matrix's sentinel: -1 on the diagonal of pixels with an empty block
__global__ void k_covmat_sentinel(double *G, long long npix, int nmap, long long N) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix;
       p += (long long)gridDim.x * blockDim.x)
    if (G[(p * nmap) * N + p * nmap] == 0)
      for (int a = 0; a < nmap; ++a) G[(p * nmap + a) * N + p * nmap + a] = -1;
}

void Engine::write_covmat() {
  const int nmap = nmap_;
  const long long npix = 12LL * par_.nside_map * par_.nside_map, N = npix * nmap;
  if ((double)N * N * 8 > 64e9)
    fail("file_covmat: the " + std::to_string(N) + " x " + std::to_string(N) +
         " matrix does not fit the device");
  const long nh = nof_ / 2 + 1;
  const SampleMap sm = sample_map(istart_d_.get(), kstart_d_.get(), (int)ninterval_, nsamp_,
                                  noba_short_, fdn_);
  DevBuf<int> sub2;
  sub2.alloc(nosubmaps_tot_ + 1);
  std::vector<int> s2(subtable2_.begin(), subtable2_.end());
  s2.resize(nosubmaps_tot_ + 1, 0);
  MADAM_CUDA(cudaMemcpyAsync(sub2.get(), s2.data(), s2.size() * sizeof(int),
                             cudaMemcpyHostToDevice, st_));
  DevBuf<double> G;
  G.alloc((size_t)(N * N));
  std::vector<double> host;
  double detweight = 0;
  for (long d = 0; d < ndet_; ++d) {
    const std::string out = par_.file_covmat + "_" + dets_[d].name + "_inv_bin.dat";
    double there = 0;
    if (writes_files()) {
      FILE *f = std::fopen(out.c_str(), "rb");
      there = f != nullptr;
      if (f) std::fclose(f);
    }
    if (ar_sum_host(there) > 0) continue;
    G.zero(st_);
    // the pointing periods of the detector (trim_interval, as the residual
    // mask), skipping the rest of an interval without a PSD
    std::vector<int> seg_of(noba_short_, -1), seg_k0, seg_n, seg_psd;
    std::vector<long long> seg_m;
    std::vector<double> seg_w;
    long long mtot = 0;
    int last_iv = -1;
    bool skip_iv = false;
    for (const Segment &s : segs_) {
      if (s.det != d) continue;
      if (s.iv != last_iv) {
        last_iv = s.iv;
        skip_iv = false;
      }
      if (skip_iv) continue;
      const long ks = s.k0 - d * noba_short_;
      const int ipd = psd_index_det(dets_[d], btime_[ks]);
      if (ipd < 0) {
        skip_iv = true;
        continue;
      }
      detweight = 1 / (dets_[d].sigmas[ipd] * dets_[d].sigmas[ipd]);
      if (detweight == 0) {
        skip_iv = true;
        continue;
      }
      if (nof_ < 2 * s.noba)
        fail("ERROR: filter is too short to reliably estimate the middle matrix");
      const int id = (int)seg_k0.size();
      for (long k = 0; k < s.noba; ++k) seg_of[ks + k] = id;
      seg_k0.push_back((int)ks);
      seg_n.push_back((int)s.noba);
      seg_m.push_back(mtot);
      seg_w.push_back(detweight);
      seg_psd.push_back(psd_index_global(psddet_, psdstart_, psdstop_, d, btime_[ks]));
      mtot += s.noba;
    }
    const int nseg = (int)seg_k0.size();
    const long long n = nsamp_;
    const int32_t *pixd = pix_.get() + (size_t)d * nsamp_;
    // the raw weights: the caller's device buffer or the staging copy kept
    // for this call (flag_and_compact)
    const float *wd = d_w_ + (size_t)d * nsamp_ * nnz_;
    if (nseg > 0) {
      // get_middlematrix: M = irfft(1 / (fcov + nshort / sigma^2)), from the
      // convolution of a unit impulse per period
      std::vector<double> spec((size_t)nseg * nh);
      for (int i = 0; i < nseg; ++i)
        for (long k = 0; k < nh; ++k)
          spec[(size_t)i * nh + k] =
              1.0 / (fcov_host()[(size_t)seg_psd[i] * nh + k] + (double)nshort_ * seg_w[i]);
      std::vector<double> imp(mtot, 0.0);
      std::vector<ConvSeg> cs(nseg);
      for (int i = 0; i < nseg; ++i) {
        imp[seg_m[i]] = 1.0;
        cs[i] = ConvSeg{seg_m[i], seg_m[i], 1, seg_n[i], i, 0};
      }
      DevBuf<double> dspec, dimp, dmm;
      DevBuf<ConvSeg> dcs;
      dspec.alloc(spec.size());
      dimp.alloc(mtot);
      dmm.alloc(mtot);
      dcs.alloc(nseg);
      MADAM_CUDA(cudaMemcpyAsync(dspec.get(), spec.data(), spec.size() * sizeof(double),
                                 cudaMemcpyHostToDevice, st_));
      MADAM_CUDA(cudaMemcpyAsync(dimp.get(), imp.data(), mtot * sizeof(double),
                                 cudaMemcpyHostToDevice, st_));
      MADAM_CUDA(cudaMemcpyAsync(dcs.get(), cs.data(), nseg * sizeof(ConvSeg),
                                 cudaMemcpyHostToDevice, st_));
      fft_->reserve(nseg);
      fft_->convolve(st_, dcs.get(), nseg, dspec.get(), (long)(spec.size() / nh), dimp.get(),
                     dmm.get());
      fft_->forget_spectra();  // dspec is a temporary
      // the non-zeros of P^T F: sorted (pixel, baseline) keys, run-length
      // encoded
      DevBuf<int> dseg_of, dk0, dn;
      DevBuf<long long> dm;
      DevBuf<double> dw;
      dseg_of.alloc(noba_short_);
      dk0.alloc(nseg);
      dn.alloc(nseg);
      dm.alloc(nseg);
      dw.alloc(nseg);
      MADAM_CUDA(cudaMemcpyAsync(dseg_of.get(), seg_of.data(), noba_short_ * sizeof(int),
                                 cudaMemcpyHostToDevice, st_));
      MADAM_CUDA(cudaMemcpyAsync(dk0.get(), seg_k0.data(), nseg * sizeof(int),
                                 cudaMemcpyHostToDevice, st_));
      MADAM_CUDA(cudaMemcpyAsync(dn.get(), seg_n.data(), nseg * sizeof(int),
                                 cudaMemcpyHostToDevice, st_));
      MADAM_CUDA(cudaMemcpyAsync(dm.get(), seg_m.data(), nseg * sizeof(long long),
                                 cudaMemcpyHostToDevice, st_));
      MADAM_CUDA(cudaMemcpyAsync(dw.get(), seg_w.data(), nseg * sizeof(double),
                                 cudaMemcpyHostToDevice, st_));
      DevBuf<unsigned long long> keys, keys2, ukeys;
      DevBuf<uint32_t> idx, idx2;
      DevBuf<int> counts, offs, nrun;
      keys.alloc(n);
      keys2.alloc(n);
      ukeys.alloc(n);
      idx.alloc(n);
      idx2.alloc(n);
      counts.alloc(n);
      offs.alloc(n + 1);
      nrun.alloc(1);
      MADAM_LAUNCH(k_covmat_keys, grid_for(n), 256, 0, st_, pixd, n, sm, dseg_of.get(),
                   (int)dummy_local_, sub2.get(), (int)nosubpix_max_, keys.get(), idx.get());
      size_t tb = 0, tb2 = 0, tb3 = 0;
      MADAM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.get(), keys2.get(), idx.get(),
                                                 idx2.get(), (int)n, 0, 64, st_));
      MADAM_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, tb2, keys2.get(), ukeys.get(),
                                                    counts.get(), nrun.get(), (int)n, st_));
      MADAM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb3, counts.get(), offs.get(), (int)n,
                                               st_));
      DevBuf<uint8_t> tmp;
      tmp.alloc(std::max({tb, tb2, tb3, (size_t)1}));
      MADAM_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, keys.get(), keys2.get(),
                                                 idx.get(), idx2.get(), (int)n, 0, 64, st_));
      MADAM_CUDA(cub::DeviceRunLengthEncode::Encode(tmp.get(), tb2, keys2.get(), ukeys.get(),
                                                    counts.get(), nrun.get(), (int)n, st_));
      int nr = 0;
      MADAM_CUDA(cudaMemcpyAsync(&nr, nrun.get(), sizeof nr, cudaMemcpyDeviceToHost, st_));
      MADAM_CUDA(cudaStreamSynchronize(st_));
      unsigned long long lastkey = 0;
      if (nr > 0)
        MADAM_CUDA(cudaMemcpy(&lastkey, ukeys.get() + nr - 1, sizeof lastkey,
                              cudaMemcpyDeviceToHost));
      const int nent = nr - (nr > 0 && lastkey == ~0ull ? 1 : 0);
      if (nent > 0) {
        MADAM_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tb3, counts.get(), offs.get(), nent,
                                                 st_));
        DevBuf<int> ent_k, ent_p;
        DevBuf<double> ptf;
        ent_k.alloc(nent);
        ent_p.alloc(nent);
        ptf.alloc((size_t)nent * nmap);
        if (nmap == 3)
          MADAM_LAUNCH(k_covmat_ptf<3>, grid_for(nent), 256, 0, st_, ukeys.get(), counts.get(),
                       offs.get(), (long long)nent, idx2.get(), wd, (int)nnz_, dseg_of.get(),
                       dw.get(), ent_k.get(), ent_p.get(), ptf.get());
        else
          MADAM_LAUNCH(k_covmat_ptf<1>, grid_for(nent), 256, 0, st_, ukeys.get(), counts.get(),
                       offs.get(), (long long)nent, idx2.get(), wd, (int)nnz_, dseg_of.get(),
                       dw.get(), ent_k.get(), ent_p.get(), ptf.get());
        // entries per hit pixel
        DevBuf<int> hp, pcount, poff, nhp;
        hp.alloc(nent);
        pcount.alloc(nent + 1);
        poff.alloc(nent + 1);
        nhp.alloc(1);
        size_t tb4 = 0, tb5 = 0;
        MADAM_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, tb4, ent_p.get(), hp.get(),
                                                      pcount.get(), nhp.get(), nent, st_));
        MADAM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb5, pcount.get(), poff.get(),
                                                 nent + 1, st_));
        DevBuf<uint8_t> tmp2;
        tmp2.alloc(std::max({tb4, tb5, (size_t)1}));
        MADAM_CUDA(cub::DeviceRunLengthEncode::Encode(tmp2.get(), tb4, ent_p.get(), hp.get(),
                                                      pcount.get(), nhp.get(), nent, st_));
        int nhit = 0;
        MADAM_CUDA(cudaMemcpyAsync(&nhit, nhp.get(), sizeof nhit, cudaMemcpyDeviceToHost, st_));
        MADAM_CUDA(cudaStreamSynchronize(st_));
        // poff[nhit] = nent: the scan over nhit + 1 counts with a zero after
        MADAM_CUDA(cudaMemsetAsync(pcount.get() + nhit, 0, sizeof(int), st_));
        MADAM_CUDA(cub::DeviceScan::ExclusiveSum(tmp2.get(), tb5, pcount.get(), poff.get(),
                                                 nhit + 1, st_));
        if (nmap == 3)
          MADAM_LAUNCH(k_covmat_pairs<3>, (unsigned)nhit, 256, 0, st_, ent_k.get(), ptf.get(),
                       poff.get(), hp.get(), nhit, dseg_of.get(), dk0.get(), dn.get(), dm.get(),
                       dmm.get(), G.get(), N);
        else
          MADAM_LAUNCH(k_covmat_pairs<1>, (unsigned)nhit, 256, 0, st_, ent_k.get(), ptf.get(),
                       poff.get(), hp.get(), nhit, dseg_of.get(), dk0.get(), dn.get(), dm.get(),
                       dmm.get(), G.get(), N);
        MADAM_CUDA(cudaStreamSynchronize(st_));
      }
    }
    if (nmap == 3)
      MADAM_LAUNCH(k_covmat_white<3>, grid_for(n), 256, 0, st_, pixd, n, wd, (int)nnz_,
                   (int)dummy_local_, sub2.get(), (int)nosubpix_max_, detweight, G.get(), N);
    else
      MADAM_LAUNCH(k_covmat_white<1>, grid_for(n), 256, 0, st_, pixd, n, wd, (int)nnz_,
                   (int)dummy_local_, sub2.get(), (int)nosubpix_max_, detweight, G.get(), N);
    ar_sum(G.get(), (size_t)(N * N));  // save_matrix's sum over the ranks
    MADAM_LAUNCH(k_covmat_sentinel, grid_for(npix), 256, 0, st_, G.get(), npix, nmap, N);
    if (writes_files()) {
      host.resize((size_t)(N * N));
      MADAM_CUDA(cudaMemcpyAsync(host.data(), G.get(), host.size() * sizeof(double),
                                 cudaMemcpyDeviceToHost, st_));
      MADAM_CUDA(cudaStreamSynchronize(st_));
      FILE *f = std::fopen(out.c_str(), "wb");
      if (!f) fail("Unable to open covmat file");
      const bool ok = std::fwrite(host.data(), sizeof(double), host.size(), f) == host.size();
      std::fclose(f);
      if (!ok) fail("Failed to write covmat file");
    }
    MADAM_CUDA(cudaStreamSynchronize(st_));
  }
}
