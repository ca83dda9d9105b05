// Destriping with higher-order baselines (basis_order > 0): every baseline
// carries basis_order + 1 amplitudes of a function basis (Legendre,
// polynomial, Chebyshev or real Fourier) evaluated over its samples.
//
// Follows the reference's basis_order > 0 path: the basis tables of
// start_timeloop (parameter_control.f90:853-933), initialize_a's right-hand
// side and F^T F blocks with their eigen-decomposed inverses
// (smadam_routines.f90:505-671), the projections baseline_to_map_{nopol,
// general} / map_to_baseline_{nopol,general} (1140-1226, 1379-1480), the
// block-diagonal preconditioner (943-957), subtract_baselines_a (1489-1539)
// and clean_tod (1545-1585).  The reference has no noise filter for this
// path (parameter_control.f90:617-618 refuses kfilter).
//
// Layout: amplitudes [baseline][order] (nb x NB doubles), blocks
// [baseline][NB x NB column-major].  One warp per baseline streams its
// samples (coalesced pointing loads); the basis values are evaluated per
// sample in registers instead of being read from tables.  The projections
// onto the map use FP64 atomics into the local map.

// basis function values of sample u of a baseline of `len` samples.  The
// reference's `dr = 2. / nsamp` divides in single precision; explicit
// round-to-nearest operations keep the reference's operation order (no
// contraction into fused multiply-adds).
template <int NB>
__device__ __forceinline__ void basis_eval(int func, long long u, long long len,
                                           double (&f)[NB]) {
  const double dr = (double)__fdiv_rn(2.0f, __ll2float_rn(len));
  const double rstart = __dsub_rn(__dmul_rn(0.5, dr), 1.0);
  const double r = __dadd_rn(rstart, __dmul_rn((double)u, dr));
  if (func == 1) {  // polynomial: r**o by binary powering
#pragma unroll
    for (int o = 0; o < NB; ++o) {
      double out = 1, x = r;
      int n = o;
      while (n > 0) {
        if (n & 1) out = __dmul_rn(out, x);
        n >>= 1;
        if (n) x = __dmul_rn(x, x);
      }
      f[o] = out;
    }
  } else if (func == 2) {  // real Fourier
    const double x = __dmul_rn((double)u, __ddiv_rn(3.141592653589793238462643383279502884197,
                                                    (double)len));
#pragma unroll
    for (int o = 0; o < NB; ++o)
      f[o] = (o % 2 == 0) ? cos(__dmul_rn((double)o, x)) : sin(__dmul_rn((double)(o + 1), x));
  } else if (func == 3) {  // Chebyshev (second kind) times (1 - r^2)^(1/4)
    const double r2 = __dmul_rn(2.0, r);
#pragma unroll
    for (int o = 0; o < NB; ++o)
      f[o] = o == 0 ? 1.0 : o == 1 ? r2 : __dsub_rn(__dmul_rn(r2, f[o - 1]), f[o - 2]);
    const double g = pow(__dsub_rn(1.0, __dmul_rn(r, r)), 0.25);
#pragma unroll
    for (int o = 0; o < NB; ++o) f[o] = __dmul_rn(f[o], g);
  } else {  // Legendre
#pragma unroll
    for (int o = 0; o < NB; ++o)
      f[o] = o == 0 ? 1.0
             : o == 1
                 ? r
                 : __ddiv_rn(__dsub_rn(__dmul_rn(__dmul_rn((double)(2 * o - 1), r), f[o - 1]),
                                       __dmul_rn((double)(o - 1), f[o - 2])),
                             (double)o);
  }
}

// initialize_a (smadam_routines.f90:505-576): yba(o) = detw sum f_o (tod -
// w.m) and nna(o2, o) = detw sum f_o f_o2 over the baseline's samples
// whose pixel survives (a zero map marks masked or rejected pixels)
template <int NMAP, int NB>
__global__ void __launch_bounds__(256) k_init_a_basis(
    const float4 *p4, const int32_t *pc, const double *tod, const uint32_t *bstart, long long nb,
    long noba, long long nsamp, const double *bw, const double *wamap, int deg_shift, int nloc,
    int func, double *yba, double *nna) {
  constexpr int NT = NB * (NB + 1) / 2;
  const long long b = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (b >= nb) return;
  const double detw = bw[b];
  if (detw == 0) return;
  const long long det = b / noba, k = b - det * noba;
  const long long i0 = det * nsamp + bstart[k], len = (long long)bstart[k + 1] - bstart[k];
  double y[NB], n[NT];
#pragma unroll
  for (int o = 0; o < NB; ++o) y[o] = 0;
#pragma unroll
  for (int e = 0; e < NT; ++e) n[e] = 0;
  for (long long u = lane; u < len; u += 32) {
    const long long i = i0 + u;
    int px;
    float4 q;
    if (NMAP == 3) {
      q = p4[i];
      px = point_pix(q);
    } else {
      px = pc[i];
    }
    if (px >= nloc) continue;
    const long long pcr = px >> deg_shift;
    double mw;
    if (NMAP == 3) {
      const double m0 = wamap[pcr * 3], m1 = wamap[pcr * 3 + 1], m2 = wamap[pcr * 3 + 2];
      if (m0 == 0 && m1 == 0 && m2 == 0) continue;
      mw = m0 * (double)q.x + m1 * (double)q.y + m2 * (double)q.z;
    } else {
      mw = wamap[pcr];
      if (mw == 0) continue;
    }
    double f[NB];
    basis_eval<NB>(func, u, len, f);
    const double t = tod[i];
    int e = 0;
#pragma unroll
    for (int o = 0; o < NB; ++o) {
      y[o] += f[o] * t - f[o] * mw;
#pragma unroll
      for (int o2 = o; o2 < NB; ++o2) n[e++] += f[o] * f[o2];
    }
  }
#pragma unroll
  for (int o = 0; o < NB; ++o) y[o] = warp_sum(y[o]);
#pragma unroll
  for (int e = 0; e < NT; ++e) n[e] = warp_sum(n[e]);
  if (lane == 0) {
    int e = 0;
#pragma unroll
    for (int o = 0; o < NB; ++o) {
      yba[b * NB + o] = y[o] * detw;
#pragma unroll
      for (int o2 = o; o2 < NB; ++o2) {
        const double v = n[e++] * detw;
        nna[b * NB * NB + o2 + NB * o] = v;
        nna[b * NB * NB + o + NB * o2] = v;
      }
    }
  }
}

// cyclic Jacobi eigen-decomposition of a symmetric N x N matrix (column-
// major, overwritten); w eigenvalues, v eigenvectors as columns.  Stands in
// for LAPACK dsyev; returns 1 on a NaN eigenvalue.
template <int N>
__device__ int jacobi_n(double *A, double *w, double *v) {
  for (int i = 0; i < N * N; ++i) v[i] = 0;
  for (int i = 0; i < N; ++i) v[i + N * i] = 1;
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = 0, diag = 0;
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i) {
        const double x = A[i + N * j] * A[i + N * j];
        if (i != j) off += x;
        else diag += x;
      }
    if (off == 0 || off <= 1e-34 * diag) break;
    for (int p = 0; p < N - 1; ++p)
      for (int q = p + 1; q < N; ++q) {
        const double apq = A[p + N * q];
        if (apq == 0) continue;
        const double app = A[p + N * p], aqq = A[q + N * q];
        const double theta = (aqq - app) / (2 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
        if (isinf(theta)) t = 0.5 / theta;
        const double c = 1 / sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < N; ++k) {
          const double akp = A[k + N * p], akq = A[k + N * q];
          A[k + N * p] = c * akp - s * akq;
          A[k + N * q] = s * akp + c * akq;
        }
        for (int k = 0; k < N; ++k) {
          const double apk = A[p + N * k], aqk = A[q + N * k];
          A[p + N * k] = c * apk - s * aqk;
          A[q + N * k] = s * apk + c * aqk;
        }
        for (int k = 0; k < N; ++k) {
          const double vkp = v[k + N * p], vkq = v[k + N * q];
          v[k + N * p] = c * vkp - s * vkq;
          v[k + N * q] = s * vkp + c * vkq;
        }
      }
  }
  int bad = 0;
  for (int i = 0; i < N; ++i) {
    w[i] = A[i + N * i];
    if (isnan(w[i])) bad = 1;
  }
  return bad;
}

// the F^T F inverses of initialize_a (smadam_routines.f90:578-653): empty
// blocks (nna(0,0) below 1e-30) zero the baseline, degenerate ones
// (eigenvalue ratio below 1e-12) keep the inverse diagonal, the others get
// V diag(1/w) V^T.  One thread per baseline.
template <int NB>
__global__ void k_nna_inv(double *nna, double *yba, double *inv, const double *bw,
                          long long nb) {
  constexpr int NN = NB * NB;
  const long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (b >= nb || bw[b] == 0) return;
  double *n = nna + b * NN, *y = yba + b * NB, *out = inv + b * NN;
  for (int e = 0; e < NN; ++e) out[e] = 0;
  double w[NB], v[NN], A[NN];
  int ierr = 0;
  if (fabs(n[0]) < (double)1e-30f) {
    for (int i = 0; i < NB; ++i) w[i] = 0;
    for (int e = 0; e < NN; ++e) v[e] = 0;
  } else {
    for (int e = 0; e < NN; ++e) A[e] = n[e];
    ierr = jacobi_n<NB>(A, w, v);
  }
  double wmin = w[0], wmax = w[0];
  for (int i = 1; i < NB; ++i) {
    wmin = fmin(wmin, w[i]);
    wmax = fmax(wmax, w[i]);
  }
  if (ierr != 0) {
    for (int e = 0; e < NN; ++e) n[e] = 0;
    for (int o = 0; o < NB; ++o) y[o] = 0;
  } else if (wmin == 0 && wmax == 0) {
    for (int e = 0; e < NN; ++e) n[e] = 0;
    for (int o = 0; o < NB; ++o) y[o] = 0;
    return;
  } else if (wmin / wmax < (double)1e-12f) {
    for (int j = 0; j < NB; ++j) out[j + NB * j] = 1 / n[j + NB * j];
    return;
  }
  for (int a = 0; a < NB; ++a)
    for (int c = 0; c < NB; ++c) {
      double t = 0;
      for (int i = 0; i < NB; ++i) t += (v[a + NB * i] / w[i]) * v[c + NB * i];
      out[a + NB * c] = t;
    }
}

// z = nna_inv r per baseline (apply_preconditioner, 943-957)
template <int NB>
__global__ void k_basis_precond(const double *inv, const double *r, double *z, long long nb) {
  const long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (b >= nb) return;
  double rv[NB];
#pragma unroll
  for (int c = 0; c < NB; ++c) rv[c] = r[b * NB + c];
#pragma unroll
  for (int a = 0; a < NB; ++a) {
    double t = 0;
#pragma unroll
    for (int c = 0; c < NB; ++c) t += inv[b * NB * NB + a + NB * c] * rv[c];
    z[b * NB + a] = t;
  }
}

// target[pix] += sign * detw * (f . amp) * w over every sample
// (baseline_to_map_* / subtract_baselines_a); one warp per baseline
template <int NMAP, int NB>
__global__ void __launch_bounds__(256) k_scatter_basis(
    const float4 *p4, const int32_t *pc, const uint32_t *bstart, long long nb, long noba,
    long long nsamp, const double *bw, const double *amp, double sign, int deg_shift, int nloc,
    int func, double *target) {
  const int lane = threadIdx.x & 31;
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long b = warp0; b < nb; b += nwarps) {
    const double detw = bw[b];
    if (detw == 0) continue;
    double a[NB];
#pragma unroll
    for (int o = 0; o < NB; ++o) a[o] = amp[b * NB + o];
    const long long det = b / noba, k = b - det * noba;
    const long long i0 = det * nsamp + bstart[k], len = (long long)bstart[k + 1] - bstart[k];
    for (long long u = lane; u < len; u += 32) {
      const long long i = i0 + u;
      int px;
      float4 q;
      if (NMAP == 3) {
        q = p4[i];
        px = point_pix(q);
      } else {
        px = pc[i];
      }
      if (px >= nloc) continue;
      double f[NB];
      basis_eval<NB>(func, u, len, f);
      double dp = 0;
#pragma unroll
      for (int o = 0; o < NB; ++o) dp += f[o] * a[o];
      const double pw = sign * (dp * detw);
      const long long pcr = px >> deg_shift;
      if (NMAP == 3) {
        atomicAdd(target + pcr * 3 + 0, (double)q.x * pw);
        atomicAdd(target + pcr * 3 + 1, (double)q.y * pw);
        atomicAdd(target + pcr * 3 + 2, (double)q.z * pw);
      } else {
        atomicAdd(target + pcr, pw);
      }
    }
  }
}

// map_to_baseline_{nopol,general} (1379-1480) + "ap = ap + ..." (870) and
// the partial p.ap (877): apnv(o) = sum f_o w.m, ap = ap + nna p - detw apnv
template <int NMAP, int NB>
__global__ void __launch_bounds__(256) k_gather_basis(
    const float4 *p4, const int32_t *pc, const uint32_t *bstart, long long nb, long noba,
    long long nsamp, const double *bw, const double *p, const double *nna, const double *m,
    int deg_shift, int nloc, int func, const uint8_t *rmask, double *ap, double *part) {
  const int lane = threadIdx.x & 31;
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  double pap = 0;
  for (long long b = warp0; b < nb; b += nwarps) {
    const double detw = bw[b];
    if (detw == 0) {
      if (lane == 0 && rmask[b])
        for (int o = 0; o < NB; ++o) pap += p[b * NB + o] * ap[b * NB + o];
      continue;
    }
    const long long det = b / noba, k = b - det * noba;
    const long long i0 = det * nsamp + bstart[k], len = (long long)bstart[k + 1] - bstart[k];
    double acc[NB];
#pragma unroll
    for (int o = 0; o < NB; ++o) acc[o] = 0;
    for (long long u = lane; u < len; u += 32) {
      const long long i = i0 + u;
      double mw;
      if (NMAP == 3) {
        const float4 q = p4[i];
        const int px = point_pix(q);
        if (px >= nloc) continue;
        const double *mm = m + (long long)(px >> deg_shift) * 3;
        mw = (double)q.x * mm[0] + (double)q.y * mm[1] + (double)q.z * mm[2];
      } else {
        const int px = pc[i];
        if (px >= nloc) continue;
        mw = m[px >> deg_shift];
      }
      double f[NB];
      basis_eval<NB>(func, u, len, f);
#pragma unroll
      for (int o = 0; o < NB; ++o) acc[o] += mw * f[o];
    }
#pragma unroll
    for (int o = 0; o < NB; ++o) acc[o] = warp_sum(acc[o]);
    if (lane == 0) {
#pragma unroll
      for (int a = 0; a < NB; ++a) {
        double t = 0;
#pragma unroll
        for (int c = 0; c < NB; ++c) t += nna[b * NB * NB + a + NB * c] * p[b * NB + c];
        const double v = ap[b * NB + a] + (t - acc[a] * detw);
        ap[b * NB + a] = v;
        if (rmask[b]) pap += p[b * NB + a] * v;
      }
    }
  }
  double v[1] = {pap};
  block_sum<1>(v);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// clean_tod (1545-1585): tod -= sum_o f_o aa_o over every sample
template <int NB>
__global__ void __launch_bounds__(256) k_clean_tod_basis(double *tod, const uint32_t *bstart,
                                                          long long nb, long noba,
                                                          long long nsamp, int func,
                                                          const double *aa) {
  const int lane = threadIdx.x & 31;
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long b = warp0; b < nb; b += nwarps) {
    double a[NB];
#pragma unroll
    for (int o = 0; o < NB; ++o) a[o] = aa[b * NB + o];
    const long long det = b / noba, k = b - det * noba;
    const long long i0 = det * nsamp + bstart[k], len = (long long)bstart[k + 1] - bstart[k];
    for (long long u = lane; u < len; u += 32) {
      double f[NB];
      basis_eval<NB>(func, u, len, f);
      double t = tod[i0 + u];
#pragma unroll
      for (int o = 0; o < NB; ++o) t = t - f[o] * a[o];
      tod[i0 + u] = t;
    }
  }
}

// ap(o) = nna(o, o) p(o) diagfilter (iterate_a 833-842)
template <int NB>
__global__ void k_diagfilter_basis(double *ap, const double *nna, const double *p, double f,
                                   long long nb) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= nb * NB) return;
  const long long b = i / NB;
  const int o = (int)(i - b * NB);
  ap[i] = nna[b * NB * NB + o * (NB + 1)] * p[i] * f;
}

// per-baseline values repeated for each order
template <typename T>
__global__ void k_repeat(const T *src, long long n, int r, T *dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n * r;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = src[i / r];
}

// ------------------------------------------------------------ host side --

// calls f(std::integral_constant<int, NB>) for the run's basis size
template <typename F>
void with_basis(int nbasis, F &&f) {
  switch (nbasis) {
    case 2: f(std::integral_constant<int, 2>()); break;
    case 3: f(std::integral_constant<int, 3>()); break;
    case 4: f(std::integral_constant<int, 4>()); break;
    case 5: f(std::integral_constant<int, 5>()); break;
    case 6: f(std::integral_constant<int, 6>()); break;
    case 7: f(std::integral_constant<int, 7>()); break;
    case 8: f(std::integral_constant<int, 8>()); break;
    default: fail("basis_order above " + std::to_string(kMaxBasis - 1) + " is not supported");
  }
}

void Engine::initialize_a_basis() {
  const long long nb = (long long)ndet_ * noba_short_;
  const int NBv = nbasis_;
  yba_.alloc(nb * NBv);
  nna_.alloc(nb * NBv * NBv);
  nna_inv_.alloc(nb * NBv * NBv);
  aa_.alloc(nb * NBv);
  yba_.zero(st_);
  nna_.zero(st_);
  nna_inv_.zero(st_);
  aa_.zero(st_);
  if (nb > 0) {
    const unsigned grid = (unsigned)((nb * 32 + 255) / 256);
    with_basis(nbasis_, [&](auto nbc) {
      constexpr int NB = decltype(nbc)::value;
      if (nmap_ == 3)
        MADAM_LAUNCH((k_init_a_basis<3, NB>), grid, 256, 0, st_, point4_.get(), pixc_.get(),
                     d_tod_, bstart_d_.get(), nb, noba_short_, nsamp_, bw_.get(), wamap_.get(),
                     (int)ndeg_shift_, (int)nloc_, par_.basis_func, yba_.get(), nna_.get());
      else
        MADAM_LAUNCH((k_init_a_basis<1, NB>), grid, 256, 0, st_, point4_.get(), pixc_.get(),
                     d_tod_, bstart_d_.get(), nb, noba_short_, nsamp_, bw_.get(), wamap_.get(),
                     (int)ndeg_shift_, (int)nloc_, par_.basis_func, yba_.get(), nna_.get());
      MADAM_LAUNCH(k_nna_inv<NB>, (unsigned)((nb + 127) / 128), 128, 0, st_, nna_.get(),
                   yba_.get(), nna_inv_.get(), bw_.get(), nb);
    });
  }
  // the blocks' (0, 0) elements mark the empty baselines (trim_interval)
  nna_host_.resize(nb);
  if (nb > 0)
    MADAM_CUDA(cudaMemcpy2DAsync(nna_host_.data(), sizeof(double), nna_.get(),
                                 (size_t)NBv * NBv * sizeof(double), sizeof(double), (size_t)nb,
                                 cudaMemcpyDeviceToHost, st_));
  MADAM_CUDA(cudaStreamSynchronize(st_));
}

void Engine::basis_vectors() {
  // per-amplitude detector weights and residual mask for the CG vectors
  const long long nb = (long long)ndet_ * noba_short_;
  bwn_.alloc(std::max<long long>(1, nb * nbasis_));
  rmaskn_.alloc(std::max<long long>(1, nb * nbasis_));
  if (nb == 0) return;
  MADAM_LAUNCH(k_repeat<double>, grid_for(nb * nbasis_), 256, 0, st_, bw_.get(), nb, nbasis_,
               bwn_.get());
  MADAM_LAUNCH(k_repeat<uint8_t>, grid_for(nb * nbasis_), 256, 0, st_, rmask_.get(), nb,
               nbasis_, rmaskn_.get());
}

void Engine::scatter_basis(const double *amp, double sign, double *target, bool fine) {
  const long long nb = (long long)ndet_ * noba_short_;
  if (nb == 0) return;
  const int deg = fine ? 0 : (int)ndeg_shift_;
  with_basis(nbasis_, [&](auto nbc) {
    constexpr int NB = decltype(nbc)::value;
    if (nmap_ == 3)
      MADAM_LAUNCH((k_scatter_basis<3, NB>), grid_for(nb * 32), 256, 0, st_, point4_.get(),
                   pixc_.get(), bstart_d_.get(), nb, noba_short_, nsamp_, bw_.get(), amp, sign,
                   deg, (int)nloc_, par_.basis_func, target);
    else
      MADAM_LAUNCH((k_scatter_basis<1, NB>), grid_for(nb * 32), 256, 0, st_, point4_.get(),
                   pixc_.get(), bstart_d_.get(), nb, noba_short_, nsamp_, bw_.get(), amp, sign,
                   deg, (int)nloc_, par_.basis_func, target);
  });
}

void Engine::apply_A_basis(const double *p, double *ap, bool timed) {
  const long long nb = (long long)ndet_ * noba_short_;
  if (timed) MADAM_CUDA(cudaEventRecord(ev_[0], st_));
  if (nloc_cross_ > 0) lmap_.zero(st_);
  scatter_basis(p, 1.0, lmap_.get(), false);
  ar_sum(lmap_.get(), (size_t)nloc_cross_ * nmap_);  // collect_map across the ranks
  if (timed) MADAM_CUDA(cudaEventRecord(ev_[1], st_));
  if (nloc_cross_ > 0) {
    if (nmap_ == 3)
      MADAM_LAUNCH(k_ccmult<3>, grid_for(nloc_cross_), 256, 0, st_, cca_.get(), lmap_.get(),
                   (long long)nloc_cross_);
    else
      MADAM_LAUNCH(k_ccmult<1>, grid_for(nloc_cross_), 256, 0, st_, cca_.get(), lmap_.get(),
                   (long long)nloc_cross_);
  }
  if (timed) MADAM_CUDA(cudaEventRecord(ev_[2], st_));
  with_basis(nbasis_, [&](auto nbc) {
    constexpr int NB = decltype(nbc)::value;
    if (par_.diagfilter != 0)
      MADAM_LAUNCH(k_diagfilter_basis<NB>, grid_for(nb * NB), 256, 0, st_, ap, nna_.get(), p,
                   par_.diagfilter, nb);
    else
      MADAM_CUDA(cudaMemsetAsync(ap, 0, nb * NB * sizeof(double), st_));
    if (timed) MADAM_CUDA(cudaEventRecord(ev_[3], st_));
    if (nmap_ == 3)
      MADAM_LAUNCH((k_gather_basis<3, NB>), kRedBlocks, 256, 0, st_, point4_.get(), pixc_.get(),
                   bstart_d_.get(), nb, noba_short_, nsamp_, bw_.get(), p, nna_.get(),
                   lmap_.get(), (int)ndeg_shift_, (int)nloc_, par_.basis_func, rmask_.get(), ap,
                   part_.get());
    else
      MADAM_LAUNCH((k_gather_basis<1, NB>), kRedBlocks, 256, 0, st_, point4_.get(), pixc_.get(),
                   bstart_d_.get(), nb, noba_short_, nsamp_, bw_.get(), p, nna_.get(),
                   lmap_.get(), (int)ndeg_shift_, (int)nloc_, par_.basis_func, rmask_.get(), ap,
                   part_.get());
  });
  finish_dots(1, 1, 0, kRedBlocks, true);
  if (timed) MADAM_CUDA(cudaEventRecord(ev_[4], st_));
}

void Engine::precondition_basis(const double *r, double *z) {
  const long long nb = (long long)ndet_ * noba_short_;
  if (nb == 0) return;
  with_basis(nbasis_, [&](auto nbc) {
    constexpr int NB = decltype(nbc)::value;
    MADAM_LAUNCH(k_basis_precond<NB>, (unsigned)((nb + 255) / 256), 256, 0, st_,
                 nna_inv_.get(), r, z, nb);
  });
}

void Engine::clean_tod_basis() {
  const long long nb = (long long)ndet_ * noba_short_;
  if (nb == 0) return;
  with_basis(nbasis_, [&](auto nbc) {
    constexpr int NB = decltype(nbc)::value;
    MADAM_LAUNCH(k_clean_tod_basis<NB>, grid_for(nb * 32), 256, 0, st_, d_tod_,
                 bstart_d_.get(), nb, noba_short_, nsamp_, par_.basis_func, aa_.get());
  });
}

