// The four-step passes of fft.cu, included once per arithmetic: FFT_NS
// names the namespace, FFT_CPLX / FFT_REAL / FFT_MK the complex type, its
// real type and its constructor (double2 for the float64 solves, float2 for
// the float32-TOD batch's filter).  The arithmetic is the same line for line.
namespace FFT_NS {

typedef FFT_CPLX cplx;
typedef FFT_REAL real;
#define MK_C FFT_MK

// Real-spectrum split of the packed transform for the pair (k, N-k), product
// with the real spectrum H and re-packing for the inverse transform.
// A = Z[k], B = Z[N-k], W = exp(-i pi k / N), Hk = H[k], Hnk = H[N-k]; on
// return A = Z'[k], B = Z'[N-k].  dc (k == 0) handles the DC / Nyquist pair
// with Hk = H[0], Hnk = H[N] (B is ignored and set equal to A).
__device__ __forceinline__ void spectral_pair(cplx &A, cplx &B, bool dc, cplx W, real Hk, real Hnk) {
  if (dc) {
    const real x0 = A.x + A.y, xn = A.x - A.y;
    const real y0 = x0 * Hk, yn = xn * Hnk;
    A = MK_C(0.5 * (y0 + yn), 0.5 * (y0 - yn));
    B = A;
    return;
  }
  const cplx Bc = cconj(B);
  const cplx E = cscale(cadd(A, Bc), 0.5);
  const cplx D = csub(A, Bc);
  const cplx O = MK_C(0.5 * D.y, -0.5 * D.x);  // -i/2 (A - conj B)
  const cplx WO = cmul(W, O);
  const cplx Xk = cadd(E, WO);
  const cplx Xnk = cconj(csub(E, WO));
  const cplx Yk = cscale(Xk, Hk);
  const cplx Ynk = cscale(Xnk, Hnk);
  // re-pack: Z'[k] = 1/2 (Yk + conj Ynk) + i/2 (Yk - conj Ynk) conj(W^k)
  const cplx Wc = cconj(W);
  const cplx e1 = cscale(cadd(Yk, cconj(Ynk)), 0.5);
  const cplx o1 = cmul(cscale(csub(Yk, cconj(Ynk)), 0.5), Wc);
  A = MK_C(e1.x - o1.y, e1.y + o1.x);
  // Z'[N-k] uses conj(W^{N-k}) = -W^k
  const cplx Wn = MK_C(-W.x, -W.y);
  const cplx e2 = cscale(cadd(Ynk, cconj(Yk)), 0.5);
  const cplx o2 = cmul(cscale(csub(Ynk, cconj(Yk)), 0.5), Wn);
  B = MK_C(e2.x - o2.y, e2.y + o2.x);
}

// ------------------------------------------------------ Stockham FFT --
// Batched radix-8 Stockham transforms for the four-step passes.  Pass p
// (sub-transform size Ns = 8^p) takes the eight elements j + k L/8 of a
// length-L transform into registers, multiplies element k by the twiddle
// w_L^{(j mod Ns) k L/(8 Ns)}, does an 8-point DFT in registers and writes
// element k to (j / Ns) 8 Ns + (j mod Ns) + k Ns: natural order in and out,
// no bit reversal.  A last radix-4 or radix-2 pass finishes lengths that are
// not powers of 8.  Every thread holds eight values per pass; shared-memory
// rows are padded one slot in nine (pad8) so that strided accesses spread
// over the banks.  The first pass may read from global memory and the last
// pass write to it through the load / store functors.
__device__ __forceinline__ int pad8(int i) { return i + (i >> 3); }

// twL[q] = exp(-2 pi i q / L), q < L: the sub-transform's twiddles, copied
// into shared memory by the kernel (load_twl) before its first transform
template <bool INV>
__device__ __forceinline__ cplx tw_l(const cplx *twL, int q) {
  const cplx w = twL[q];
  return INV ? cconj(w) : w;
}

__device__ __forceinline__ void load_twl(cplx *twL, int L, const cplx *tw) {
  for (int q = threadIdx.x; q < L; q += blockDim.x) twL[q] = tw[q];
}

// The twiddles of the radix-8 passes p >= 1 (sub-transform size Ns = 8^p)
// in the order the threads read them: ptw[off_p + (k - 1) Ns + r] =
// exp(-2 pi i r k L / (8 Ns) / L) for k = 1..7, r < Ns, so that consecutive
// threads (consecutive r) read consecutive entries with no bank conflicts.
// At most L - 8 entries; the values are those of tw.
__device__ __forceinline__ void load_pass_tw(cplx *ptw, int L, int logL, const cplx *tw) {
  const int n8 = logL / 3;
  int off = 0;
  for (int p = 1, Ns = 8; p < n8; ++p, Ns *= 8) {
    const int step = L / (8 * Ns);
    for (int e = threadIdx.x; e < 7 * Ns; e += blockDim.x) {
      const int k = e / Ns + 1, r = e % Ns;
      ptw[off + e] = tw[r * step * k];
    }
    off += 7 * Ns;
  }
}

template <bool INV>
__device__ __forceinline__ cplx mul_mi(cplx a) {  // a * (-i), inverse a * i
  return INV ? MK_C(-a.y, a.x) : MK_C(a.y, -a.x);
}

template <bool INV>
__device__ __forceinline__ cplx mul_w8(cplx a) {  // a * exp(-+ 2 pi i / 8)
  const real c = (real)0.70710678118654752440;
  return INV ? MK_C(c * (a.x - a.y), c * (a.x + a.y))
             : MK_C(c * (a.x + a.y), c * (a.y - a.x));
}

template <bool INV>
__device__ __forceinline__ cplx mul_w83(cplx a) {  // a * exp(-+ 6 pi i / 8)
  const real c = (real)0.70710678118654752440;
  return INV ? MK_C(-c * (a.x + a.y), c * (a.x - a.y))
             : MK_C(c * (a.y - a.x), -c * (a.x + a.y));
}

// 8-point DFT in registers, natural order in and out
template <bool INV>
__device__ __forceinline__ void dft8(cplx *v) {
  const cplx a0 = cadd(v[0], v[4]), b0 = csub(v[0], v[4]);
  const cplx a1 = cadd(v[1], v[5]), b1 = mul_w8<INV>(csub(v[1], v[5]));
  const cplx a2 = cadd(v[2], v[6]), b2 = mul_mi<INV>(csub(v[2], v[6]));
  const cplx a3 = cadd(v[3], v[7]), b3 = mul_w83<INV>(csub(v[3], v[7]));
  const cplx c0 = cadd(a0, a2), d0 = csub(a0, a2), c1 = cadd(a1, a3);
  const cplx d1 = mul_mi<INV>(csub(a1, a3));
  v[0] = cadd(c0, c1);
  v[4] = csub(c0, c1);
  v[2] = cadd(d0, d1);
  v[6] = csub(d0, d1);
  const cplx e0 = cadd(b0, b2), f0 = csub(b0, b2), e1 = cadd(b1, b3);
  const cplx f1 = mul_mi<INV>(csub(b1, b3));
  v[1] = cadd(e0, e1);
  v[5] = csub(e0, e1);
  v[3] = cadd(f0, f1);
  v[7] = csub(f0, f1);
}

template <bool INV>
__device__ __forceinline__ void dft4(cplx *v) {
  const cplx c0 = cadd(v[0], v[2]), d0 = csub(v[0], v[2]), c1 = cadd(v[1], v[3]);
  const cplx d1 = mul_mi<INV>(csub(v[1], v[3]));
  v[0] = cadd(c0, c1);
  v[2] = csub(c0, c1);
  v[1] = cadd(d0, d1);
  v[3] = csub(d0, d1);
}

// Last radix-R pass (R = 2 or 4, Ns = L / R): butterflies j < L / R over the
// elements j + k L / R; each thread takes 8 / R butterflies.
template <int R, bool INV, bool FFAST, typename Store>
__device__ __forceinline__ void last_pass(cplx *s, int S, int L, int nfft, const cplx *twL,
                                          int nb8, Store store) {
  constexpr int PER = 8 / R;
  const int Lr = L / R, t = threadIdx.x;
  cplx v[PER][R];
  int ff[PER], jj[PER];
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int q = t + u * nb8;
    ff[u] = -1;
    jj[u] = 0;
    if (q < nfft * Lr) {
      ff[u] = FFAST ? q % nfft : q / Lr;
      jj[u] = FFAST ? q / nfft : q % Lr;
#pragma unroll
      for (int k = 0; k < R; ++k) v[u][k] = s[ff[u] * S + pad8(jj[u] + k * Lr)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    if (ff[u] < 0) continue;
#pragma unroll
    for (int k = 1; k < R; ++k) v[u][k] = cmul(v[u][k], tw_l<INV>(twL, jj[u] * k));
    if (R == 4) {
      dft4<INV>(v[u]);
    } else {
      const cplx a = v[u][0], b = v[u][1];
      v[u][0] = cadd(a, b);
      v[u][1] = csub(a, b);
    }
#pragma unroll
    for (int k = 0; k < R; ++k) store(ff[u], jj[u] + k * Lr, v[u][k]);
  }
  __syncthreads();
}

// nfft transforms of length L (>= 64) at s + f * S; blockDim.x >= nfft L / 8.
// FFAST: consecutive threads take consecutive transforms f (else consecutive
// j).  load(f, i) gives input element i of transform f for the first pass;
// store(f, i, v) takes output element i of the last pass.
template <bool INV, bool FFAST, typename Load, typename Store>
__device__ __forceinline__ void fft_block(cplx *s, int S, int L, int logL, int nfft,
                                          const cplx *twL, const cplx *ptw, Load load,
                                          Store store) {
  const int L8 = L >> 3, n8 = logL / 3, rem = logL - 3 * n8;
  const int nb8 = nfft * L8;
  const int t = threadIdx.x;
  int Ns = 1, poff = 0;
  for (int pass = 0; pass < n8; ++pass) {
    const bool first = pass == 0, last = pass == n8 - 1 && rem == 0;
    const bool act = t < nb8;
    const int f = FFAST ? t % nfft : t / L8;
    const int j = FFAST ? t / nfft : t % L8;
    cplx v[8];
    if (act) {
#pragma unroll
      for (int k = 0; k < 8; ++k)
        v[k] = first ? load(f, j + k * L8) : s[f * S + pad8(j + k * L8)];
    }
    __syncthreads();
    if (act) {
      if (!first) {
        const cplx *pt = ptw + poff + (j & (Ns - 1));
#pragma unroll
        for (int k = 1; k < 8; ++k) {
          const cplx w = pt[(k - 1) * Ns];
          v[k] = cmul(v[k], INV ? cconj(w) : w);
        }
      }
      dft8<INV>(v);
      if (last) {
#pragma unroll
        for (int k = 0; k < 8; ++k) store(f, j + k * L8, v[k]);
      } else {
        const int base = (j / Ns) * Ns * 8 + (j & (Ns - 1));
#pragma unroll
        for (int k = 0; k < 8; ++k) s[f * S + pad8(base + k * Ns)] = v[k];
      }
    }
    __syncthreads();
    if (pass > 0) poff += 7 * Ns;
    Ns *= 8;
  }
  if (rem == 1) last_pass<2, INV, FFAST>(s, S, L, nfft, twL, nb8, store);
  else if (rem == 2) last_pass<4, INV, FFAST>(s, S, L, nfft, twL, nb8, store);
}

// ------------------------------------------------------- four-step path --
// Pass 1: forward column FFTs (length R) of G adjacent columns, twiddled.
__global__ void __launch_bounds__(512, 2) k_conv_cols_fwd(const ConvSeg *segs, const double *x,
                                                       const double *part, cplx *work, int R,
                                                       int logR, int C, int G,
                                                       const cplx *__restrict__ twrow,
                                                       const cplx *__restrict__ twr) {
  extern __shared__ __align__(16) unsigned char smraw[];
  cplx *sm = (cplx *)smraw;
  const int S = pad8(R) + 1;
  cplx *twL = sm + G * S, *ptw = twL + R;
  load_twl(twL, R, twr);
  load_pass_tw(ptw, R, logR, twr);
  const int seg = blockIdx.y;
  const ConvSeg sg = segs[seg];
  const double mean = seg_mean(part, seg, sg.n_in, sg.flags & 1);
  const int c0 = blockIdx.x * G;
  const long long N = (long long)R * C;
  cplx *W = work + (long long)seg * N;
  auto load = [&](int f, int n1) {
    const long long m = (long long)C * n1 + c0 + f;
    return MK_C(seg_input(x, sg, 2 * m, mean), seg_input(x, sg, 2 * m + 1, mean));
  };
  auto store = [&](int f, int k1, cplx v) {
    const long long i = (long long)k1 * C + c0 + f;
    W[i] = cmul(v, twrow[i]);
  };
  fft_block<false, true>(sm, S, R, logR, G, twL, ptw, load, store);
}

// Pass 2: forward row FFTs of rows k1 and R-k1, spectral product, inverse
// row FFTs, inverse twiddles.  Hrows holds the spectra in rows of the split
// (Hr[k1][k2] = H[k1 + R k2]); the Nyquist value H[N] comes from spectra.
__global__ void __launch_bounds__(1024) k_conv_rows(const ConvSeg *segs,
                                                    const real *__restrict__ Hrows,
                                                    const double *__restrict__ spectra,
                                                    long long spec_len, cplx *work, int R,
                                                    int C, int logC,
                                                    const cplx *__restrict__ twrow,
                                                    const cplx *__restrict__ wrow,
                                                    const cplx *__restrict__ twc) {
  extern __shared__ __align__(16) unsigned char smraw[];
  cplx *sm = (cplx *)smraw;
  const int S = pad8(C) + 1;
  cplx *s = sm;  // 2 rows
  cplx *twL = sm + 2 * S, *ptw = twL + C;
  load_twl(twL, C, twc);
  load_pass_tw(ptw, C, logC, twc);
  const int seg = blockIdx.y;
  const ConvSeg sg = segs[seg];
  const long long N = (long long)R * C;
  cplx *W = work + (long long)seg * N;
  const int j = blockIdx.x;            // 0 .. R/2
  const int ka = j, kb = (R - j) % R;  // row pair (equal for j = 0, R/2)
  const int nrows = (ka == kb) ? 1 : 2;
  auto gload = [&](int f, int n2) { return W[(long long)(f ? kb : ka) * C + n2]; };
  auto sload = [&](int f, int n2) { return s[f * S + pad8(n2)]; };
  auto sstore = [&](int f, int n2, cplx v) { s[f * S + pad8(n2)] = v; };
  fft_block<false, false>(s, S, C, logC, nrows, twL, ptw, gload, sstore);
  const real *Hr = Hrows + (long long)sg.spec * N;
  const real *Ha = Hr + (long long)ka * C, *Hb = Hr + (long long)kb * C;
  const cplx *Wa = wrow + (long long)ka * C;
  auto at = [&](int f, int n2) -> cplx & { return s[f * S + pad8(n2)]; };
  if (ka == 0) {
    // row 0: (0, k2) <-> (0, C - k2); k = R k2, N - k = R (C - k2)
    for (int k2 = threadIdx.x; k2 <= C / 2; k2 += blockDim.x) {
      const int p2 = (C - k2) % C;
      cplx A = at(0, k2), B = at(0, p2);
      const real Hnk = k2 ? Ha[C - k2] : (real)spectra[(long long)sg.spec * spec_len + N];
      spectral_pair(A, B, k2 == 0, Wa[k2], Ha[k2], Hnk);
      at(0, k2) = A;
      if (p2 != k2) at(0, p2) = B;
    }
  } else if (ka == kb) {
    // row R/2: (R/2, k2) <-> (R/2, C - 1 - k2)
    for (int k2 = threadIdx.x; k2 < C / 2; k2 += blockDim.x) {
      const int p2 = C - 1 - k2;
      cplx A = at(0, k2), B = at(0, p2);
      spectral_pair(A, B, false, Wa[k2], Ha[k2], Ha[p2]);
      at(0, k2) = A;
      at(0, p2) = B;
    }
  } else {
    // rows ka, kb = R - ka: (ka, k2) <-> (kb, C - 1 - k2)
    for (int k2 = threadIdx.x; k2 < C; k2 += blockDim.x) {
      const int p2 = C - 1 - k2;
      cplx A = at(0, k2), B = at(1, p2);
      spectral_pair(A, B, false, Wa[k2], Ha[k2], Hb[p2]);
      at(0, k2) = A;
      at(1, p2) = B;
    }
  }
  __syncthreads();
  auto gstore = [&](int f, int n2, cplx v) {
    const long long i = (long long)(f ? kb : ka) * C + n2;
    W[i] = cmul(v, cconj(twrow[i]));
  };
  fft_block<true, false>(s, S, C, logC, nrows, twL, ptw, sload, gstore);
}

// Pass 3: inverse column FFTs and real output.
__global__ void __launch_bounds__(512, 2) k_conv_cols_inv(const ConvSeg *segs, const cplx *work,
                                                       double *y, int R, int logR, int C, int G,
                                                       const cplx *__restrict__ twr) {
  extern __shared__ __align__(16) unsigned char smraw[];
  cplx *sm = (cplx *)smraw;
  const int S = pad8(R) + 1;
  cplx *twL = sm + G * S, *ptw = twL + R;
  load_twl(twL, R, twr);
  load_pass_tw(ptw, R, logR, twr);
  const int seg = blockIdx.y;
  const ConvSeg sg = segs[seg];
  const int c0 = blockIdx.x * G;
  const long long N = (long long)R * C;
  const cplx *W = work + (long long)seg * N;
  const double scale = 1.0 / (double)N;
  auto load = [&](int f, int k1) { return W[(long long)k1 * C + c0 + f]; };
  auto store = [&](int f, int n1, cplx v) {
    const long long m = (long long)C * n1 + c0 + f;
    if (2 * m < sg.n_out) y[sg.y_off + 2 * m] = v.x * scale;
    if (2 * m + 1 < sg.n_out) y[sg.y_off + 2 * m + 1] = v.y * scale;
  };
  fft_block<true, true>(sm, S, R, logR, G, twL, ptw, load, store);
}

#undef MK_C

}  // namespace FFT_NS
