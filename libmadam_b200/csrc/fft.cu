// Batched real-FFT convolution for sm_100a (see fft.cuh).
//
// A real vector of length nof is packed into N = nof/2 complex values
// z[m] = x[2m] + i x[2m+1]; the complex transform is split N = R x C
// (four-step: length-R column FFTs, twiddles w_N^{n2 k1}, length-C row
// FFTs).  The spectrum is never transposed: the row pass holds rows k1 and
// R-k1 together, which contain every conjugate pair (k, N-k) of the real
// transform, so the real-spectrum split, the multiplication by H and the
// re-packing for the inverse happen in shared memory between the forward and
// the inverse row FFTs.  The inverse column pass then writes the real output.
// Shared-memory FFTs are radix-2: decimation in time (bit-reversed load) for
// the forward transforms and decimation in frequency (bit-reversed store) for
// the inverse ones, so no separate permutation pass is needed.
#include "engine.h"
#include "fft.cuh"

namespace madam {
namespace {

typedef double2 cplx;

__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ cplx cconj(cplx a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ cplx cscale(cplx a, double s) { return make_double2(a.x * s, a.y * s); }

// exp(-2 pi i num / den) computed with sincospi for full double accuracy
__device__ __forceinline__ cplx twiddle(long long num, long long den) {
  long long r = num % den;
  double s, c;
  sincospi(-2.0 * (double)r / (double)den, &s, &c);
  return make_double2(c, s);
}

// T2[m] = exp(-2 pi i m / (2N)), m < 2N, precomputed once per plan; N is a
// power of two
__device__ __forceinline__ cplx tw_n(const cplx *T2, long long num, long long N) {
  return T2[2 * (num & (N - 1))];
}

__global__ void k_fill_table(cplx *T2, long long n2) {
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < n2;
       m += (long long)gridDim.x * blockDim.x)
    T2[m] = twiddle(m, n2);
}

__device__ __forceinline__ unsigned bitrev(unsigned v, int bits) {
  return __brev(v) >> (32 - bits);
}

// table[j] = exp(-2 pi i j / L), j < L/2, from the plan table of length 2N
__device__ void fill_twiddles(cplx *table, int L, const cplx *T2, long long N) {
  const long long step = 2 * N / L;
  for (int j = threadIdx.x; j < L / 2; j += blockDim.x) table[j] = T2[j * step];
}

// nfft independent length-L transforms stored contiguously in s (s[f*L + i]),
// input in bit-reversed order, output natural order; sign -1 forward.
// Two radix-2 stages (spans h and 2h) are done per round in registers on the
// four elements i, i+h, i+2h, i+3h; a single radix-2 stage finishes odd
// lengths.
__device__ void fft_dit(cplx *s, int L, int nfft, const cplx *tw, bool inverse) {
  int h = 1;
  for (; 4 * h <= L; h *= 4) {
    const int quarter = L / 4, total = nfft * quarter;
    const int st1 = L / (2 * h), st2 = L / (4 * h);
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int f = b / quarter, j = b - f * quarter;
      const int g = j / h, pos = j - g * h;
      const int i0 = f * L + g * 4 * h + pos;
      cplx w1 = tw[pos * st1], w2 = tw[pos * st2], w3 = tw[(pos + h) * st2];
      if (inverse) {
        w1 = cconj(w1);
        w2 = cconj(w2);
        w3 = cconj(w3);
      }
      cplx a0 = s[i0], a1 = s[i0 + h], a2 = s[i0 + 2 * h], a3 = s[i0 + 3 * h];
      cplx t = cmul(a1, w1);
      a1 = csub(a0, t);
      a0 = cadd(a0, t);
      t = cmul(a3, w1);
      a3 = csub(a2, t);
      a2 = cadd(a2, t);
      t = cmul(a2, w2);
      s[i0 + 2 * h] = csub(a0, t);
      s[i0] = cadd(a0, t);
      t = cmul(a3, w3);
      s[i0 + 3 * h] = csub(a1, t);
      s[i0 + h] = cadd(a1, t);
    }
    __syncthreads();
  }
  if (h < L) {  // last radix-2 stage, span h = L/2
    const int half = h, total = nfft * (L / 2), stride = L / (2 * h);
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int f = b / (L / 2), j = b - f * (L / 2);
      const int i0 = f * L + j, i1 = i0 + half;
      cplx w = tw[j * stride];
      if (inverse) w = cconj(w);
      const cplx t = cmul(s[i1], w), u = s[i0];
      s[i0] = cadd(u, t);
      s[i1] = csub(u, t);
    }
    __syncthreads();
  }
}

// natural-order input, bit-reversed output (decimation in frequency); stages
// with spans 2h then h are fused per round
__device__ void fft_dif(cplx *s, int L, int nfft, const cplx *tw, bool inverse) {
  int lg = 0;
  while ((1 << lg) < L) ++lg;
  int h;
  if (lg & 1) {  // first radix-2 stage, span L/2
    const int half = L / 2, total = nfft * half;
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int f = b / half, j = b - f * half;
      const int i0 = f * L + j, i1 = i0 + half;
      cplx w = tw[j];
      if (inverse) w = cconj(w);
      const cplx u = s[i0], v = s[i1];
      s[i0] = cadd(u, v);
      s[i1] = cmul(csub(u, v), w);
    }
    __syncthreads();
    h = L / 8;
  } else {
    h = L / 4;
  }
  for (; h >= 1; h /= 4) {
    const int quarter = L / 4, total = nfft * quarter;
    const int st1 = L / (2 * h), st2 = L / (4 * h);
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      const int f = b / quarter, j = b - f * quarter;
      const int g = j / h, pos = j - g * h;
      const int i0 = f * L + g * 4 * h + pos;
      cplx w1 = tw[pos * st1], w2 = tw[pos * st2], w3 = tw[(pos + h) * st2];
      if (inverse) {
        w1 = cconj(w1);
        w2 = cconj(w2);
        w3 = cconj(w3);
      }
      cplx a0 = s[i0], a1 = s[i0 + h], a2 = s[i0 + 2 * h], a3 = s[i0 + 3 * h];
      // span 2h: (a0, a2) with w2, (a1, a3) with w3
      cplx u = a0, v = a2;
      a0 = cadd(u, v);
      a2 = cmul(csub(u, v), w2);
      u = a1;
      v = a3;
      a1 = cadd(u, v);
      a3 = cmul(csub(u, v), w3);
      // span h: (a0, a1) and (a2, a3) with w1
      s[i0] = cadd(a0, a1);
      s[i0 + h] = cmul(csub(a0, a1), w1);
      s[i0 + 2 * h] = cadd(a2, a3);
      s[i0 + 3 * h] = cmul(csub(a2, a3), w1);
    }
    __syncthreads();
  }
}

// Real-spectrum split of the packed transform for the pair (k, N-k), product
// with the real spectrum H and re-packing for the inverse transform.
// A = Z[k], B = Z[N-k], W = exp(-i pi k / N), Hk = H[k], Hnk = H[N-k]; on
// return A = Z'[k], B = Z'[N-k].  dc (k == 0) handles the DC / Nyquist pair
// with Hk = H[0], Hnk = H[N] (B is ignored and set equal to A).
__device__ __forceinline__ void spectral_pair(cplx &A, cplx &B, bool dc, cplx W, double Hk,
                                              double Hnk) {
  if (dc) {
    const double x0 = A.x + A.y, xn = A.x - A.y;
    const double y0 = x0 * Hk, yn = xn * Hnk;
    A = make_double2(0.5 * (y0 + yn), 0.5 * (y0 - yn));
    B = A;
    return;
  }
  const cplx Bc = cconj(B);
  const cplx E = cscale(cadd(A, Bc), 0.5);
  const cplx D = csub(A, Bc);
  const cplx O = make_double2(0.5 * D.y, -0.5 * D.x);  // -i/2 (A - conj B)
  const cplx WO = cmul(W, O);
  const cplx Xk = cadd(E, WO);
  const cplx Xnk = cconj(csub(E, WO));
  const cplx Yk = cscale(Xk, Hk);
  const cplx Ynk = cscale(Xnk, Hnk);
  // re-pack: Z'[k] = 1/2 (Yk + conj Ynk) + i/2 (Yk - conj Ynk) conj(W^k)
  const cplx Wc = cconj(W);
  const cplx e1 = cscale(cadd(Yk, cconj(Ynk)), 0.5);
  const cplx o1 = cmul(cscale(csub(Yk, cconj(Ynk)), 0.5), Wc);
  A = make_double2(e1.x - o1.y, e1.y + o1.x);
  // Z'[N-k] uses conj(W^{N-k}) = -W^k
  const cplx Wn = make_double2(-W.x, -W.y);
  const cplx e2 = cscale(cadd(Ynk, cconj(Yk)), 0.5);
  const cplx o2 = cmul(cscale(csub(Ynk, cconj(Yk)), 0.5), Wn);
  B = make_double2(e2.x - o2.y, e2.y + o2.x);
}

__device__ __forceinline__ double seg_input(const double *x, const ConvSeg &sg, long long i,
                                            double mean) {
  return i < sg.n_in ? x[sg.x_off + i] - mean : 0.0;
}

// ---------------------------------------------------------------- means --
// Segment sums in two stages: kMeanBlocks CTAs per segment write partial sums;
// consumers add the partials of their segment.
constexpr int kMeanBlocks = 32;

__global__ void k_seg_sum(const ConvSeg *segs, const double *v, int out, double *part) {
  const ConvSeg sg = segs[blockIdx.y];
  const bool on = out ? (sg.flags & 2) : (sg.flags & 1);
  const long long n = out ? sg.n_out : sg.n_in;
  const long long off = out ? sg.y_off : sg.x_off;
  double acc[1] = {0.0};
  if (on) {
    const long long a = n * blockIdx.x / gridDim.x, e = n * (blockIdx.x + 1) / gridDim.x;
    for (long long i = a + threadIdx.x; i < e; i += blockDim.x) acc[0] += v[off + i];
  }
  block_sum<1>(acc);
  if (threadIdx.x == 0) part[(long long)blockIdx.y * gridDim.x + blockIdx.x] = acc[0];
}

__device__ __forceinline__ double seg_mean(const double *part, int seg, long long n, bool on) {
  if (!on || n == 0) return 0.0;
  double s = 0;
  for (int b = 0; b < kMeanBlocks; ++b) s += part[(long long)seg * kMeanBlocks + b];
  return s / (double)n;
}

__global__ void k_seg_sub_mean(const ConvSeg *segs, double *y, const double *part) {
  const ConvSeg sg = segs[blockIdx.y];
  if (!(sg.flags & 2)) return;
  const double m = seg_mean(part, blockIdx.y, sg.n_out, true);
  const long long n = sg.n_out;
  const long long a = n * blockIdx.x / gridDim.x, e = n * (blockIdx.x + 1) / gridDim.x;
  for (long long i = a + threadIdx.x; i < e; i += blockDim.x) y[sg.y_off + i] -= m;
}

// ------------------------------------------------------ single-CTA path --
// One CTA per segment; N complex values in shared memory.
__global__ void k_conv_small(const ConvSeg *segs, const double *spectra, long long spec_len,
                             const double *x, double *y, const double *part, int N, int logN,
                             const cplx *T2) {
  extern __shared__ double2 sm[];
  cplx *s = sm;
  cplx *tw = sm + N;
  const ConvSeg sg = segs[blockIdx.x];
  const double mean = seg_mean(part, blockIdx.x, sg.n_in, sg.flags & 1);
  fill_twiddles(tw, N, T2, N);
  for (int m = threadIdx.x; m < N; m += blockDim.x) {
    const double a = seg_input(x, sg, 2LL * m, mean);
    const double b = seg_input(x, sg, 2LL * m + 1, mean);
    s[bitrev(m, logN)] = make_double2(a, b);
  }
  __syncthreads();
  fft_dit(s, N, 1, tw, false);
  const double *H = spectra + (long long)sg.spec * spec_len;
  for (int k = threadIdx.x; k <= N / 2; k += blockDim.x) {
    const int nk = (N - k) % N;
    cplx A = s[k], B = s[nk];
    spectral_pair(A, B, k == 0, T2[k], H[k], H[N - k]);
    s[k] = A;
    if (nk != k) s[nk] = B;
  }
  __syncthreads();
  fft_dif(s, N, 1, tw, true);
  const double scale = 1.0 / (double)N;  // 1/nof times the factor 2 of the packing
  for (int m = threadIdx.x; m < N; m += blockDim.x) {
    const cplx v = s[bitrev(m, logN)];
    const long long i0 = 2LL * m;
    if (i0 < sg.n_out) y[sg.y_off + i0] = v.x * scale;
    if (i0 + 1 < sg.n_out) y[sg.y_off + i0 + 1] = v.y * scale;
  }
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
  return INV ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

template <bool INV>
__device__ __forceinline__ cplx mul_w8(cplx a) {  // a * exp(-+ 2 pi i / 8)
  const double c = 0.70710678118654752440;
  return INV ? make_double2(c * (a.x - a.y), c * (a.x + a.y))
             : make_double2(c * (a.x + a.y), c * (a.y - a.x));
}

template <bool INV>
__device__ __forceinline__ cplx mul_w83(cplx a) {  // a * exp(-+ 6 pi i / 8)
  const double c = 0.70710678118654752440;
  return INV ? make_double2(-c * (a.x + a.y), c * (a.x - a.y))
             : make_double2(c * (a.y - a.x), -c * (a.x + a.y));
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
                                                       const double *part, double2 *work, int R,
                                                       int logR, int C, int G,
                                                       const cplx *__restrict__ twrow,
                                                       const cplx *__restrict__ twr) {
  extern __shared__ double2 sm[];
  const int S = pad8(R) + 1;
  cplx *twL = sm + G * S, *ptw = twL + R;
  load_twl(twL, R, twr);
  load_pass_tw(ptw, R, logR, twr);
  const int seg = blockIdx.y;
  const ConvSeg sg = segs[seg];
  const double mean = seg_mean(part, seg, sg.n_in, sg.flags & 1);
  const int c0 = blockIdx.x * G;
  const long long N = (long long)R * C;
  double2 *W = work + (long long)seg * N;
  auto load = [&](int f, int n1) {
    const long long m = (long long)C * n1 + c0 + f;
    return make_double2(seg_input(x, sg, 2 * m, mean), seg_input(x, sg, 2 * m + 1, mean));
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
                                                    const double *__restrict__ Hrows,
                                                    const double *__restrict__ spectra,
                                                    long long spec_len, double2 *work, int R,
                                                    int C, int logC,
                                                    const cplx *__restrict__ twrow,
                                                    const cplx *__restrict__ wrow,
                                                    const cplx *__restrict__ twc) {
  extern __shared__ double2 sm[];
  const int S = pad8(C) + 1;
  cplx *s = sm;  // 2 rows
  cplx *twL = sm + 2 * S, *ptw = twL + C;
  load_twl(twL, C, twc);
  load_pass_tw(ptw, C, logC, twc);
  const int seg = blockIdx.y;
  const ConvSeg sg = segs[seg];
  const long long N = (long long)R * C;
  double2 *W = work + (long long)seg * N;
  const int j = blockIdx.x;            // 0 .. R/2
  const int ka = j, kb = (R - j) % R;  // row pair (equal for j = 0, R/2)
  const int nrows = (ka == kb) ? 1 : 2;
  auto gload = [&](int f, int n2) { return W[(long long)(f ? kb : ka) * C + n2]; };
  auto sload = [&](int f, int n2) { return s[f * S + pad8(n2)]; };
  auto sstore = [&](int f, int n2, cplx v) { s[f * S + pad8(n2)] = v; };
  fft_block<false, false>(s, S, C, logC, nrows, twL, ptw, gload, sstore);
  const double *Hr = Hrows + (long long)sg.spec * N;
  const double *Ha = Hr + (long long)ka * C, *Hb = Hr + (long long)kb * C;
  const cplx *Wa = wrow + (long long)ka * C;
  auto at = [&](int f, int n2) -> cplx & { return s[f * S + pad8(n2)]; };
  if (ka == 0) {
    // row 0: (0, k2) <-> (0, C - k2); k = R k2, N - k = R (C - k2)
    for (int k2 = threadIdx.x; k2 <= C / 2; k2 += blockDim.x) {
      const int p2 = (C - k2) % C;
      cplx A = at(0, k2), B = at(0, p2);
      const double Hnk = k2 ? Ha[C - k2] : spectra[(long long)sg.spec * spec_len + N];
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
__global__ void __launch_bounds__(512, 2) k_conv_cols_inv(const ConvSeg *segs, const double2 *work,
                                                       double *y, int R, int logR, int C, int G,
                                                       const cplx *__restrict__ twr) {
  extern __shared__ double2 sm[];
  const int S = pad8(R) + 1;
  cplx *twL = sm + G * S, *ptw = twL + R;
  load_twl(twL, R, twr);
  load_pass_tw(ptw, R, logR, twr);
  const int seg = blockIdx.y;
  const ConvSeg sg = segs[seg];
  const int c0 = blockIdx.x * G;
  const long long N = (long long)R * C;
  const double2 *W = work + (long long)seg * N;
  const double scale = 1.0 / (double)N;
  auto load = [&](int f, int k1) { return W[(long long)k1 * C + c0 + f]; };
  auto store = [&](int f, int n1, cplx v) {
    const long long m = (long long)C * n1 + c0 + f;
    if (2 * m < sg.n_out) y[sg.y_off + 2 * m] = v.x * scale;
    if (2 * m + 1 < sg.n_out) y[sg.y_off + 2 * m + 1] = v.y * scale;
  };
  fft_block<true, true>(sm, S, R, logR, G, twL, ptw, load, store);
}

// The row-ordered tables of the four-step split (FFTPlan), from T2.
__global__ void k_fill_row_tables(const cplx *T2, long long N, int R, int C, cplx *twrow,
                                  cplx *wrow, cplx *twr, cplx *twc) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k1 = i / C, n2 = i % C;
    twrow[i] = tw_n(T2, n2 * k1, N);
    wrow[i] = T2[k1 + (long long)R * n2];
    if (i < R) twr[i] = T2[i * (2 * N / R)];
    if (i < C) twc[i] = T2[i * (2 * N / C)];
  }
}

// rows[s][k1][k2] = H[s][k1 + R k2]: the transpose of each spectrum viewed
// as a C x R matrix, through 32 x 32 shared-memory tiles
__global__ void k_spectra_rows(const double *H, long long spec_len, int R, int C, double *rows) {
  __shared__ double t[32][33];
  const int s = blockIdx.z;
  const double *h = H + (long long)s * spec_len;
  double *o = rows + (long long)s * R * C;
  const int k1b = blockIdx.x * 32, k2b = blockIdx.y * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y)
    t[y][threadIdx.x] = h[(long long)(k2b + y) * R + k1b + threadIdx.x];
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y)
    o[(long long)(k1b + y) * C + k2b + threadIdx.x] = t[threadIdx.x][y];
}

int ilog2(long v) {
  int l = 0;
  while ((1L << l) < v) ++l;
  return l;
}

}  // namespace

FFTPlan::FFTPlan(long nof_) : nof(nof_), N(nof_ / 2) {
  if (nof < 4 || (nof & (nof - 1))) fail("FFT length must be a power of two >= 4");
  if (N > (1L << 24)) fail("FFT length too large");
  if (N > 2048) {
    int l = ilog2(N);
    R = 1 << (l / 2);
    C = (int)(N / R);
    G = std::max(1, std::min(16, 4096 / R));
    if (G > C) G = C;
  }
  // column passes: G transforms of length R, G R / 8 threads; row pass: two
  // rows of length C, C / 4 threads
}

FFTPlan::~FFTPlan() {
  forget_spectra();
  for (double *p : {table, work, means, twrow, wrow, twr, twc})
    if (p) dev_free(p);
}

void FFTPlan::forget_spectra() {
  for (RowSpectra &c : cache) {
    if (c.rows) dev_free(c.rows);
    c = RowSpectra{};
  }
}

void FFTPlan::make_tables(cudaStream_t st) {
  if (twrow || !R) return;
  twrow = (double *)dev_alloc((size_t)N * sizeof(double2));
  wrow = (double *)dev_alloc((size_t)N * sizeof(double2));
  twr = (double *)dev_alloc((size_t)R * sizeof(double2));
  twc = (double *)dev_alloc((size_t)C * sizeof(double2));
  MADAM_LAUNCH(k_fill_row_tables, (unsigned)std::min<long long>(4096, (N + 255) / 256), 256, 0,
               st, (const cplx *)table, (long long)N, R, C, (cplx *)twrow, (cplx *)wrow,
               (cplx *)twr, (cplx *)twc);
}

const double *FFTPlan::row_spectra(cudaStream_t st, const double *spectra, long nspec) {
  for (const RowSpectra &c : cache)
    if (c.rows && c.src == spectra && c.nspec == nspec) return c.rows;
  // a free slot, else the first one is dropped
  RowSpectra *slot = &cache[0];
  for (RowSpectra &c : cache)
    if (!c.rows) {
      slot = &c;
      break;
    }
  if (slot->rows) dev_free(slot->rows);
  slot->src = spectra;
  slot->nspec = nspec;
  slot->rows = (double *)dev_alloc((size_t)std::max<long>(1, nspec) * N * sizeof(double));
  if (nspec > 0) {
    if (nspec > 65535) fail("too many filter spectra");
    MADAM_LAUNCH(k_spectra_rows, dim3(R / 32, C / 32, (unsigned)nspec), dim3(32, 8), 0, st,
                 spectra, (long long)N + 1, R, C, slot->rows);
  }
  return slot->rows;
}

void FFTPlan::reserve(long nseg) {
  if (nseg <= nseg_max) return;
  if (work) dev_free(work);
  if (means) dev_free(means);
  work = nullptr;
  means = nullptr;
  if (R) work = (double *)dev_alloc((size_t)nseg * N * sizeof(double2));
  means = (double *)dev_alloc((size_t)nseg * kMeanBlocks * sizeof(double));
  nseg_max = nseg;
}

void FFTPlan::convolve(cudaStream_t st, const ConvSeg *segs, long nseg, const double *spectra,
                       long nspec, const double *x, double *y) {
  if (nseg == 0) return;
  if (!table) {
    table = (double *)dev_alloc((size_t)2 * N * sizeof(double2));
    MADAM_LAUNCH(k_fill_table, (unsigned)std::min<long long>(4096, (2 * N + 255) / 256), 256, 0,
                 st, (double2 *)table, 2LL * N);
  }
  const cplx *T2 = (const cplx *)table;
  if (nseg > 65535) fail("too many filter segments in one batch");
  reserve(nseg);
  const long long spec_len = N + 1;
  const dim3 gm(kMeanBlocks, (unsigned)nseg);
  MADAM_LAUNCH(k_seg_sum, gm, 256, 0, st, segs, x, 0, means);
  if (R == 0) {
    const int logN = ilog2(N);
    size_t smem = (size_t)(N + N / 2) * sizeof(double2);
    static bool attr_small = false;
    if (!attr_small) {
      MADAM_CUDA(cudaFuncSetAttribute(k_conv_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      64 * 1024));
      attr_small = true;
    }
    MADAM_LAUNCH(k_conv_small, (unsigned)nseg, 256, smem, st, segs, spectra, spec_len, x, y,
                 means, (int)N, logN, T2);
  } else {
    const int logR = ilog2(R), logC = ilog2(C);
    auto padded = [](long L) { return L + L / 8 + 1; };
    // rows padded one slot in nine, then the sub-transform twiddle table and
    // the passes' twiddles (8^(log8 L) - 8 entries)
    auto passes = [](int logL) { return logL >= 6 ? (1L << (3 * (logL / 3))) - 8 : 0L; };
    size_t smem_cols = (size_t)(G * padded(R) + R + passes(logR)) * sizeof(double2);
    size_t smem_rows = (size_t)(2 * padded(C) + C + passes(logC)) * sizeof(double2);
    constexpr size_t kSmemMax = 227 * 1024;
    if (smem_cols > kSmemMax || smem_rows > kSmemMax)
      fail("FFT length too large for the four-step filter");
    const unsigned tcols = (unsigned)std::max(32, G * R / 8);
    const unsigned trows = (unsigned)std::max(32, C / 4);
    static bool attr = false;
    if (!attr) {
      MADAM_CUDA(cudaFuncSetAttribute(k_conv_cols_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kSmemMax));
      MADAM_CUDA(cudaFuncSetAttribute(k_conv_cols_inv, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kSmemMax));
      MADAM_CUDA(cudaFuncSetAttribute(k_conv_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kSmemMax));
      attr = true;
    }
    make_tables(st);
    const double *Hrows = row_spectra(st, spectra, nspec);
    dim3 gc(C / G, (unsigned)nseg), gr(R / 2 + 1, (unsigned)nseg);
    MADAM_LAUNCH(k_conv_cols_fwd, gc, tcols, smem_cols, st, segs, x, means, (double2 *)work, R,
                 logR, C, G, (const cplx *)twrow, (const cplx *)twr);
    MADAM_LAUNCH(k_conv_rows, gr, trows, smem_rows, st, segs, Hrows, spectra, spec_len,
                 (double2 *)work, R, C, logC, (const cplx *)twrow, (const cplx *)wrow,
                 (const cplx *)twc);
    MADAM_LAUNCH(k_conv_cols_inv, gc, tcols, smem_cols, st, segs, (const double2 *)work, y, R,
                 logR, C, G, (const cplx *)twr);
  }
  MADAM_LAUNCH(k_seg_sum, gm, 256, 0, st, segs, y, 1, means);
  MADAM_LAUNCH(k_seg_sub_mean, gm, 256, 0, st, segs, y, means);
}

}  // namespace madam
