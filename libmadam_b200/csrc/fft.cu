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
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

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
// (fft_steps.inl) the four-step passes in float64 and in float32
#define FFT_NS fs64
#define FFT_CPLX double2
#define FFT_REAL double
#define FFT_MK make_double2
#include "fft_steps.inl"
#undef FFT_NS
#undef FFT_CPLX
#undef FFT_REAL
#undef FFT_MK
#define FFT_NS fs32
#define FFT_CPLX float2
#define FFT_REAL float
#define FFT_MK make_float2
#include "fft_steps.inl"
#undef FFT_NS
#undef FFT_CPLX
#undef FFT_REAL
#undef FFT_MK

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

// float32 copies of tables (complex and real)
__global__ void k_d2f_c(const double2 *a, float2 *b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = make_float2((float)a[i].x, (float)a[i].y);
}
__global__ void k_d2f(const double *a, float *b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
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
  if (tw32) dev_free(tw32);
}

void FFTPlan::forget_spectra() {
  for (RowSpectra &c : cache) {
    if (c.rows) dev_free(c.rows);
    if (c.rows32) dev_free(c.rows32);
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
  tw32 = (float *)dev_alloc((size_t)(2 * N + R + C) * sizeof(float2));
  float2 *t = (float2 *)tw32;
  const unsigned g = (unsigned)std::min<long long>(4096, (N + 255) / 256);
  MADAM_LAUNCH(k_d2f_c, g, 256, 0, st, (const double2 *)twrow, t, (long long)N);
  MADAM_LAUNCH(k_d2f_c, g, 256, 0, st, (const double2 *)wrow, t + N, (long long)N);
  MADAM_LAUNCH(k_d2f_c, g, 256, 0, st, (const double2 *)twr, t + 2 * N, (long long)R);
  MADAM_LAUNCH(k_d2f_c, g, 256, 0, st, (const double2 *)twc, t + 2 * N + R, (long long)C);
}

FFTPlan::RowSpectra &FFTPlan::row_spectra(cudaStream_t st, const double *spectra, long nspec) {
  for (RowSpectra &c : cache)
    if (c.rows && c.src == spectra && c.nspec == nspec) return c;
  // a free slot, else the first one is dropped
  RowSpectra *slot = &cache[0];
  for (RowSpectra &c : cache)
    if (!c.rows) {
      slot = &c;
      break;
    }
  if (slot->rows) dev_free(slot->rows);
  if (slot->rows32) dev_free(slot->rows32);
  slot->rows32 = nullptr;
  slot->src = spectra;
  slot->nspec = nspec;
  slot->rows = (double *)dev_alloc((size_t)std::max<long>(1, nspec) * N * sizeof(double));
  if (nspec > 0) {
    if (nspec > 65535) fail("too many filter spectra");
    MADAM_LAUNCH(k_spectra_rows, dim3(R / 32, C / 32, (unsigned)nspec), dim3(32, 8), 0, st,
                 spectra, (long long)N + 1, R, C, slot->rows);
  }
  return *slot;
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
                       long nspec, const double *x, double *y, bool f32) {
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
      for (const void *k : {(const void *)fs64::k_conv_cols_fwd, (const void *)fs64::k_conv_cols_inv,
                            (const void *)fs64::k_conv_rows, (const void *)fs32::k_conv_cols_fwd,
                            (const void *)fs32::k_conv_cols_inv, (const void *)fs32::k_conv_rows})
        MADAM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kSmemMax));
      attr = true;
    }
    make_tables(st);
    RowSpectra &rs = row_spectra(st, spectra, nspec);
    dim3 gc(C / G, (unsigned)nseg), gr(R / 2 + 1, (unsigned)nseg);
    if (!f32) {
      MADAM_LAUNCH(fs64::k_conv_cols_fwd, gc, tcols, smem_cols, st, segs, x, means,
                   (double2 *)work, R, logR, C, G, (const double2 *)twrow, (const double2 *)twr);
      MADAM_LAUNCH(fs64::k_conv_rows, gr, trows, smem_rows, st, segs, rs.rows, spectra, spec_len,
                   (double2 *)work, R, C, logC, (const double2 *)twrow, (const double2 *)wrow,
                   (const double2 *)twc);
      MADAM_LAUNCH(fs64::k_conv_cols_inv, gc, tcols, smem_cols, st, segs, (const double2 *)work,
                   y, R, logR, C, G, (const double2 *)twr);
    } else {
      if (!rs.rows32) {
        const long long nr = (long long)std::max<long>(1, nspec) * N;
        rs.rows32 = (float *)dev_alloc((size_t)nr * sizeof(float));
        MADAM_LAUNCH(k_d2f, (unsigned)std::min<long long>(4096, (nr + 255) / 256), 256, 0, st,
                     rs.rows, rs.rows32, nr);
      }
      const float2 *t = (const float2 *)tw32;
      const float2 *trow = t, *wr = t + N, *tr = t + 2 * N, *tc = t + 2 * N + R;
      // float2 elements: half the shared memory of the float64 passes
      MADAM_LAUNCH(fs32::k_conv_cols_fwd, gc, tcols, smem_cols / 2, st, segs, x, means,
                   (float2 *)work, R, logR, C, G, trow, tr);
      MADAM_LAUNCH(fs32::k_conv_rows, gr, trows, smem_rows / 2, st, segs, rs.rows32, spectra,
                   spec_len, (float2 *)work, R, C, logC, trow, wr, tc);
      MADAM_LAUNCH(fs32::k_conv_cols_inv, gc, tcols, smem_cols / 2, st, segs,
                   (const float2 *)work, y, R, logR, C, G, tr);
    }
  }
  MADAM_LAUNCH(k_seg_sum, gm, 256, 0, st, segs, y, 1, means);
  MADAM_LAUNCH(k_seg_sub_mean, gm, 256, 0, st, segs, y, means);
}

}  // namespace madam
