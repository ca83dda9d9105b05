// Deduplicated band Cholesky preconditioner with a chunk-parallel exact solve.
//
// construct_preconditioner (noise_routines.f90:1028-1120) factors
// A = Toeplitz(invcov[0:nband]) + diag(nna) per trimmed segment (DPBTRF 'L');
// preconditioning_band (1159-1256) solves L L^T z = r (DPBTRS).
//
// Factor.  Row j of L is R_j[d] = L(j, j-d), d = 0..w (w = nband - 1), and
// depends only on rows j-w..j-1 and on nna_j.  Computed left-looking, in the
// update order of DPBTF2 (m increasing), rows settle to a bitwise fixed point
// after ~100 rows wherever nna is constant; once w+1 consecutive rows are
// identical and nna_j == nna_{j-1} the next row is a copy, so it is not
// recomputed.  The factor is stored as a table of distinct rows plus a run
// list (first row, table entry).  Exact: every stored row is the row the
// column algorithm would produce for that input.
//
// Solve.  The forward recurrence y_j = (r_j - sum_d R_j[d] y_{j-d}) / R_j[0]
// is cut into chunks.  Pass 1 solves every chunk with a zero initial state;
// a warp per segment then propagates the true state across chunks with the
// w x w transfer matrices T_c (homogeneous response of the chunk's last w rows
// to its w initial values, precomputed, shared between chunks whose rows are
// one run); pass 2 re-solves every chunk from its true initial state.  The
// backward solve L^T x = y does the same from the end of the segment.
#include <algorithm>

#include "band2.cuh"
#include "engine.h"

namespace madam {
namespace {

constexpr int kRing = 128;  // >= w + 1

// One thread per segment.  urows: worst-case region of n * nb doubles at
// seg.row_off; runs: worst-case n entries at seg.run_off.
__global__ void k_band2_factor(const PSeg *segs, int nseg, const int *spec, const double *invcov,
                               long long nof, const double *nna, double *urows, PRun *runs,
                               int *status, int *nunique, int *nruns) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  const PSeg g = segs[s];
  const int nb = g.nb, w = nb - 1;
  const double *ic = invcov + (long long)spec[s] * nof;
  const double *nn = nna + g.k0;
  double *rowbase = urows + g.row_off;
  PRun *rl = runs + g.run_off;
  // window of the last w rows (pointers into the unique table)
  const double *win[kRing];
  int nu = 0, nr = 0, same = 0;
  const double *prev = nullptr;
  for (int j = 0; j < g.n; ++j) {
    if (prev && same >= w + 1 && nn[j] == nn[j - 1]) {
      // steady state: row j equals row j-1
      win[j & (kRing - 1)] = prev;
      ++same;
      continue;
    }
    double *R = rowbase + (long long)nu * nb;
    for (int d = 0; d < nb; ++d) R[d] = 0.0;
    // off-diagonal entries, d = w..1 (k = j - d increasing)
    for (int d = min(w, j); d >= 1; --d) {
      const double *Rk = win[(j - d) & (kRing - 1)];
      double acc = ic[d];
      // subtract L(j, m) L(k, m) for m = j-w .. k-1 in increasing m
      for (int e = min(w, j); e > d; --e) acc -= R[e] * Rk[e - d];
      R[d] = acc * (1.0 / Rk[0]);
    }
    double dg = ic[0] + nn[j];
    for (int e = min(w, j); e >= 1; --e) dg -= R[e] * R[e];
    if (!(dg > 0)) {
      status[s] = j + 1;
      nunique[s] = 0;
      nruns[s] = 0;
      return;
    }
    R[0] = sqrt(dg);
    bool eq = prev != nullptr;
    if (eq)
      for (int d = 0; d < nb; ++d)
        if (R[d] != prev[d]) { eq = false; break; }
    if (eq) {
      win[j & (kRing - 1)] = prev;
      ++same;
    } else {
      rl[nr].start = j;
      rl[nr].row_off = g.row_off + (long long)nu * nb;
      ++nr;
      ++nu;
      prev = R;
      win[j & (kRing - 1)] = R;
      same = 1;
    }
  }
  status[s] = 0;
  nunique[s] = nu;
  nruns[s] = nr;
}

// Forward solve of rows [a, b) of one segment.  state: y_{a-w..a-1} (or
// nullptr for zeros); writes y (if out) and the last w values (if tail).
__device__ void fwd_rows(const PSeg &g, const PRun *runs, const double *urows, int run,
                         int a, int b, const double *r, const double *state, double *out,
                         double *tail) {
  const int w = g.nb - 1;
  double ring[kRing];
  for (int i = 0; i < w; ++i) ring[(a - w + i) & (kRing - 1)] = state ? state[i] : 0.0;
  const int rend = g.run_off + g.nrun;
  int next = (run + 1 < rend) ? runs[run + 1].start : 0x7fffffff;
  const double *R = urows + runs[run].row_off;
  for (int j = a; j < b; ++j) {
    while (j >= next) {
      ++run;
      R = urows + runs[run].row_off;
      next = (run + 1 < rend) ? runs[run + 1].start : 0x7fffffff;
    }
    double acc = r ? r[g.k0 + j] : 0.0;
    for (int d = w; d >= 1; --d) acc -= R[d] * ring[(j - d) & (kRing - 1)];
    const double y = acc / R[0];
    ring[j & (kRing - 1)] = y;
    if (out) out[g.k0 + j] = y;
  }
  if (tail)
    for (int i = 0; i < w; ++i) tail[i] = (b - w + i >= a - w) ? ring[(b - w + i) & (kRing - 1)] : 0.0;
}

// Backward solve of rows [a, b) (descending).  state: x_{b..b+w-1} (zeros
// beyond the segment end, or nullptr); writes x (if out) and the first w
// values (if head).  run_hi: the run containing row min(b + w, n) - 1.
__device__ void bwd_rows(const PSeg &g, const PRun *runs, const double *urows, int run_hi,
                         int a, int b, const double *y, const double *state, double *out,
                         double *head) {
  const int w = g.nb - 1;
  double xr[kRing];
  const double *pr[kRing];
  int rr = run_hi;
  const int top = min(b + w, g.n) - 1;
  for (int q = top; q >= a; --q) {
    // row pointer of q
    while (q < runs[rr].start) --rr;
    pr[q & (kRing - 1)] = urows + runs[rr].row_off;
    if (q >= b) xr[q & (kRing - 1)] = state ? state[q - b] : 0.0;
    if (q < b) {
      const int j = q;
      double t = y ? y[g.k0 + j] : 0.0;
      const int dmax = min(w, g.n - 1 - j);
      for (int d = 1; d <= dmax; ++d) t -= pr[(j + d) & (kRing - 1)][d] * xr[(j + d) & (kRing - 1)];
      const double x = t / pr[j & (kRing - 1)][0];
      xr[j & (kRing - 1)] = x;
      if (out) out[g.k0 + j] = x;
    }
  }
  if (head)
    for (int i = 0; i < w; ++i) head[i] = (a + i < b) ? xr[(a + i) & (kRing - 1)] : 0.0;
}

__global__ void k_band2_fwd(const PSeg *segs, const PChunk *ch, int nch, const PRun *runs,
                            const double *urows, const double *r, const double *tstate,
                            double *out, double *tails) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nch) return;
  const PChunk k = ch[c];
  const PSeg g = segs[k.seg];
  const double *st = (tstate && k.first == 0) ? tstate + (long long)(c - 1) * kRing : nullptr;
  double *tl = (tails && k.last == 0) ? tails + (long long)c * kRing : nullptr;
  fwd_rows(g, runs, urows, k.run, k.a, k.b, r, st, out, tl);
}

__global__ void k_band2_bwd(const PSeg *segs, const PChunk *ch, int nch, const PRun *runs,
                            const double *urows, const double *y, const double *hstate,
                            double *out, double *heads) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nch) return;
  const PChunk k = ch[c];
  const PSeg g = segs[k.seg];
  const double *st = (hstate && k.last == 0) ? hstate + (long long)(c + 1) * kRing : nullptr;
  double *hd = (heads && k.first == 0) ? heads + (long long)c * kRing : nullptr;
  bwd_rows(g, runs, urows, k.run_hi, k.a, k.b, y, st, out, hd);
}

// Transfer matrices: column q of T = response to the unit state e_q.
__global__ void k_band2_transfer(const PSeg *segs, const PChunk *ch, const PTrans *tr, int ntr,
                                 const PRun *runs, const double *urows, double *T) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntr) return;
  const PTrans e = tr[t];
  const PChunk k = ch[e.chunk];
  const PSeg g = segs[k.seg];
  const int w = g.nb - 1;
  double unit[kRing], res[kRing];
  double *Tm = T + e.off;
  for (int q = 0; q < w; ++q) {
    for (int i = 0; i < w; ++i) unit[i] = (i == q) ? 1.0 : 0.0;
    if (e.dir == 0) fwd_rows(g, runs, urows, k.run, k.a, k.b, nullptr, unit, nullptr, res);
    else bwd_rows(g, runs, urows, k.run_hi, k.a, k.b, nullptr, unit, nullptr, res);
    for (int i = 0; i < w; ++i) Tm[(long long)i * w + q] = res[i];
  }
}

// State propagation across chunks, one warp per segment.
// dir 0: s[c] = p[c] + T_c s[c-1] for c = c0+1 .. c0+n-2 (s[c0] = p[c0])
// dir 1: s[c] = p[c] + T_c s[c+1] for c = c0+n-2 .. c0+1 (s[last] = p[last])
// The particular states and transfer offsets of the next kScanBlock chunks are
// staged in shared memory before the sequential steps, so a step waits only on
// the w x w product.
constexpr int kScanBlock = 16;
constexpr int kScanWarps = 2;

__global__ void k_band2_scan(const PSeg *segs, int nseg, const PChunk *ch, const double *T,
                             const double *p, double *s, int dir) {
  __shared__ double pbuf[kScanWarps][kScanBlock][kRing];
  __shared__ double curb[kScanWarps][kRing];
  __shared__ int toffb[kScanWarps][kScanBlock];
  const int wl = threadIdx.x >> 5;
  const int seg = blockIdx.x * kScanWarps + wl;
  const int lane = threadIdx.x & 31;
  if (seg >= nseg) return;
  const PSeg g = segs[seg];
  const int w = g.nb - 1;
  if (g.nch <= 1 || w <= 0) return;
  double *cur = curb[wl];
  const int c0 = g.ch_off, cl = g.ch_off + g.nch - 1;
  const int start = dir == 0 ? c0 : cl;
  const int stop = dir == 0 ? cl : c0;  // exclusive
  const int step = dir == 0 ? 1 : -1;
  for (int i = lane; i < w; i += 32) {
    const double v = p[(long long)start * kRing + i];
    cur[i] = v;
    s[(long long)start * kRing + i] = v;
  }
  __syncwarp();
  for (int cb = start + step; cb != stop;) {
    int nblk = 0;
    for (int u = 0, c = cb; u < kScanBlock && c != stop; ++u, c += step) ++nblk;
    for (int e = lane; e < nblk * w; e += 32) {
      const int u = e / w, i = e - u * w;
      pbuf[wl][u][i] = p[(long long)(cb + u * step) * kRing + i];
    }
    if (lane < nblk) {
      const int c = cb + lane * step;
      toffb[wl][lane] = dir == 0 ? ch[c].tf : ch[c].tb;
    }
    __syncwarp();
    for (int u = 0; u < nblk; ++u) {
      const double *Tm = T + toffb[wl][u];
      double v[kRing / 32];
      int ni = 0;
      for (int i = lane; i < w; i += 32, ++ni) {
        double acc = pbuf[wl][u][i];
        const double *Ti = Tm + (long long)i * w;
        for (int q = 0; q < w; ++q) acc += Ti[q] * cur[q];
        v[ni] = acc;
      }
      __syncwarp();
      ni = 0;
      const long long c = cb + u * step;
      for (int i = lane; i < w; i += 32, ++ni) {
        cur[i] = v[ni];
        s[c * kRing + i] = v[ni];
      }
      __syncwarp();
    }
    cb += nblk * step;
  }
}

}  // namespace

void band2_factor(cudaStream_t st, const PSeg *segs, int nseg, const int *spec,
                  const double *invcov, long long nof, const double *nna, double *urows,
                  PRun *runs, int *status, int *nunique, int *nruns) {
  if (nseg == 0) return;
  MADAM_LAUNCH(k_band2_factor, (nseg + 31) / 32, 32, 0, st, segs, nseg, spec, invcov, nof, nna,
               urows, runs, status, nunique, nruns);
}

void band2_transfer(cudaStream_t st, const PSeg *segs, const PChunk *ch, const PTrans *tr, int ntr,
                    const PRun *runs, const double *urows, double *T) {
  if (ntr == 0) return;
  MADAM_LAUNCH(k_band2_transfer, (ntr + 63) / 64, 64, 0, st, segs, ch, tr, ntr, runs, urows, T);
}

void band2_solve(cudaStream_t st, const PSeg *segs, int nseg, const PChunk *ch, int nch,
                 const PRun *runs, const double *urows, const double *T, const double *r,
                 double *z, double *work_p, double *work_s) {
  if (nch == 0) return;
  const unsigned gc = (nch + 127) / 128;
  const unsigned gs = (nseg + kScanWarps - 1) / kScanWarps;
  // forward: particular, state scan, final
  MADAM_LAUNCH(k_band2_fwd, gc, 128, 0, st, segs, ch, nch, runs, urows, r, nullptr, nullptr,
               work_p);
  MADAM_LAUNCH(k_band2_scan, gs, 32 * kScanWarps, 0, st, segs, nseg, ch, T, work_p, work_s, 0);
  MADAM_LAUNCH(k_band2_fwd, gc, 128, 0, st, segs, ch, nch, runs, urows, r, work_s, z, nullptr);
  // backward, in place on z
  MADAM_LAUNCH(k_band2_bwd, gc, 128, 0, st, segs, ch, nch, runs, urows, z, nullptr, nullptr,
               work_p);
  MADAM_LAUNCH(k_band2_scan, gs, 32 * kScanWarps, 0, st, segs, nseg, ch, T, work_p, work_s, 1);
  MADAM_LAUNCH(k_band2_bwd, gc, 128, 0, st, segs, ch, nch, runs, urows, z, work_s, z, nullptr);
}

}  // namespace madam
