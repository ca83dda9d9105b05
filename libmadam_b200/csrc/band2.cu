// Deduplicated band Cholesky preconditioner with a chunk-parallel exact solve.
//
// construct_preconditioner (noise_routines.f90:1028-1120) factors
// A = Toeplitz(invcov[0:nband]) + diag(nna) per trimmed segment (DPBTRF 'L');
// preconditioning_band (1159-1256) solves L L^T z = r (DPBTRS).
//
// Factor.  Row j of L is R_j[d] = L(j, j-d), d = 0..w (w = nband - 1), and
// depends only on rows j-w..j-1 and on nna_j.  Computed left-looking, in the
// update order of DPBTF2 (m increasing), rows settle to a fixed point after
// ~100 rows wherever nna is constant.  A row that agrees with its
// predecessor to 4 ulp in every entry is taken to be that row (in FMA
// arithmetic the fixed point can end in a last-bit limit cycle instead of a
// bitwise fixed point), and once w+1 consecutive rows are one row and
// nna_j == nna_{j-1} the next row is that row without recomputation.  The
// factor is stored as a table of distinct rows plus a run list (first row,
// table entry).
//
// Solve.  Both triangular solves are one recurrence over positions p,
//   v_p = (in_p - sum_{d=w..1} K_p[d] v_{p-d}) * (1 / K_p[0]),
// forward with p = j and K_p = row j of L (DTBSV 'L','N' order: d = w first),
// backward with p = n-1-j and K_p = column j of L, K_p[d] = L(j+d, j)
// (DTBSV 'L','T' order).  A column inside a run of equal rows is that row;
// the w columns before each run boundary and at the segment end are
// assembled into extra entries.  The positions are cut into chunks; pass 1
// solves every chunk from a zero state, a warp per segment propagates the
// true state across chunks with the w x w transfer matrices T_c (the
// response of the chunk's last w values to its w initial values,
// precomputed, one per distinct coefficient entry for chunks inside one
// run), and pass 2 re-solves each chunk from its true state.  The forward
// final pass and the backward pass 1 of a chunk run in one thread.  Widths
// up to 32 keep the recurrence window and the coefficients in registers.
#include <algorithm>
#include <climits>

#include "band2.cuh"
#include "engine.h"

namespace madam {
namespace {

constexpr int kRing = 128;               // generic window (>= w + 1)
constexpr double kFreezeTol = 0x1p-50;   // 4 ulp relative

// One warp per segment: lane 0 computes the rows; where the factor has
// reached its steady state the warp scans nna for the next change (8 values
// per lane per step) and the rows in between are copies.  rows: worst-case
// region of n * (nb + 1) doubles at seg.row_off; runs: worst-case n entries
// at seg.run_off.
constexpr int kScanPerLane = 8;

__global__ void k_band2_factor(const PSeg *segs, int nseg, const int *spec, const double *invcov,
                               long long nof, const double *nna, double *rows, PRun *runs,
                               int *status, int *nunique, int *nruns) {
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (s >= nseg) return;
  const PSeg g = segs[s];
  const int nb = g.nb, w = nb - 1, S = nb + 1;
  const double *ic = invcov + (long long)spec[s] * nof;
  const double *nn = nna + g.k0;
  double *rowbase = rows + g.row_off;
  PRun *rl = runs + g.run_off;
  const double *win[kRing];  // lane 0: the last w rows (pointers into the table)
  int nu = 0, nr = 0, same = 0;
  const double *prev = nullptr;
  int j = 0;
  while (j < g.n) {
    int jn = j;
    if (lane == 0) {
      for (; jn < g.n; ++jn) {
        if (prev && same >= w + 1 && nn[jn] == nn[jn - 1]) break;  // steady: warp scan
        double *R = rowbase + (long long)nu * S;
        for (int d = 0; d < nb; ++d) R[d] = 0.0;
        // off-diagonal entries, d = w..1 (k = jn - d increasing)
        for (int d = min(w, jn); d >= 1; --d) {
          const double *Rk = win[(jn - d) & (kRing - 1)];
          double acc = ic[d];
          // subtract L(jn, m) L(k, m) for m = jn-w .. k-1 in increasing m
          for (int e = min(w, jn); e > d; --e) acc -= R[e] * Rk[e - d];
          R[d] = acc * (1.0 / Rk[0]);
        }
        double dg = ic[0] + nn[jn];
        for (int e = min(w, jn); e >= 1; --e) dg -= R[e] * R[e];
        if (!(dg > 0)) {
          status[s] = jn + 1;
          nunique[s] = 0;
          nruns[s] = 0;
          jn = -1;
          break;
        }
        R[0] = sqrt(dg);
        bool eq = prev != nullptr;
        if (eq)
          for (int d = 0; d < nb; ++d)
            if (!(fabs(R[d] - prev[d]) <= kFreezeTol * fabs(prev[d]))) {
              eq = false;
              break;
            }
        if (eq) {
          win[jn & (kRing - 1)] = prev;
          ++same;
        } else {
          R[nb] = 1.0 / R[0];
          rl[nr].start = jn;
          rl[nr].fill = 0;
          rl[nr].off = g.row_off + (long long)nu * S;
          ++nr;
          ++nu;
          prev = R;
          win[jn & (kRing - 1)] = R;
          same = 1;
        }
      }
    }
    jn = __shfl_sync(0xffffffffu, jn, 0);
    if (jn < 0) return;
    if (jn >= g.n) break;
    // rows jn.. repeat the previous row while nna keeps its value
    const double v0 = nn[jn - 1];
    int je = jn;
    for (;;) {
      unsigned stop = 0;
#pragma unroll
      for (int u = 0; u < kScanPerLane; ++u) {
        const int idx = je + u * 32 + lane;
        if (idx >= g.n || nn[idx] != v0) stop |= 1u << u;
      }
      int first = INT_MAX;
#pragma unroll
      for (int u = 0; u < kScanPerLane; ++u) {
        const unsigned ball = __ballot_sync(0xffffffffu, (stop >> u) & 1u);
        if (ball && first == INT_MAX) first = je + u * 32 + __ffs(ball) - 1;
      }
      if (first != INT_MAX) {
        je = min(first, g.n);
        break;
      }
      je += kScanPerLane * 32;
    }
    if (lane == 0) {
      same += je - jn;
      for (int r = max(jn, je - w); r < je; ++r) win[r & (kRing - 1)] = prev;
    }
    j = je;
  }
  if (lane == 0) {
    status[s] = 0;
    nunique[s] = nu;
    nruns[s] = nr;
  }
}

// Backward entries: column j of L, C[d] = L(j+d, j) = R_{j+d}[d] (zero past
// the segment end), C[w+1] = 1 / C[0].  Block row y = segment.
__global__ void k_band2_columns(const PSeg *segs, const PRun *runs, const PRun *cruns,
                                double *tab) {
  const PSeg g = segs[blockIdx.y];
  const int w = g.nb - 1;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.ncrun; e += gridDim.x * blockDim.x) {
    const PRun c = cruns[g.crun_off + e];
    if (!c.fill) continue;
    const int j = g.n - 1 - c.start;
    double *C = tab + c.off;
    for (int d = 0; d <= w; ++d) {
      const int row = j + d;
      if (row >= g.n) {
        C[d] = 0.0;
        continue;
      }
      int lo = g.run_off, hi = g.run_off + g.nrun - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (runs[mid].start <= row) lo = mid;
        else hi = mid - 1;
      }
      const double *Rr = tab + runs[lo].off;
      C[d] = Rr[d];
      if (d == 0) C[w + 1] = Rr[w + 1];
    }
  }
}

// One direction of one segment: run list, entry table and the map from
// position p to the vector index gbase + gstep * p.
struct Seq {
  const PRun *runs;
  int rend;  // one past the segment's last run
  const double *tab;
  long long gbase;
  int gstep;
};

__device__ __forceinline__ Seq fwd_seq(const PSeg &g, const PRun *runs, const double *tab) {
  return Seq{runs, g.run_off + g.nrun, tab, g.k0, 1};
}

__device__ __forceinline__ Seq bwd_seq(const PSeg &g, const PRun *cruns, const double *tab) {
  return Seq{cruns, g.crun_off + g.ncrun, tab, g.k0 + g.n - 1, -1};
}

// Positions [p0, p1), window of any width w <= kRing - 1 in local memory.
// state: v_{p0-w..p0-1} (nullptr = zeros); writes v (if out) and the last w
// values (if tail).
__device__ void recur_generic(int w, const Seq &q, int run, int p0, int p1, const double *in,
                              const double *state, double *out, double *tail) {
  double ring[kRing];
  for (int i = 0; i < w; ++i) ring[(p0 - w + i) & (kRing - 1)] = state ? state[i] : 0.0;
  int next = (run + 1 < q.rend) ? q.runs[run + 1].start : INT_MAX;
  const double *K = q.tab + q.runs[run].off;
  for (int p = p0; p < p1; ++p) {
    while (p >= next) {
      ++run;
      K = q.tab + q.runs[run].off;
      next = (run + 1 < q.rend) ? q.runs[run + 1].start : INT_MAX;
    }
    const long long gi = q.gbase + (long long)q.gstep * p;
    double acc = in ? in[gi] : 0.0;
    for (int d = w; d >= 1; --d) acc -= K[d] * ring[(p - d) & (kRing - 1)];
    const double v = acc * K[w + 1];
    ring[p & (kRing - 1)] = v;
    if (out) out[gi] = v;
  }
  if (tail)
    for (int i = 0; i < w; ++i) tail[i] = ring[(p1 - w + i) & (kRing - 1)];
}

// The same recurrence with a compile-time window W >= w held in registers:
// the loop is unrolled by W + 1 so every window slot is a fixed register;
// taps d > w have zero coefficients.  A block of W + 1 positions that lies in
// one run and in [p0, p1) runs without branches; the inputs of the next
// block are loaded while the current one is computed (W <= 16).
template <int W, bool HAS_IN, bool HAS_OUT>
__device__ __forceinline__ void recur_reg(int w, const Seq &q, int run, int p0, int p1,
                                          const double *in, const double *state, double *out,
                                          double *tail) {
  constexpr int R = W + 1;
  constexpr bool kAhead = W <= 16;
  double v[R];  // slot of position p: (p - p0) mod R
#pragma unroll
  for (int s = 0; s < R; ++s) {
    const int m = R - s;  // slot s >= 1 holds v_{p0-m}
    v[s] = (s >= 1 && m <= w && state) ? state[w - m] : 0.0;
  }
  double K[W + 1];
  double kinv;
  int next;
  auto load = [&](int rr) {
    const double *E = q.tab + q.runs[rr].off;
#pragma unroll
    for (int d = 1; d <= W; ++d) K[d] = d <= w ? E[d] : 0.0;
    kinv = E[w + 1];
    next = (rr + 1 < q.rend) ? q.runs[rr + 1].start : INT_MAX;
  };
  load(run);
  const long long gs = q.gstep;
  double buf[kAhead ? R : 1];
  auto fetch = [&](int pb) {
#pragma unroll
    for (int t = 0; t < R; ++t) {
      const int p = pb + t;
      buf[t] = (HAS_IN && p < p1) ? in[q.gbase + gs * p] : 0.0;
    }
  };
  if (kAhead) fetch(p0);
  for (int pb = p0; pb < p1; pb += R) {
    double cur[R];
    if (kAhead) {
#pragma unroll
      for (int t = 0; t < R; ++t) cur[t] = buf[t];
      fetch(pb + R);
    } else {
#pragma unroll
      for (int t = 0; t < R; ++t) {
        const int p = pb + t;
        cur[t] = (HAS_IN && p < p1) ? in[q.gbase + gs * p] : 0.0;
      }
    }
    if (pb + R <= p1 && pb + R <= next) {
#pragma unroll
      for (int t = 0; t < R; ++t) {
        double acc = cur[t];
#pragma unroll
        for (int d = W; d >= 1; --d) acc -= K[d] * v[(t - d + 2 * R) % R];
        v[t] = acc * kinv;
        if (HAS_OUT) out[q.gbase + gs * (pb + t)] = v[t];
      }
    } else {
#pragma unroll
      for (int t = 0; t < R; ++t) {
        const int p = pb + t;
        if (p < p1) {
          if (p >= next) {
            while (p >= next) {
              ++run;
              next = (run + 1 < q.rend) ? q.runs[run + 1].start : INT_MAX;
            }
            load(run);
          }
          double acc = cur[t];
#pragma unroll
          for (int d = W; d >= 1; --d) acc -= K[d] * v[(t - d + 2 * R) % R];
          v[t] = acc * kinv;
          if (HAS_OUT) out[q.gbase + gs * p] = v[t];
        }
      }
    }
  }
  if (tail) {
    const int base = (((p1 - p0 - w) % R) + R) % R;  // slot of v_{p1-w}
#pragma unroll
    for (int s = 0; s < R; ++s) {
      int i = s - base;
      if (i < 0) i += R;
      if (i < w) tail[i] = v[s];
    }
  }
}

template <int W, bool HAS_IN, bool HAS_OUT>
__device__ __forceinline__ void recur(int w, const Seq &q, int run, int p0, int p1,
                                      const double *in, const double *state, double *out,
                                      double *tail) {
  if (W == 0) recur_generic(w, q, run, p0, p1, HAS_IN ? in : nullptr, state,
                            HAS_OUT ? out : nullptr, tail);
  else recur_reg<(W > 0 ? W : 1), HAS_IN, HAS_OUT>(w, q, run, p0, p1, in, state, out, tail);
}

// ------------------------------------------------------ staged passes --
// A warp takes 32 consecutive chunks, one per lane.  Each lane's positions are
// read and written through shared-memory tiles: for every chunk of the warp
// the lanes copy 32 consecutive values with 8-byte cp.async (one 256-byte
// segment per copy round instead of 32 scattered lines), the next tile
// streaming in while the current one is solved.  Tiles are TP positions, a
// multiple of the window R = W + 1, so the register window keeps its slot
// mapping across tiles.
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int W>
struct Stage {
  static constexpr int R = W + 1;
  static constexpr int TP = R * ((32 + R - 1) / R);  // tile positions
  static constexpr int LD = TP + 1;                  // padded row
  static constexpr int M = (TP + 31) / 32;           // copy rounds per row
  static constexpr size_t kSmem = (size_t)3 * 32 * LD * sizeof(double);
};

// One lane's chunk in one direction: positions t in [0, len) are vector index
// base + step * t and recurrence position p0 + t.
struct Lane {
  long long base;
  int step, len, p0, run;
  const PRun *runs;
  int rend;
};

template <int W, bool HAS_OUT>
__device__ void staged_recur(double *tin, double *tout, long long *sb, int *ss, int *sl,
                             const double *tab, const Lane &L, int w, const double *in,
                             const double *state, double *out, double *tail) {
  using G = Stage<W>;
  constexpr int R = G::R, TP = G::TP, LD = G::LD, M = G::M;
  const int lane = threadIdx.x & 31;
  __syncwarp();
  sb[lane] = L.base;
  ss[lane] = L.step;
  sl[lane] = L.len;
  int maxlen = L.len;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, o));
  __syncwarp();
  const int ntile = (maxlen + TP - 1) / TP;
  auto stage = [&](int k, int b) {
    double *dst = tin + (size_t)b * 32 * LD;
    for (int j = 0; j < 32; ++j) {
      const int len = sl[j];
      const long long base = sb[j];
      const int step = ss[j];
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int x = lane + 32 * m;
        const int t = k * TP + x;
        if (x < TP && t < len) cp_async8(dst + j * LD + x, in + base + (long long)step * t);
      }
    }
  };
  // register window: slot of position t is t mod R
  double v[R];
#pragma unroll
  for (int s = 0; s < R; ++s) {
    const int m = R - s;  // slot s >= 1 holds the value m positions before the start
    v[s] = (s >= 1 && m <= w && state) ? state[w - m] : 0.0;
  }
  double K[W + 1];
  double kinv = 0;
  int run = L.run, next = INT_MAX;
  auto load = [&](int rr) {
    const double *E = tab + L.runs[rr].off;
#pragma unroll
    for (int d = 1; d <= W; ++d) K[d] = d <= w ? E[d] : 0.0;
    kinv = E[w + 1];
    next = (rr + 1 < L.rend) ? L.runs[rr + 1].start : INT_MAX;
  };
  if (L.len > 0) load(run);
  if (ntile > 0) stage(0, 0);
  cp_async_commit();
  for (int k = 0; k < ntile; ++k) {
    if (k + 1 < ntile) stage(k + 1, (k + 1) & 1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncwarp();
    const double *row = tin + (size_t)(k & 1) * 32 * LD + lane * LD;
    double *orow = tout + lane * LD;
#pragma unroll 1
    for (int b0 = 0; b0 < TP; b0 += R) {
      const int t0 = k * TP + b0;
      if (t0 >= L.len) break;
      const int pb = L.p0 + t0;
      if (t0 + R <= L.len && pb + R <= next) {
#pragma unroll
        for (int t = 0; t < R; ++t) {
          double acc = row[b0 + t];
#pragma unroll
          for (int d = W; d >= 1; --d) acc -= K[d] * v[(t - d + 2 * R) % R];
          v[t] = acc * kinv;
          if (HAS_OUT) orow[b0 + t] = v[t];
        }
      } else {
#pragma unroll
        for (int t = 0; t < R; ++t) {
          if (t0 + t < L.len) {
            const int p = pb + t;
            if (p >= next) {
              while (p >= next) {
                ++run;
                next = (run + 1 < L.rend) ? L.runs[run + 1].start : INT_MAX;
              }
              load(run);
            }
            double acc = row[b0 + t];
#pragma unroll
            for (int d = W; d >= 1; --d) acc -= K[d] * v[(t - d + 2 * R) % R];
            v[t] = acc * kinv;
            if (HAS_OUT) orow[b0 + t] = v[t];
          }
        }
      }
    }
    __syncwarp();
    if (HAS_OUT) {
      for (int j = 0; j < 32; ++j) {
        const int len = sl[j];
        const long long base = sb[j];
        const int step = ss[j];
#pragma unroll
        for (int m = 0; m < M; ++m) {
          const int x = lane + 32 * m;
          const int t = k * TP + x;
          if (x < TP && t < len) out[base + (long long)step * t] = tout[j * LD + x];
        }
      }
      __syncwarp();
    }
  }
  cp_async_wait<0>();
  __syncwarp();
  if (tail && L.len > 0) {
    const int base = (((L.len - w) % R) + R) % R;  // slot of the value w before the end
#pragma unroll
    for (int s = 0; s < R; ++s) {
      int i = s - base;
      if (i < 0) i += R;
      if (i < w) tail[i] = v[s];
    }
  }
}

// mode 0: forward pass 1 (tails -> wp)
// mode 1: forward pass 2 (state ws[c-1], writes z), then backward pass 1 on
//         the chunk's own rows of z (tails -> wp)
// mode 2: backward pass 2 (state ws[c+1], z in place)
template <int W>
__global__ void __launch_bounds__(32) k_band2_pass_staged(
    const PSeg *segs, const PChunk *ch, int c0, int c1, const PRun *runs, const PRun *cruns,
    const double *tab, int mode, const double *r, double *z, const double *ws, double *wp) {
  extern __shared__ double bsm[];
  __shared__ long long sb[32];
  __shared__ int ss[32], sl[32];
  using G = Stage<W>;
  double *tin = bsm, *tout = bsm + 2 * 32 * G::LD;
  const int lane = threadIdx.x & 31;
  const int c = c0 + blockIdx.x * 32 + lane;
  const bool act = c < c1;
  PChunk k{};
  PSeg g{};
  if (act) {
    k = ch[c];
    g = segs[k.seg];
  }
  const int w = g.nb - 1;
  Lane f{}, b{};
  if (act) {
    f = Lane{g.k0 + k.a, 1, k.b - k.a, k.a, k.run_f, runs, g.run_off + g.nrun};
    b = Lane{g.k0 + k.b - 1, -1, k.b - k.a, g.n - k.b, k.run_b, cruns, g.crun_off + g.ncrun};
  }
  if (mode == 0) {
    staged_recur<W, false>(tin, tout, sb, ss, sl, tab, f, w, r, nullptr, nullptr,
                           (act && !k.last) ? wp + (long long)c * kBand2State : nullptr);
    return;
  }
  if (mode == 1) {
    staged_recur<W, true>(tin, tout, sb, ss, sl, tab, f, w, r,
                          (act && !k.first) ? ws + (long long)(c - 1) * kBand2State : nullptr,
                          z, nullptr);
    __threadfence_block();
    __syncwarp();
    staged_recur<W, false>(tin, tout, sb, ss, sl, tab, b, w, z, nullptr, nullptr,
                           (act && !k.first) ? wp + (long long)c * kBand2State : nullptr);
    return;
  }
  staged_recur<W, true>(tin, tout, sb, ss, sl, tab, b, w, z,
                        (act && !k.last) ? ws + (long long)(c + 1) * kBand2State : nullptr, z,
                        nullptr);
}

// Widths above 32: one thread per chunk, window in local memory.
__global__ void __launch_bounds__(64) k_band2_pass_generic(
    const PSeg *segs, const PChunk *ch, int c0, int c1, const PRun *runs, const PRun *cruns,
    const double *tab, int mode, const double *r, double *z, const double *ws, double *wp) {
  const int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= c1) return;
  const PChunk k = ch[c];
  const PSeg g = segs[k.seg];
  const int w = g.nb - 1;
  if (mode <= 1) {
    const Seq f = fwd_seq(g, runs, tab);
    if (mode == 0) {
      recur_generic(w, f, k.run_f, k.a, k.b, r, nullptr, nullptr,
                    k.last ? nullptr : wp + (long long)c * kBand2State);
      return;
    }
    recur_generic(w, f, k.run_f, k.a, k.b, r,
                  k.first ? nullptr : ws + (long long)(c - 1) * kBand2State, z, nullptr);
    const Seq b = bwd_seq(g, cruns, tab);
    recur_generic(w, b, k.run_b, g.n - k.b, g.n - k.a, z, nullptr, nullptr,
                  k.first ? nullptr : wp + (long long)c * kBand2State);
    return;
  }
  const Seq b = bwd_seq(g, cruns, tab);
  recur_generic(w, b, k.run_b, g.n - k.b, g.n - k.a, z,
                k.last ? nullptr : ws + (long long)(c + 1) * kBand2State, z, nullptr);
}

// ------------------------------------------------------- guarded solve --
// One warp (one block) takes 32 guarded chunks, one per lane, and walks them
// in tiles of TP positions (a multiple of the window R = W + 1, so the
// register window keeps its slot mapping across tiles).  A lane's positions
// of one tile are contiguous in memory (ascending forward, descending
// backward), so the lane stages them with one 1-D bulk copy
// (cp.async.bulk, completion on an mbarrier, no cluster multicast) into its
// shared-memory row, the next tile streaming in while the current one is
// solved; the outputs go to a second row and back with one bulk store per
// lane (the 16-byte-aligned interior) plus plain stores of at most two edge
// values.  Bulk copies move whole aligned 16-byte blocks, so a row holds
// the tile from the 16-byte boundary at or below its lowest address; reading
// the whole blocks never leaves the pages the tile lies in.  Waits on the
// mbarrier are bounded: a wait that runs out sets *err and the warp returns.
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes,
                                          unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void bulk_store(void *dst, const void *src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst),
               "r"(smem_u32(src)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read0() {
  asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
}
__device__ __forceinline__ void bulk_wait0() {
  asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// Tiles of about 32 positions, 3 in flight per lane (measured on B200: 2
// and 4 run alike, tiles of 16 or 64 positions slower).
template <int W>
struct GStage {
  static constexpr int R = W + 1;
  static constexpr int TP = R * (R > 32 ? 1 : 32 / R);  // tile positions
  // row length: the tile plus one double of alignment slack on either side,
  // even (16-byte rows) and 2 mod 16 (consecutive rows start 2 banks apart)
  static constexpr int L0 = TP + 2;
  static constexpr int LD = L0 + (((2 - L0) % 16) + 16) % 16;
  static constexpr int NS = 3;  // tiles in flight (ring of row buffers)
  static constexpr size_t kSmem = (size_t)NS * 32 * LD * sizeof(double);
};
constexpr long kGuardWaitLimit = 1L << 22;

// One step of the recurrence at window slot t (positions ahead of the
// previous are v[(t - d) mod R]): the older taps d = W..2 summed in two
// interleaved partial sums, then the tap d = 1.  (DTBSV sums d = w..1 in one
// sequence; this order differs by rounding only.)
template <int W>
__device__ __forceinline__ double guard_step(const double (&K)[W + 1], const double (&v)[W + 1],
                                             int t, double x, double kinv) {
  constexpr int R = W + 1;
  double a0 = x, a1 = 0.0;
#pragma unroll
  for (int d = W; d >= 2; --d) {
    if ((d & 1) == (W & 1)) a0 -= K[d] * v[(t - d + 2 * R) % R];
    else a1 -= K[d] * v[(t - d + 2 * R) % R];
  }
  return ((a0 + a1) - K[1] * v[(t - 1 + 2 * R) % R]) * kinv;
}

// DIR 0: forward (ascending indices), 1: backward (descending).  Tiles
// stream through a ring of NS row buffers; each value's output overwrites
// its input slot (it is not read again), and the row goes back with the bulk
// store when `in` and `out` share their 16-byte phase at the tile (else with
// plain stores).
template <int W, int DIR>
__global__ void __launch_bounds__(32) k_band2_guard_pass(
    const PSeg *segs, const GChunk *gc, int c0, int c1, const PRun *runs, const PRun *cruns,
    const double *tab, const double *in, double *out, int *err) {
  using G = GStage<W>;
  constexpr int R = G::R, TP = G::TP, LD = G::LD, NS = G::NS;
  constexpr int S = DIR == 0 ? 1 : -1;  // index step per position
  extern __shared__ __align__(16) double gsm[];
  __shared__ __align__(8) unsigned long long bar[NS];
  const int lane = threadIdx.x & 31;
  const int c = c0 + blockIdx.x * 32 + lane;
  // this lane's chunk: positions t in [0, len) at vector index base + S t,
  // recurrence position p0 + t; positions below skip are the guard
  long long base = 0;
  int len = 0, p0 = 0, skip = 0, run = 0, rend = 0, w = 0;
  const PRun *rl = DIR == 0 ? runs : cruns;
  if (c < c1) {
    const GChunk k = gc[c];
    const PSeg g = segs[k.seg];
    w = g.nb - 1;
    if (DIR == 0) {
      base = g.k0 + k.ga;
      len = k.b - k.ga;
      p0 = k.ga;
      skip = k.a - k.ga;
      run = k.run_fg;
      rend = g.run_off + g.nrun;
    } else {
      base = g.k0 + g.n - 1 - k.gp;
      len = g.n - k.a - k.gp;
      p0 = k.gp;
      skip = g.n - k.b - k.gp;
      run = k.run_bg;
      rend = g.crun_off + g.ncrun;
    }
  }
  int maxlen = len;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, o));
  const int ntile = (maxlen + TP - 1) / TP;
  if (lane == 0) {
#pragma unroll
    for (int b = 0; b < NS; ++b) mbar_init(&bar[b], 32);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncwarp();
  // lowest vector index of tile k's positions [t0, t1) (nt = t1 - t0 > 0)
  auto tile_lo = [&](int k, int &nt) -> long long {
    const int t0 = k * TP, t1 = min(len, t0 + TP);
    nt = t1 - t0;
    return DIR == 0 ? base + t0 : base - (t1 - 1);
  };
  auto issue = [&](int k) {
    const int b = k % NS;
    int nt = 0;
    const long long lo = tile_lo(k, nt);
    unsigned bytes = 0;
    const char *src = nullptr;
    if (nt > 0) {
      const uintptr_t a0 = (uintptr_t)(in + lo) & ~(uintptr_t)15;
      const uintptr_t a1 = ((uintptr_t)(in + lo + nt - 1) + 8 + 15) & ~(uintptr_t)15;
      src = (const char *)a0;
      bytes = (unsigned)(a1 - a0);
    }
    mbar_arrive_tx(&bar[b], bytes);
    if (bytes) bulk_load(gsm + (b * 32 + lane) * LD, src, bytes, &bar[b]);
  };
  double v[R];
#pragma unroll
  for (int q = 0; q < R; ++q) v[q] = 0.0;
  double K[W + 1];
  K[0] = 0.0;
  double kinv = 0;
  int next = INT_MAX;
  auto load = [&](int rr) {
    const double *E = tab + rl[rr].off;
#pragma unroll
    for (int d = 1; d <= W; ++d) K[d] = d <= w ? E[d] : 0.0;
    kinv = E[w + 1];
    next = (rr + 1 < rend) ? rl[rr + 1].start : INT_MAX;
  };
  if (len > 0) load(run);
  for (int k = 0; k < NS - 1 && k < ntile; ++k) issue(k);
  for (int k = 0; k < ntile; ++k) {
    if (k + NS - 1 < ntile) {
      // the ring slot of tile k - 1: its bulk store has read it
      bulk_wait_read0();
      fence_proxy_async();
      issue(k + NS - 1);
    }
    {
      const unsigned parity = (unsigned)(k / NS) & 1u;
      long it = 0;
      while (!mbar_try_wait(&bar[k % NS], parity)) {
        if (++it > kGuardWaitLimit) {
          if (lane == 0) atomicOr(err, 1);
          bulk_wait0();
          return;
        }
      }
    }
    int nt = 0;
    const long long lo = tile_lo(k, nt);
    // index i sits at slot lead + (i - lo) of the row (lead: 8-byte offset of
    // in + lo in its 16-byte block); position t0 + x is index lo + x
    // forward, lo + nt - 1 - x backward
    double *row = gsm + ((k % NS) * 32 + lane) * LD;
    const int lead = nt > 0 ? (int)(((uintptr_t)(in + lo) >> 3) & 1) : 0;
    double *ip = row + lead + (DIR == 0 ? 0 : nt - 1);
#pragma unroll 1
    for (int b0 = 0; b0 < TP; b0 += R) {
      const int t0 = k * TP + b0;
      if (t0 >= len) break;
      const int pb = p0 + t0;
      if (t0 + R <= len && pb + R <= next) {
#pragma unroll
        for (int t = 0; t < R; ++t) {
          v[t] = guard_step<W>(K, v, t, ip[S * (b0 + t)], kinv);
          ip[S * (b0 + t)] = v[t];
        }
      } else {
#pragma unroll
        for (int t = 0; t < R; ++t) {
          if (t0 + t < len) {
            const int p = pb + t;
            if (p >= next) {
              while (p >= next) {
                ++run;
                next = (run + 1 < rend) ? rl[run + 1].start : INT_MAX;
              }
              load(run);
            }
            v[t] = guard_step<W>(K, v, t, ip[S * (b0 + t)], kinv);
            ip[S * (b0 + t)] = v[t];
          }
        }
      }
    }
    // write the tile's outputs past the guard: positions [max(t0, skip), t1)
    const int tw0 = max(k * TP, skip), tw1 = min(len, (k + 1) * TP);
    if (tw1 > tw0) {
      const long long wlo = DIR == 0 ? base + tw0 : base - (tw1 - 1);
      const long long whi = DIR == 0 ? base + (tw1 - 1) : base - tw0;
      const int olead = (int)(((uintptr_t)(out + lo) >> 3) & 1);
      if (olead != lead) {
        for (long long i = wlo; i <= whi; ++i) out[i] = row[lead + (i - lo)];
      } else {
        // [alo, aend): the written bytes; [ilo, iend): their whole 16-byte
        // blocks (bulk store); a value in a partly written block is stored
        // alone (at most one at either end)
        const uintptr_t alo = (uintptr_t)(out + wlo), aend = (uintptr_t)(out + whi) + 8;
        const uintptr_t ilo = (alo + 15) & ~(uintptr_t)15, iend = aend & ~(uintptr_t)15;
        if (alo < ilo) out[wlo] = row[lead + (wlo - lo)];
        if (aend > iend) out[whi] = row[lead + (whi - lo)];
        if (iend > ilo) {
          const long long i0 = (long long)((const double *)ilo - out);
          fence_proxy_async();
          bulk_store((void *)ilo, row + lead + (i0 - lo), (unsigned)(iend - ilo));
        }
      }
    }
    bulk_commit();
    __syncwarp();
  }
  bulk_wait0();
}

// Guard check: thread (chunk, direction, q) runs the recurrence over the
// guard from the unit state e_q with zero input and records the largest
// entry of the state it reaches (a max over non-negative doubles, as bits).
template <int W>
__global__ void k_band2_guard_check(const PSeg *segs, const GChunk *gc, int c0, int c1,
                                    const PRun *runs, const PRun *cruns, const double *tab,
                                    unsigned long long *worst) {
  constexpr int WS = W > 0 ? W : kRing - 1;
  const long long gid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long c = c0 + gid / (2 * WS);
  const int rem = (int)(gid % (2 * WS));
  const int dir = rem / WS, qq = rem % WS;
  if (c >= c1) return;
  const GChunk k = gc[c];
  const PSeg g = segs[k.seg];
  const int w = g.nb - 1;
  if (qq >= w) return;
  const int p0 = dir == 0 ? k.ga : k.gp;
  const int p1 = dir == 0 ? k.a : g.n - k.b;
  if (p1 <= p0) return;
  double unit[WS], res[WS];
  for (int i = 0; i < w; ++i) unit[i] = (i == qq) ? 1.0 : 0.0;
  if (dir == 0)
    recur<W, false, false>(w, fwd_seq(g, runs, tab), k.run_fg, p0, p1, nullptr, unit, nullptr,
                           res);
  else
    recur<W, false, false>(w, bwd_seq(g, cruns, tab), k.run_bg, p0, p1, nullptr, unit, nullptr,
                           res);
  double m = 0;
  for (int i = 0; i < w; ++i) m = fmax(m, fabs(res[i]));
  if (!(m <= 1e300)) m = 1e300;  // a NaN or an overflow fails the check
  atomicMax(worst + c, (unsigned long long)__double_as_longlong(m));
}

// Transfer matrices: column q of T = response of the tail to the unit state
// e_q with zero input; one thread per (matrix, q).
template <int W>
__global__ void k_band2_transfer(const PSeg *segs, const PChunk *ch, const PTrans *tr, int t0,
                                 int t1, const PRun *runs, const PRun *cruns, const double *tab,
                                 double *T) {
  constexpr int WS = W > 0 ? W : kRing - 1;
  const long long gid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long t = t0 + gid / WS;
  const int qq = (int)(gid % WS);
  if (t >= t1) return;
  const PTrans e = tr[t];
  const PChunk k = ch[e.chunk];
  const PSeg g = segs[k.seg];
  const int w = g.nb - 1;
  if (qq >= w) return;
  double unit[WS], res[WS];
  for (int i = 0; i < w; ++i) unit[i] = (i == qq) ? 1.0 : 0.0;
  if (e.dir == 0)
    recur<W, false, false>(w, fwd_seq(g, runs, tab), k.run_f, k.a, k.b, nullptr, unit, nullptr,
                           res);
  else
    recur<W, false, false>(w, bwd_seq(g, cruns, tab), k.run_b, g.n - k.b, g.n - k.a, nullptr,
                           unit, nullptr, res);
  for (int i = 0; i < w; ++i) T[e.off + (long long)i * w + qq] = res[i];
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
  __shared__ double pbuf[kScanWarps][kScanBlock][kBand2State];
  __shared__ double curb[kScanWarps][kBand2State];
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
    const double v = p[(long long)start * kBand2State + i];
    cur[i] = v;
    s[(long long)start * kBand2State + i] = v;
  }
  __syncwarp();
  for (int cb = start + step; cb != stop;) {
    int nblk = 0;
    for (int u = 0, c = cb; u < kScanBlock && c != stop; ++u, c += step) ++nblk;
    for (int e = lane; e < nblk * w; e += 32) {
      const int u = e / w, i = e - u * w;
      pbuf[wl][u][i] = p[(long long)(cb + u * step) * kBand2State + i];
    }
    if (lane < nblk) {
      const int c = cb + lane * step;
      toffb[wl][lane] = dir == 0 ? ch[c].tf : ch[c].tb;
    }
    __syncwarp();
    for (int u = 0; u < nblk; ++u) {
      const double *Tm = T + toffb[wl][u];
      double v[kBand2State / 32];
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
        s[c * kBand2State + i] = v[ni];
      }
      __syncwarp();
    }
    cb += nblk * step;
  }
}

// The same propagation with the state in registers (lane i holds s_i,
// w <= W <= 32): lane i keeps row i of the current T_c in registers (reloaded
// only when the matrix changes) and gathers the state by shuffles; the next
// chunk's particular state and matrix offset are loaded one step ahead.
// The same propagation with the state in registers (lane i holds s_i,
// w <= W <= 32): lane i keeps row i of the current T_c in registers (reloaded
// only when the matrix changes) and gathers the state by shuffles.  The
// particular states and matrix offsets of the next 32 chunks are copied into
// shared memory (cp.async) while the current 32 steps run, so a step waits
// only on its own arithmetic.  One warp per segment.
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}

template <int W>
__global__ void __launch_bounds__(32) k_band2_scan_reg(const PSeg *segs, int s0, const int *toff,
                                                       const double *T, const double *p,
                                                       double *s, int dir) {
  constexpr int B = 32;  // steps per staged block
  __shared__ double pbuf[2][B][W];
  __shared__ int tbuf[2][B];
  const int seg = s0 + blockIdx.x;
  const int lane = threadIdx.x & 31;
  const PSeg g = segs[seg];
  const int w = g.nb - 1;
  if (g.nch <= 1 || w <= 0) return;
  const bool on = lane < w;
  const int start = dir == 0 ? g.ch_off : g.ch_off + g.nch - 1;
  const int step = dir == 0 ? 1 : -1;
  const int nsteps = g.nch - 2;  // chunks after start whose state is needed
  double cur = on ? p[(long long)start * kBand2State + lane] : 0.0;
  if (on) s[(long long)start * kBand2State + lane] = cur;
  if (nsteps <= 0) return;
  const int nblk = (nsteps + B - 1) / B;
  auto stage = [&](int blk, int b) {
    for (int r = 0; r < B; ++r) {
      const int u = blk * B + r;
      if (u >= nsteps) break;
      const long long c = start + (long long)(u + 1) * step;
      if (on) cp_async8(&pbuf[b][r][lane], p + c * kBand2State + lane);
      if (lane == 0) cp_async4(&tbuf[b][r], toff + c);
    }
  };
  double Tr[W];
  int tcur = -1;
  stage(0, 0);
  cp_async_commit();
  for (int blk = 0; blk < nblk; ++blk) {
    if (blk + 1 < nblk) stage(blk + 1, (blk + 1) & 1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncwarp();
    const int b = blk & 1;
    const int nr = min(B, nsteps - blk * B);
    for (int r = 0; r < nr; ++r) {
      const double pc = on ? pbuf[b][r][lane] : 0.0;
      const int tc = tbuf[b][r];
      if (tc != tcur) {
#pragma unroll
        for (int qq = 0; qq < W; ++qq)
          Tr[qq] = (on && qq < w) ? T[tc + (long long)lane * w + qq] : 0.0;
        tcur = tc;
      }
      double a0 = pc, a1 = 0, a2 = 0, a3 = 0;
#pragma unroll
      for (int qq = 0; qq < W; qq += 4) {
        a0 += Tr[qq] * __shfl_sync(0xffffffffu, cur, qq);
        if (qq + 1 < W) a1 += Tr[qq + 1] * __shfl_sync(0xffffffffu, cur, qq + 1);
        if (qq + 2 < W) a2 += Tr[qq + 2] * __shfl_sync(0xffffffffu, cur, qq + 2);
        if (qq + 3 < W) a3 += Tr[qq + 3] * __shfl_sync(0xffffffffu, cur, qq + 3);
      }
      cur = on ? (a0 + a1) + (a2 + a3) : 0.0;
      const long long c = start + (long long)(blk * B + r + 1) * step;
      if (on) s[c * kBand2State + lane] = cur;
    }
    __syncwarp();
  }
  cp_async_wait<0>();
}

template <int W>
void launch_pass(cudaStream_t st, const PSeg *segs, const PChunk *ch, int c0, int c1,
                 const PRun *runs, const PRun *cruns, const double *tab, int mode, const double *r,
                 double *z, const double *ws, double *wp) {
  if (W == 0) {
    const unsigned grid = (unsigned)((c1 - c0 + 63) / 64);
    MADAM_LAUNCH(k_band2_pass_generic, grid, 64, 0, st, segs, ch, c0, c1, runs, cruns, tab, mode,
                 r, z, ws, wp);
    return;
  }
  constexpr int WW = W > 0 ? W : 1;
  static bool attr = false;
  if (!attr) {
    MADAM_CUDA(cudaFuncSetAttribute(k_band2_pass_staged<WW>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)Stage<WW>::kSmem));
    attr = true;
  }
  const unsigned grid = (unsigned)((c1 - c0 + 31) / 32);
  MADAM_LAUNCH(k_band2_pass_staged<WW>, grid, 32, Stage<WW>::kSmem, st, segs, ch, c0, c1, runs,
               cruns, tab, mode, r, z, ws, wp);
}

// Register widths compiled: the band widths precond_width_min = 10 gives
// (10, 20, 30) exactly, others padded to the next width.
constexpr int kWidths[] = {1, 2, 4, 8, 9, 12, 16, 19, 24, 29, 32};

void pass_class(int W, cudaStream_t st, const PSeg *segs, const PChunk *ch, int c0, int c1,
                const PRun *runs, const PRun *cruns, const double *tab, int mode, const double *r,
                double *z, const double *ws, double *wp) {
  switch (W) {
#define MADAM_BAND2_CASE(X) \
  case X: launch_pass<X>(st, segs, ch, c0, c1, runs, cruns, tab, mode, r, z, ws, wp); break;
    MADAM_BAND2_CASE(1)
    MADAM_BAND2_CASE(2)
    MADAM_BAND2_CASE(4)
    MADAM_BAND2_CASE(8)
    MADAM_BAND2_CASE(9)
    MADAM_BAND2_CASE(12)
    MADAM_BAND2_CASE(16)
    MADAM_BAND2_CASE(19)
    MADAM_BAND2_CASE(24)
    MADAM_BAND2_CASE(29)
    MADAM_BAND2_CASE(32)
#undef MADAM_BAND2_CASE
    default: launch_pass<0>(st, segs, ch, c0, c1, runs, cruns, tab, mode, r, z, ws, wp); break;
  }
}

}  // namespace

int band2_class_width(int w) {
  for (int W : kWidths)
    if (W >= w) return W;
  return 0;
}

void band2_factor(cudaStream_t st, const PSeg *segs, int nseg, const int *spec,
                  const double *invcov, long long nof, const double *nna, double *rows,
                  PRun *runs, int *status, int *nunique, int *nruns) {
  if (nseg == 0) return;
  MADAM_LAUNCH(k_band2_factor, (unsigned)nseg, 32, 0, st, segs, nseg, spec, invcov, nof, nna,
               rows, runs, status, nunique, nruns);
}

void band2_columns(cudaStream_t st, const PSeg *segs, int nseg, int max_ncrun, const PRun *runs,
                   const PRun *cruns, double *tab) {
  if (nseg == 0 || max_ncrun == 0) return;
  const dim3 grid((unsigned)std::min(64, (max_ncrun + 255) / 256), (unsigned)nseg);
  MADAM_LAUNCH(k_band2_columns, grid, 256, 0, st, segs, runs, cruns, tab);
}

void band2_transfer(cudaStream_t st, const PSeg *segs, const PChunk *ch, const PTrans *tr,
                    const int *cls_w, const int *tcls_begin, int ncls, const PRun *runs,
                    const PRun *cruns, const double *tab, double *T) {
  for (int i = 0; i < ncls; ++i) {
    const int t0 = tcls_begin[i], t1 = tcls_begin[i + 1];
    if (t1 <= t0) continue;
    const int W = cls_w[i];
    const long long nthr = (long long)(t1 - t0) * (W > 0 ? W : kRing - 1);
    const unsigned grid = (unsigned)((nthr + 63) / 64);
    switch (W) {
#define MADAM_BAND2_CASE(X)                                                                 \
  case X:                                                                                   \
    MADAM_LAUNCH(k_band2_transfer<X>, grid, 64, 0, st, segs, ch, tr, t0, t1, runs, cruns, tab, \
                 T);                                                                        \
    break;
      MADAM_BAND2_CASE(1)
      MADAM_BAND2_CASE(2)
      MADAM_BAND2_CASE(4)
      MADAM_BAND2_CASE(8)
      MADAM_BAND2_CASE(9)
      MADAM_BAND2_CASE(12)
      MADAM_BAND2_CASE(16)
      MADAM_BAND2_CASE(19)
      MADAM_BAND2_CASE(24)
      MADAM_BAND2_CASE(29)
      MADAM_BAND2_CASE(32)
#undef MADAM_BAND2_CASE
      default:
        MADAM_LAUNCH(k_band2_transfer<0>, grid, 64, 0, st, segs, ch, tr, t0, t1, runs, cruns, tab,
                     T);
        break;
    }
  }
}

void band2_solve(cudaStream_t st, const PSeg *segs, int nseg, const PChunk *ch, int nch,
                 const int *toff_f, const int *toff_b, const int *cls_w, const int *cls_begin,
                 const int *cls_seg, int ncls, const PRun *runs, const PRun *cruns,
                 const double *tab, const double *T, const double *r, double *z, double *work_p,
                 double *work_s) {
  if (nch == 0) return;
  auto passes = [&](int mode) {
    for (int i = 0; i < ncls; ++i)
      if (cls_begin[i + 1] > cls_begin[i])
        pass_class(cls_w[i], st, segs, ch, cls_begin[i], cls_begin[i + 1], runs, cruns, tab, mode,
                   r, z, work_s, work_p);
  };
  auto scans = [&](int dir) {
    for (int i = 0; i < ncls; ++i) {
      const int s0 = cls_seg[i], s1 = cls_seg[i + 1];
      if (s1 <= s0) continue;
      const unsigned grid = (unsigned)(s1 - s0);
      switch (cls_w[i]) {
#define MADAM_BAND2_CASE(X)                                                                   \
  case X:                                                                                     \
    MADAM_LAUNCH(k_band2_scan_reg<X>, grid, 32, 0, st, segs, s0, dir == 0 ? toff_f : toff_b,   \
                 T, work_p, work_s, dir);                                                     \
    break;
        MADAM_BAND2_CASE(1)
        MADAM_BAND2_CASE(2)
        MADAM_BAND2_CASE(4)
        MADAM_BAND2_CASE(8)
        MADAM_BAND2_CASE(9)
        MADAM_BAND2_CASE(12)
        MADAM_BAND2_CASE(16)
        MADAM_BAND2_CASE(19)
        MADAM_BAND2_CASE(24)
        MADAM_BAND2_CASE(29)
        MADAM_BAND2_CASE(32)
#undef MADAM_BAND2_CASE
        default:
          MADAM_LAUNCH(k_band2_scan, (unsigned)((s1 - s0 + kScanWarps - 1) / kScanWarps),
                       32 * kScanWarps, 0, st, segs + s0, s1 - s0, ch, T, work_p, work_s, dir);
          break;
      }
    }
  };
  passes(0);
  scans(0);
  passes(1);
  scans(1);
  passes(2);
}

void band2_guard_check(cudaStream_t st, const PSeg *segs, const GChunk *gc, const int *cls_w,
                       const int *gcls_begin, int ncls, const PRun *runs, const PRun *cruns,
                       const double *tab, double *worst) {
  const int n = gcls_begin[ncls];
  if (n == 0) return;
  MADAM_CUDA(cudaMemsetAsync(worst, 0, (size_t)n * sizeof(double), st));
  for (int i = 0; i < ncls; ++i) {
    const int c0 = gcls_begin[i], c1 = gcls_begin[i + 1];
    if (c1 <= c0) continue;
    const int W = cls_w[i];
    const long long nthr = (long long)(c1 - c0) * 2 * (W > 0 ? W : kRing - 1);
    const unsigned grid = (unsigned)((nthr + 63) / 64);
    unsigned long long *wb = (unsigned long long *)worst;
    switch (W) {
#define MADAM_BAND2_CASE(X)                                                                  \
  case X:                                                                                    \
    MADAM_LAUNCH(k_band2_guard_check<X>, grid, 64, 0, st, segs, gc, c0, c1, runs, cruns, tab, \
                 wb);                                                                        \
    break;
      MADAM_BAND2_CASE(1)
      MADAM_BAND2_CASE(2)
      MADAM_BAND2_CASE(4)
      MADAM_BAND2_CASE(8)
      MADAM_BAND2_CASE(9)
      MADAM_BAND2_CASE(12)
      MADAM_BAND2_CASE(16)
      MADAM_BAND2_CASE(19)
      MADAM_BAND2_CASE(24)
      MADAM_BAND2_CASE(29)
      MADAM_BAND2_CASE(32)
#undef MADAM_BAND2_CASE
      default:
        MADAM_LAUNCH(k_band2_guard_check<0>, grid, 64, 0, st, segs, gc, c0, c1, runs, cruns,
                     tab, wb);
        break;
    }
  }
}

namespace {
template <int W>
void launch_guard(cudaStream_t st, const PSeg *segs, const GChunk *gc, int c0, int c1,
                  const PRun *runs, const PRun *cruns, const double *tab, int dir,
                  const double *in, double *out, int *err) {
  static bool attr = false;
  if (!attr) {
    MADAM_CUDA(cudaFuncSetAttribute(k_band2_guard_pass<W, 0>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)GStage<W>::kSmem));
    MADAM_CUDA(cudaFuncSetAttribute(k_band2_guard_pass<W, 1>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)GStage<W>::kSmem));
    attr = true;
  }
  const unsigned grid = (unsigned)((c1 - c0 + 31) / 32);
  if (dir == 0)
    MADAM_LAUNCH((k_band2_guard_pass<W, 0>), grid, 32, GStage<W>::kSmem, st, segs, gc, c0, c1,
                 runs, cruns, tab, in, out, err);
  else
    MADAM_LAUNCH((k_band2_guard_pass<W, 1>), grid, 32, GStage<W>::kSmem, st, segs, gc, c0, c1,
                 runs, cruns, tab, in, out, err);
}
}  // namespace

void band2_solve_guarded(cudaStream_t st, const PSeg *segs, const GChunk *gc, const int *cls_w,
                         const int *gcls_begin, int ncls, const PRun *runs, const PRun *cruns,
                         const double *tab, const double *r, double *y, double *z, int *err) {
  for (int dir = 0; dir < 2; ++dir)
    for (int i = 0; i < ncls; ++i) {
      const int c0 = gcls_begin[i], c1 = gcls_begin[i + 1];
      if (c1 <= c0) continue;
      const double *in = dir == 0 ? r : y;
      double *out = dir == 0 ? y : z;
      switch (cls_w[i]) {
#define MADAM_BAND2_CASE(X) \
  case X: launch_guard<X>(st, segs, gc, c0, c1, runs, cruns, tab, dir, in, out, err); break;
        MADAM_BAND2_CASE(1)
        MADAM_BAND2_CASE(2)
        MADAM_BAND2_CASE(4)
        MADAM_BAND2_CASE(8)
        MADAM_BAND2_CASE(9)
        MADAM_BAND2_CASE(12)
        MADAM_BAND2_CASE(16)
        MADAM_BAND2_CASE(19)
        MADAM_BAND2_CASE(24)
        MADAM_BAND2_CASE(29)
        MADAM_BAND2_CASE(32)
#undef MADAM_BAND2_CASE
        default:
          fail("band2_solve_guarded: band width class without registers");
      }
    }
}

}  // namespace madam
