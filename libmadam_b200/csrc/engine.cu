// Destriping engine: setup, PCG iteration and finalisation on sm_100a.
//
// Data layout in HBM
//   pointing  float4 {w_I, w_Q, w_U, compacted pixel} per sample, [det][sample]
//             (int32 compacted pixel only, for temperature-only data)
//   signal    float64 [det][sample]
//   maps      compacted pixel space (hit submaps only), pixel-major
//             (cc / cca: 6 doubles = symmetric 3x3; maps: 3 doubles)
//   baselines float64 [det][baseline] (the reference's aa(0, k, idet) order)
// Scatter passes (map <- samples) run over "runs": maximal stretches of one
// detector's samples inside one tile of <= 1024 compacted pixels.  Runs are
// bucketed by tile, each CTA accumulates a tile in shared memory and flushes
// it with one global atomic per touched pixel value.  Gather passes
// (baselines <- samples) use one warp per baseline in time order.
#include <cub/cub.cuh>
#include <type_traits>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <tuple>
#include <omp.h>

#include "engine.h"
#include "fft.cuh"
#include "fits.h"
#include "kernels.cuh"
#include "pixmat.cuh"
#include "band2.cuh"
#include "precond.cuh"

namespace madam {

std::atomic<unsigned long long> g_kernel_launches{0};

namespace {

constexpr int kTileMax = 1024;        // pixels per scatter tile (fine res)
constexpr uint32_t kRunMax = 1024;    // samples per run
constexpr long long kItemSamples = 1 << 16;  // samples per scatter work item

enum Scal { S_RZ = 0, S_RR, S_PAP, S_RZ2, S_RZO, S_ALPHA, S_BETA, S_SHARD = 12, S_NSCAL = 16 };

__device__ __forceinline__ int find_iv(const long long *istart, int niv, long long s) {
  int lo = 0, hi = niv - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (istart[mid] <= s) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// global baseline index (det * noba_short + k) of sample s of detector det
__device__ __forceinline__ long long baseline_of(const SampleMap &m, long long det,
                                                 long long s) {
  const int iv = find_iv(m.istart, m.ninterval, s);
  return det * m.noba_short + m.kstart[iv] + m.fdn.div((uint32_t)(s - m.istart[iv]));
}

template <int NNZ>
__device__ __forceinline__ int sample_pix(const float4 *p4, const int32_t *pc, long long i) {
  if (NNZ == 3) return point_pix(p4[i]);
  return pc[i];
}

// ---------------------------------------------------------------- setup --
// samples outside [rg[2i], rg[2i+1]) of every interval i take the dummy pixel
__global__ void k_subchunk_mask(int32_t *pix, long long n, long long nsamp, const long long *rg,
                                int nrange, int dummy) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long s = i % nsamp;
    bool in = false;
    for (int r = 0; r < nrange; ++r)
      if (rg[2 * r] <= s && s < rg[2 * r + 1]) in = true;
    if (!in) pix[i] = dummy;
  }
}

__global__ void k_minmax(const int32_t *pix, long long n, int *out) {
  int mn = INT_MAX, mx = INT_MIN;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int v = pix[i];
    mn = min(mn, v);
    mx = max(mx, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(out, mn);
    atomicMax(out + 1, mx);
  }
}

// check_files: samples whose weights are all zero get pixel -1
// (read_data.f90:243-252)
__global__ void k_flag_zero_weight(int32_t *pix, const float *w, int nnz, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    bool allz = true;
    for (int j = 0; j < nnz; ++j)
      if (w[i * nnz + j] != 0.0f) allz = false;
    if (allz && !(pix[i] < 0)) pix[i] = -1;
  }
}

__global__ void k_count_good(const int32_t *pix, long long n, SampleMap sm, int niv,
                             unsigned long long *counts) {
  for (long long i0 = blockIdx.x * (long long)blockDim.x; i0 < n;
       i0 += (long long)gridDim.x * blockDim.x) {
    const long long i = i0 + threadIdx.x;
    int key = -1;
    bool good = false;
    if (i < n) {
      const long long det = i / sm.nsamp, s = i - det * sm.nsamp;
      key = (int)(det * niv + find_iv(sm.istart, sm.ninterval, s));
      good = pix[i] >= 0;
    }
    const unsigned grp = __match_any_sync(0xffffffffu, key);
    const unsigned ball = __ballot_sync(0xffffffffu, good);
    const int lane = threadIdx.x & 31;
    if (key >= 0 && lane == __ffs(grp) - 1) {
      const unsigned c = __popc(grp & ball);
      if (c) atomicAdd(counts + key, (unsigned long long)c);
    }
  }
}

// check_files: periods with less than 0.1 % good samples are flagged
// (read_data.f90:255-272)
__global__ void k_flag_sparse(int32_t *pix, long long n, SampleMap sm, int niv,
                              const unsigned long long *counts, const long long *ivlen) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long det = i / sm.nsamp, s = i - det * sm.nsamp;
    const int iv = find_iv(sm.istart, sm.ninterval, s);
    const unsigned long long c = counts[det * niv + iv];
    if (c == 0) continue;
    if ((double)c / (double)ivlen[iv] < fsp(1e-3f)) pix[i] = -1;
  }
}

// where (pixels < 0) pixels = dummy_pixel; hit-submap flags (pointing.f90:125-131)
__global__ void k_dummy_ksub(int32_t *pix, long long n, int dummy, int nosubpix, int *ksub) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    int v = pix[i];
    if (v < 0) {
      v = dummy;
      pix[i] = v;
    }
    const int sm = v / nosubpix;
    if (ksub[sm] == 0) ksub[sm] = 1;
  }
}

// reduce_pixels compaction (pointing.f90:150-156) and packing of the pointing
template <int NNZ>
__global__ void k_compact(int32_t *pix, const float *w, long long n, const int *sub1,
                          int nosubpix, float4 *p4, int32_t *pc) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int v = pix[i];
    const int c = v - sub1[v / nosubpix] * nosubpix;
    pix[i] = c;
    if (NNZ == 3) {
      p4[i] = make_float4(w[3 * i], w[3 * i + 1], w[3 * i + 2], __int_as_float(c));
    } else {
      pc[i] = c;
    }
  }
}

// per-baseline detector weight, 0 for (det, period) pairs the reference skips
__global__ void k_baseline_weights(double *bw, long long nb, long noba, const int *kstart,
                                   int niv, const double *detw_iv) {
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nb;
       b += (long long)gridDim.x * blockDim.x) {
    const long long det = b / noba, k = b - det * noba;
    int lo = 0, hi = niv - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (kstart[mid] <= k) lo = mid;
      else hi = mid - 1;
    }
    bw[b] = detw_iv[det * niv + lo];
  }
}

// flag_bad_baselines (read_data.f90:30-74): one warp per baseline
template <int NNZ>
__global__ void k_bad_baselines(int32_t *pix, float4 *p4, int32_t *pc, long long nb,
                                long noba, long long nsamp, const uint32_t *bstart,
                                int dummy_global, double frac) {
  const long long b = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (b >= nb) return;
  const long long det = b / noba, k = b - det * noba;
  const long long s0 = bstart[k], s1 = bstart[k + 1];
  int ngood = 0;
  for (long long s = s0 + lane; s < s1; s += 32)
    if (pix[det * nsamp + s] != dummy_global) ++ngood;
  ngood = warp_sum(ngood);
  const long long len = s1 - s0;
  if (ngood > 0 && ngood < frac * len) {
    for (long long s = s0 + lane; s < s1; s += 32) {
      const long long i = det * nsamp + s;
      pix[i] = dummy_global;
      if (NNZ == 3) p4[i].w = __int_as_float(dummy_global);
      else pc[i] = dummy_global;
    }
  }
}

// run boundaries: a sample is inside a run if its pixel is a real compacted
// pixel and its (det, period) is not skipped
template <int NNZ>
__global__ void k_run_flags(const float4 *p4, const int32_t *pc, long long n, SampleMap sm,
                            const double *bw, int nloc, int tile_shift, uint8_t *sflag,
                            uint8_t *eflag) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long det = i / sm.nsamp, s = i - det * sm.nsamp;
    const int iv = find_iv(sm.istart, sm.ninterval, s);
    const int px = sample_pix<NNZ>(p4, pc, i);
    const bool valid = px < nloc && bw[det * sm.noba_short + sm.kstart[iv]] != 0.0;
    uint8_t st = 0, en = 0;
    if (valid) {
      const int tile = px >> tile_shift;
      // previous sample
      if (s == 0 || s == sm.istart[iv]) {
        st = 1;
      } else {
        const int pp = sample_pix<NNZ>(p4, pc, i - 1);
        st = !(pp < nloc && (pp >> tile_shift) == tile);
      }
      const long long ivend = sm.istart[iv + 1];
      if (s + 1 == sm.nsamp || s + 1 == ivend) {
        en = 1;
      } else {
        const int pn = sample_pix<NNZ>(p4, pc, i + 1);
        en = !(pn < nloc && (pn >> tile_shift) == tile);
      }
    }
    sflag[i] = st;
    eflag[i] = en;
  }
}

__global__ void k_run_pieces(const long long *starts, const long long *ends, long long nr,
                             long long *pieces) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nr;
       r += (long long)gridDim.x * blockDim.x) {
    const long long len = ends[r] - starts[r] + 1;
    pieces[r] = (len + kRunMax - 1) / kRunMax;
  }
}

template <int NNZ>
__global__ void k_run_emit(const long long *starts, const long long *ends,
                           const long long *piece_off, long long nr, SampleMap sm,
                           const float4 *p4, const int32_t *pc, int tile_shift, Run *runs,
                           int *keys, int *lens) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < nr;
       r += (long long)gridDim.x * blockDim.x) {
    const long long a = starts[r], e = ends[r];
    long long o = piece_off[r];
    for (long long s0 = a; s0 <= e; s0 += kRunMax, ++o) {
      const uint32_t len = (uint32_t)min((long long)kRunMax, e - s0 + 1);
      const long long det = s0 / sm.nsamp, s = s0 - det * sm.nsamp;
      const int iv = find_iv(sm.istart, sm.ninterval, s);
      Run R;
      R.s_lo = (uint32_t)(s0 & 0xffffffffu);
      R.hi_len = ((uint32_t)(s0 >> 32) << 24) | len;
      R.kbase = (int32_t)(det * sm.noba_short + sm.kstart[iv]);
      R.offiv = (uint32_t)(s - sm.istart[iv]);
      runs[o] = R;
      keys[o] = sample_pix<NNZ>(p4, pc, s0) >> tile_shift;
      lens[o] = (int)len;
    }
  }
}

__global__ void k_gather_runs(const int *perm, const Run *in, const int *lens_in, long long n,
                              Run *out, int *lens_out) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    out[r] = in[perm[r]];
    lens_out[r] = lens_in[perm[r]];
  }
}

__global__ void k_item_flags(const int *keys, const long long *pref, long long n, uint8_t *f) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    f[r] = (r == 0 || keys[r] != keys[r - 1] ||
            pref[r] / kItemSamples != pref[r - 1] / kItemSamples);
  }
}

__global__ void k_item_tiles(const long long *begins, long long nitem, const int *keys,
                             int *item_begin, int *item_tile) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nitem;
       t += (long long)gridDim.x * blockDim.x) {
    item_begin[t] = (int)begins[t];
    item_tile[t] = keys[begins[t]];
  }
}

// pixel_matrix + count_hits + bin_tod (smadam_routines.f90:111-422), fused,
// shared-memory privatised per tile, at the map (fine) resolution
template <int NMAP>
__global__ void k_setup_scatter(const int *item_begin, const int *item_tile, const Run *runs,
                                const float4 *p4, const int32_t *pc, const double *tod,
                                const double *bw, FastDiv fdn, int tile_shift, double *cc,
                                double *bin, int *hits) {
  constexpr int NCC = NMAP == 3 ? 6 : 1;
  extern __shared__ double sm[];
  const int T = 1 << tile_shift;
  double *scc = sm;
  double *sbin = sm + NCC * T;
  int *shits = (int *)(sbin + NMAP * T);
  for (int e = threadIdx.x; e < NCC * T; e += blockDim.x) scc[e] = 0;
  for (int e = threadIdx.x; e < NMAP * T; e += blockDim.x) sbin[e] = 0;
  for (int e = threadIdx.x; e < T; e += blockDim.x) shits[e] = 0;
  __syncthreads();
  const int it = blockIdx.x;
  const int rb = item_begin[it], re = item_begin[it + 1];
  const int tile = item_tile[it];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int r = rb + wid; r < re; r += nw) {
    const Run R = runs[r];
    const uint64_t s0 = run_start(R);
    const uint32_t len = run_len(R);
    const double detw = bw[R.kbase];
    const double sqw = sqrt(detw);
    for (uint32_t u = lane; u < len; u += 32) {
      const uint64_t i = s0 + u;
      const double t = tod[i];
      if (NMAP == 3) {
        const float4 q = p4[i];
        const int loc = point_pix(q) & (T - 1);
        const double w0 = (double)q.x * sqw, w1 = (double)q.y * sqw, w2 = (double)q.z * sqw;
        double *c = scc + 6 * loc;
        atomicAdd(c + 0, w0 * w0);
        atomicAdd(c + 1, w0 * w1);
        atomicAdd(c + 2, w0 * w2);
        atomicAdd(c + 3, w1 * w1);
        atomicAdd(c + 4, w1 * w2);
        atomicAdd(c + 5, w2 * w2);
        double *bm = sbin + 3 * loc;
        atomicAdd(bm + 0, (double)q.x * t * detw);
        atomicAdd(bm + 1, (double)q.y * t * detw);
        atomicAdd(bm + 2, (double)q.z * t * detw);
        atomicAdd(shits + loc, 1);
      } else {
        const int loc = pc[i] & (T - 1);
        atomicAdd(scc + loc, detw);
        atomicAdd(sbin + loc, t * detw);
        atomicAdd(shits + loc, 1);
      }
    }
  }
  __syncthreads();
  const long long base = (long long)tile * T;
  for (int p = threadIdx.x; p < T; p += blockDim.x) {
    if (shits[p] == 0) continue;
    atomicAdd(hits + base + p, shits[p]);
    for (int j = 0; j < NCC; ++j) atomicAdd(cc + (base + p) * NCC + j, scc[NCC * p + j]);
    for (int j = 0; j < NMAP; ++j) atomicAdd(bin + (base + p) * NMAP + j, sbin[NMAP * p + j]);
  }
}

// collect to the cross resolution: sum groups of ndeg consecutive pixels
__global__ void k_degrade(const double *fine, double *coarse, long long ncoarse, int nv,
                          int ndeg) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ncoarse * nv;
       e += (long long)gridDim.x * blockDim.x) {
    const long long p = e / nv;
    const int j = (int)(e - p * nv);
    double s = 0;
    for (int d = 0; d < ndeg; ++d) s += fine[(p * ndeg + d) * nv + j];
    coarse[e] = s;
  }
}

template <int NMAP>
__global__ void k_invert_cross(double *cc, long long n, MatrixRules mr) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    if (NMAP == 1) {
      const double c = cc[p];
      cc[p] = (c != 0) ? 1.0 / c : 0.0;
    } else {
      double s6[6];
      for (int j = 0; j < 6; ++j) s6[j] = cc[p * 6 + j];
      invert_cross_pixel(s6, mr.pixmode, mr.pixlim, mr.allow_decoupling, mr.incomplete);
      for (int j = 0; j < 6; ++j) cc[p * 6 + j] = s6[j];
    }
  }
}

template <int NMAP>
__global__ void k_invert_map(double *cc, long long n, MatrixRules mr, int *mask, float *crit) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    if (NMAP == 1) {
      const double c = cc[p];
      if (c != 0) {
        cc[p] = 1.0 / c;
        mask[p] = 1;
      } else {
        cc[p] = 0;
        mask[p] = 0;
      }
    } else {
      double s6[6];
      for (int j = 0; j < 6; ++j) s6[j] = cc[p * 6 + j];
      float cr = 0.0f;
      mask[p] = invert_map_pixel(s6, mr.pixmode, mr.pixlim, mr.allow_decoupling, mr.incomplete,
                                 cr);
      crit[p] = cr;
      for (int j = 0; j < 6; ++j) cc[p * 6 + j] = s6[j];
    }
  }
}

// ccmultiply (map_routines.f90:24-77)
template <int NMAP>
__global__ void k_ccmult(const double *cc, double *m, long long n) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    if (NMAP == 1) {
      const double c = cc[p];
      m[p] = (c == 0) ? 0.0 : c * m[p];
    } else {
      const double *c = cc + p * 6;
      double *v = m + p * 3;
      if (c[0] == 0) {
        v[0] = v[1] = v[2] = 0;
      } else {
        const double a = v[0], b = v[1], d = v[2];
        const double tm = c[0] * a + c[1] * b + c[2] * d;
        const double qm = c[1] * a + c[3] * b + c[4] * d;
        const double um = c[2] * a + c[4] * b + c[5] * d;
        v[0] = tm;
        v[1] = qm;
        v[2] = um;
      }
    }
  }
}

// ccmultiply of the PCG (iterate_a, smadam_routines.f90:809-812) that also
// writes the copy of the map the gather reads: FP64 padded to 32 bytes a
// pixel ({I, Q}, {U, 0}: one aligned sector per lookup) or, in the FP32-TOD
// form, float32 {I, Q, U, 0} (one 16-byte load)
template <bool F32>
__global__ void k_ccmult_copy(const double *cc, double *m, long long n, double2 *mg,
                              float4 *mf) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    const double *c = cc + p * 6;
    double *v = m + p * 3;
    double tm = 0, qm = 0, um = 0;
    if (c[0] != 0) {
      const double a = v[0], b = v[1], d = v[2];
      tm = fma(c[2], d, fma(c[1], b, c[0] * a));
      qm = fma(c[4], d, fma(c[3], b, c[1] * a));
      um = fma(c[5], d, fma(c[4], b, c[2] * a));
    }
    v[0] = tm;
    v[1] = qm;
    v[2] = um;
    if (F32) {
      mf[p] = make_float4((float)tm, (float)qm, (float)um, 0.f);
    } else {
      mg[2 * p] = make_double2(tm, qm);
      mg[2 * p + 1] = make_double2(um, 0.0);
    }
  }
}

// initialize_a (smadam_routines.f90:508-653): one warp per baseline
template <int NMAP>
__global__ void k_init_a(const float4 *p4, const int32_t *pc, const double *tod,
                         const uint32_t *bstart, long long nb, long noba, long long nsamp,
                         const double *bw, const double *wamap, int deg_shift, int nloc,
                         double *yba, double *nna) {
  const long long b = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (b >= nb) return;
  const double detw = bw[b];
  if (detw == 0) return;
  const long long det = b / noba, k = b - det * noba;
  const long long i0 = det * nsamp + bstart[k], i1 = det * nsamp + bstart[k + 1];
  double y = 0, cnt = 0;
  for (long long i = i0 + lane; i < i1; i += 32) {
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
    if (NMAP == 3) {
      const double m0 = wamap[pcr * 3], m1 = wamap[pcr * 3 + 1], m2 = wamap[pcr * 3 + 2];
      if (m0 == 0 && m1 == 0 && m2 == 0) continue;
      y += tod[i] - (m0 * (double)q.x + m1 * (double)q.y + m2 * (double)q.z);
    } else {
      const double m0 = wamap[pcr];
      if (m0 == 0) continue;
      y += tod[i] - m0;
    }
    cnt += 1.0;
  }
  y = warp_sum(y);
  cnt = warp_sum(cnt);
  if (lane == 0) {
    double n = cnt * detw, yy = y * detw;
    if (fabs(n) < fsp(1e-30f)) {
      n = 0;
      yy = 0;
    }
    yba[b] = yy;
    nna[b] = n;
  }
}

// baseline_to_map (smadam_routines.f90:1074-1111) / subtract_baselines_a
// (1489-1539): target[pix] += w * pw[k], privatised per tile
template <int NMAP>
__global__ void k_scatter(const int *item_begin, const int *item_tile, const Run *runs,
                          const float4 *p4, const int32_t *pc, const double *pw, FastDiv fdn,
                          int tile_shift, int deg_shift, int tilec, double *target) {
  extern __shared__ double sacc[];
  for (int e = threadIdx.x; e < tilec * NMAP; e += blockDim.x) sacc[e] = 0;
  __syncthreads();
  const int it = blockIdx.x;
  const int rb = item_begin[it], re = item_begin[it + 1];
  const long long base_c = ((long long)item_tile[it] << tile_shift) >> deg_shift;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int r = rb + wid; r < re; r += nw) {
    const Run R = runs[r];
    const uint64_t s0 = run_start(R);
    const uint32_t len = run_len(R);
    for (uint32_t u = lane; u < len; u += 32) {
      const uint64_t i = s0 + u;
      const double v = pw[R.kbase + fdn.div(R.offiv + u)];
      if (NMAP == 3) {
        const float4 q = p4[i];
        const int loc = (int)((point_pix(q) >> deg_shift) - base_c);
        atomicAdd(sacc + 3 * loc + 0, (double)q.x * v);
        atomicAdd(sacc + 3 * loc + 1, (double)q.y * v);
        atomicAdd(sacc + 3 * loc + 2, (double)q.z * v);
      } else {
        const int loc = (int)((pc[i] >> deg_shift) - base_c);
        atomicAdd(sacc + loc, v);
      }
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < tilec * NMAP; e += blockDim.x) {
    const double v = sacc[e];
    if (v != 0) atomicAdd(target + base_c * NMAP + e, v);
  }
}

// map_to_baseline (smadam_routines.f90:1282-1329) + "ap = ap + ..." (870)
// and the partial p.ap of the PCG (877): one warp per baseline
template <int NMAP>
__global__ void k_gather(const float4 *p4, const int32_t *pc, const uint32_t *bstart,
                         long long nb, long noba, long long nsamp, const double *bw,
                         const double *p, const double *nna, const double *m, int deg_shift,
                         int nloc, const uint8_t *rmask, double *ap, double *part) {
  const int lane = threadIdx.x & 31;
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  double pap = 0;
  for (long long b = warp0; b < nb; b += nwarps) {
    const double detw = bw[b];
    if (detw != 0) {
      const long long det = b / noba, k = b - det * noba;
      const long long i0 = det * nsamp + bstart[k], i1 = det * nsamp + bstart[k + 1];
      double apn = 0;
      for (long long i = i0 + lane; i < i1; i += 32) {
        if (NMAP == 3) {
          const float4 q = p4[i];
          const int px = point_pix(q);
          if (px >= nloc) continue;
          const double *mm = m + (long long)(px >> deg_shift) * 3;
          apn += (double)q.x * mm[0] + (double)q.y * mm[1] + (double)q.z * mm[2];
        } else {
          const int px = pc[i];
          if (px >= nloc) continue;
          apn += m[px >> deg_shift];
        }
      }
      apn = warp_sum(apn);
      if (lane == 0) {
        const double v = ap[b] + (nna[b] * p[b] - apn * detw);
        ap[b] = v;
        if (rmask[b]) pap += p[b] * v;
      }
    } else if (lane == 0 && rmask[b]) {
      pap += p[b] * ap[b];
    }
  }
  double v[1] = {pap};
  block_sum<1>(v);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// map_to_baseline, block-tiled: a CTA takes `kb` consecutive baselines of one
// detector (<= kGatherTile samples), streams their samples once (coalesced
// float4 loads, four independent loads in flight per thread), stages w.m per
// sample in shared memory and sums each baseline with one warp.  Used when
// every baseline is at most kGatherTile / 2 samples long.
constexpr int kGatherTile = 2048;
// k_gather_chunks: resident CTAs per SM (its register budget) and a grid of
// exactly one wave of them
constexpr int kGatherChunkBlocksPerSM = 4;
constexpr int kGatherChunkBlocks = 148 * kGatherChunkBlocksPerSM;
constexpr int kGatherUnroll = 4;
constexpr int kScatterUnroll = 8;

template <int NMAP>
__device__ __forceinline__ double wm_sample(const float4 *__restrict__ p4,
                                            const int32_t *__restrict__ pc,
                                            const double *__restrict__ m, long long i,
                                            int deg_shift, int nloc) {
  if (NMAP == 3) {
    const float4 q = __ldcs(p4 + i);
    const int px = point_pix(q);
    if (px >= nloc) return 0.0;
    const double *mm = m + (long long)(px >> deg_shift) * 3;
    return (double)q.x * mm[0] + (double)q.y * mm[1] + (double)q.z * mm[2];
  } else {
    const int px = __ldcs(pc + i);
    if (px >= nloc) return 0.0;
    return m[px >> deg_shift];
  }
}


template <int NMAP>
__global__ void __launch_bounds__(256) k_gather_tiled(
    const float4 *__restrict__ p4, const int32_t *__restrict__ pc,
    const uint32_t *__restrict__ bstart, long noba, long long nsamp, int kb,
    long long ntiles_det, int ndet, const double *__restrict__ bw, const double *__restrict__ p,
    const double *__restrict__ nna, const double *__restrict__ m, int deg_shift, int nloc,
    const uint8_t *__restrict__ rmask, double *__restrict__ ap, double *__restrict__ part) {
  __shared__ double vals[kGatherTile];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double pap = 0;
  const long long ntiles = ntiles_det * ndet;
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const long long det = t / ntiles_det;
    const long long k0 = (t - det * ntiles_det) * kb;
    const long long k1 = min(k0 + kb, (long long)noba);
    const int s0 = (int)bstart[k0], ns = (int)(bstart[k1] - bstart[k0]);
    const long long base = det * nsamp + s0;
    for (int u0 = threadIdx.x; u0 < ns; u0 += kGatherUnroll * blockDim.x) {
      double v[kGatherUnroll];
#pragma unroll
      for (int r = 0; r < kGatherUnroll; ++r) {
        const int u = u0 + r * blockDim.x;
        v[r] = u < ns ? wm_sample<NMAP>(p4, pc, m, base + u, deg_shift, nloc) : 0.0;
      }
#pragma unroll
      for (int r = 0; r < kGatherUnroll; ++r) {
        const int u = u0 + r * blockDim.x;
        if (u < ns) vals[u] = v[r];
      }
    }
    __syncthreads();
    for (long long k = k0 + wid; k < k1; k += nw) {
      const long long b = det * noba + k;
      const double detw = bw[b];
      if (detw == 0) {
        if (lane == 0 && rmask[b]) pap += p[b] * ap[b];
        continue;
      }
      const int a0 = (int)(bstart[k] - s0), a1 = (int)(bstart[k + 1] - s0);
      double apn = 0;
      for (int i = a0 + lane; i < a1; i += 32) apn += vals[i];
      apn = warp_sum(apn);
      if (lane == 0) {
        const double v = ap[b] + (nna[b] * p[b] - apn * detw);
        ap[b] = v;
        if (rmask[b]) pap += p[b] * v;
      }
    }
    __syncthreads();
  }
  double v[1] = {pap};
  block_sum<1>(v);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

// w . m with the pixel's (T, Q, U, pad) fetched by one 256-bit load (sm_100):
// one L1 wavefront per lane instead of two for the random map lookups; the
// padded copy is 32-byte aligned (k_ccmult_copy) and read-only here
__device__ __forceinline__ double map_dot(const double2 *__restrict__ mg, long long cp,
                                          const float4 &q) {
  double t, qq, u, pad;
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(t), "=d"(qq), "=d"(u), "=d"(pad)
      : "l"(mg + 2 * cp));
  (void)pad;
  return fma((double)q.z, u, fma((double)q.y, qq, (double)q.x * t));
}
__device__ __forceinline__ double map_dot(const float4 *__restrict__ mf, long long cp,
                                          const float4 &q) {
  const float4 a = __ldg(mf + cp);
  return fma((double)q.z, (double)a.z, fma((double)q.y, (double)a.y, (double)q.x * a.x));
}

// Per-baseline sums of a warp chunk of at most kGatherChunk staged values
// (map_to_baseline's inner sum, smadam_routines.f90:1018-1032, for up to 32
// consecutive baselines at once), for chunks of few long baselines.  vb
// holds the chunk's values in time order with entry i at vb[i + i / 8]
// (entries n..255 are zero); baseline j < nbl owns entries [a0, a1) (lane
// j's arguments).  Lane L adds entries 8L..8L+7 in order; a segmented warp
// scan joins the parts of a baseline that spans lanes.  bsum[j] receives
// baseline j's sum (0 when empty).  The padding keeps both the strided
// staging writes and these lane-contiguous reads free of bank conflicts.
// Where a chunk holds a few long baselines this replaces up to 256 serial
// shared-memory reads by one or two lanes with 8 reads by every lane.
struct ChunkSmem {
  double bsum[32];
  unsigned heads[8];        // bit e: entry e starts a nonempty baseline
  unsigned char ord2b[32];  // k-th nonempty baseline -> its lane
};

__device__ __forceinline__ void chunk_baseline_sums(const double *vb, int nbl, int a0, int a1,
                                                    ChunkSmem &cs, int lane) {
  const unsigned full = 0xffffffffu;
  cs.bsum[lane] = 0.0;
  if (lane < 8) cs.heads[lane] = 0u;
  __syncwarp();
  const bool ne = lane < nbl && a1 > a0;
  const unsigned nem = __ballot_sync(full, ne);
  if (ne) {
    cs.ord2b[__popc(nem & ((1u << lane) - 1u))] = (unsigned char)lane;
    atomicOr(&cs.heads[a0 >> 5], 1u << (a0 & 31));
  }
  __syncwarp();
  const int wl = lane >> 2, sh = (lane & 3) * 8;
  int cnt = 0;  // heads before entry 8L
#pragma unroll
  for (int w = 0; w < 8; ++w) {
    const unsigned x = cs.heads[w];
    if (w < wl) cnt += __popc(x);
    else if (w == wl) cnt += __popc(x & ((1u << sh) - 1u));
  }
  const unsigned bits = (cs.heads[wl] >> sh) & 0xffu;
  const int nh0 = cnt;
  double w[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) w[r] = vb[9 * lane + r];
  double run = 0.0, first = 0.0;
  bool seen = false;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    if ((bits >> r) & 1u) {
      if (!seen) {
        first = run;
        seen = true;
      } else {
        cs.bsum[cs.ord2b[cnt - 1]] = run;
      }
      run = 0.0;
      ++cnt;
    }
    run += w[r];
  }
  // segmented inclusive scan of (run, seen) over the lanes, left to right
  double sc = run;
  int fl = seen ? 1 : 0;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const double so = __shfl_up_sync(full, sc, d);
    const int fo = __shfl_up_sync(full, fl, d);
    if (lane >= d) {
      if (!fl) sc = so + sc;
      fl |= fo;
    }
  }
  const double carry = __shfl_up_sync(full, sc, 1);
  if (seen && nh0 > 0) cs.bsum[cs.ord2b[nh0 - 1]] = carry + first;
  if (lane == 31 && cnt > 0) cs.bsum[cs.ord2b[cnt - 1]] = sc;
  __syncwarp();
}

// map_to_baseline, warp chunks: a warp takes a chunk of consecutive
// baselines of one detector (at most kGatherChunk samples, at most 32
// baselines), loads all of its samples (8 per lane, coalesced) with their map
// values in flight together, stages w.m in the warp's shared-memory slice and
// lets lane j sum baseline j in time order; fused with the p.ap partial sums.
// No block barriers: warps run independently.  Used when every baseline is
// at most kGatherChunk samples long.
constexpr int kGatherChunk = 256;
static_assert(kGatherChunk == 256, "chunk_baseline_sums takes 8 entries a lane");

// MAPT (NMAP = 3): the map copy it reads, double2 (padded FP64, two 16-byte
// loads in one sector) or float4 (FP32-TOD form, one load).
template <int NMAP, class MAPT>
__global__ void __launch_bounds__(256, kGatherChunkBlocksPerSM) k_gather_chunks(
    const int2 *__restrict__ chunks, long long nchunks, const float4 *__restrict__ p4,
    const int32_t *__restrict__ pc, const uint32_t *__restrict__ bstart, long noba,
    long long nsamp, const double *__restrict__ bw, const double *__restrict__ p,
    const double *__restrict__ nna, const double *__restrict__ m, const MAPT *__restrict__ mx,
    int deg_shift, int nloc, const uint8_t *__restrict__ rmask, double *__restrict__ ap,
    double *__restrict__ part) {
  __shared__ double vbuf[8][kGatherChunk];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double *vb = vbuf[wid];
  const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  constexpr int U = kGatherChunk / 32;
  double pap = 0;
  for (long long c = w0; c < nchunks; c += nwarps) {
    const int2 ck = chunks[c];  // {first global baseline, baselines}
    const long long det = ck.x / noba, k0 = ck.x - det * noba;
    const int s0 = (int)bstart[k0];
    const int n = (int)(bstart[k0 + ck.y] - s0);
    const long long base = det * nsamp + s0;
    // lane j < ck.y: scalars of baseline j, in flight with the samples
    double detw = 0, pb = 0, apb = 0, npb = 0;
    int a0 = 0, a1 = 0;
    bool rm = false;
    if (lane < ck.y) {
      const long long b = ck.x + lane;
      detw = bw[b];
      pb = p[b];
      apb = ap[b];
      npb = nna[b] * pb;
      rm = rmask[b] != 0;
      a0 = (int)(bstart[k0 + lane] - s0);
      a1 = (int)(bstart[k0 + lane + 1] - s0);
    }
    double v[U];
    if (NMAP == 3) {
      float4 q[U];
#pragma unroll
      for (int r = 0; r < U; ++r) {
        const int i = r * 32 + lane;
        q[r] = i < n ? __ldcs(p4 + base + i) : make_float4(0.f, 0.f, 0.f, __int_as_float(nloc));
      }
#pragma unroll
      for (int r = 0; r < U; ++r) {
        const int px = point_pix(q[r]);
        v[r] = 0.0;
        if (px < nloc) v[r] = map_dot(mx, px >> deg_shift, q[r]);
      }
    } else {
      int px[U];
#pragma unroll
      for (int r = 0; r < U; ++r) {
        const int i = r * 32 + lane;
        px[r] = i < n ? __ldcs(pc + base + i) : nloc;
      }
#pragma unroll
      for (int r = 0; r < U; ++r) v[r] = px[r] < nloc ? m[px[r] >> deg_shift] : 0.0;
    }
#pragma unroll
    for (int r = 0; r < U; ++r) vb[r * 32 + lane] = v[r];
    __syncwarp();
    if (lane < ck.y) {
      const long long b = ck.x + lane;
      if (detw == 0) {
        if (rm) pap += pb * apb;
      } else {
        double apn = 0;
        for (int i = a0; i < a1; ++i) apn += vb[i];
        const double val = apb + fma(-apn, detw, npb);
        ap[b] = val;
        if (rm) pap += pb * val;
      }
    }
    __syncwarp();
  }
  double pv[1] = {pap};
  block_sum<1>(pv);
  if (threadIdx.x == 0) part[blockIdx.x] = pv[0];
}

// baseline_to_map (smadam_routines.f90:1074-1111) as a pixel-major gather:
// the pointing is also stored sorted by cross pixel (time order inside a
// pixel) as {w_I, w_Q, w_U, global baseline}.  Each pixel's entries are cut
// into fixed chunks of at most kScatterChunk; one warp sums a chunk with all
// of its entry and pw loads in flight (8 per lane).  A pixel of one chunk is
// written directly; the chunk sums of larger pixels go to `partial` and
// k_scatter_combine adds them in chunk order.  No atomics, deterministic.
constexpr int kScatterChunk = 256;

template <int NMAP>
__global__ void __launch_bounds__(256) k_scatter_chunks(
    const int4 *__restrict__ chunks, long long nchunks, const float4 *__restrict__ sp4,
    const int2 *__restrict__ sp2, const double *__restrict__ pw, double *__restrict__ target,
    double *__restrict__ partial) {
  const int lane = threadIdx.x & 31;
  const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  constexpr int U = kScatterChunk / 32;
  for (long long c = w0; c < nchunks; c += nwarps) {
    const int4 ck = chunks[c];  // {pixel, first entry, entries, partial slot or -1}
    double a0 = 0, a1 = 0, a2 = 0;
    if (NMAP == 3) {
      float4 q[U];
#pragma unroll
      for (int r = 0; r < U; ++r) {
        const int i = r * 32 + lane;
        q[r] = i < ck.z ? __ldcs(sp4 + ck.y + i) : make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
      }
      double wv[U];
#pragma unroll
      for (int r = 0; r < U; ++r) {
        const int k = __float_as_int(q[r].w);
        wv[r] = k >= 0 ? pw[k] : 0.0;
      }
#pragma unroll
      for (int r = 0; r < U; ++r) {
        a0 = fma((double)q[r].x, wv[r], a0);
        a1 = fma((double)q[r].y, wv[r], a1);
        a2 = fma((double)q[r].z, wv[r], a2);
      }
    } else {
      int k[U];
#pragma unroll
      for (int r = 0; r < U; ++r) {
        const int i = r * 32 + lane;
        k[r] = i < ck.z ? __ldcs(&sp2[ck.y + i].x) : -1;
      }
#pragma unroll
      for (int r = 0; r < U; ++r) a0 += k[r] >= 0 ? pw[k[r]] : 0.0;
    }
    a0 = warp_sum(a0);
    if (NMAP == 3) {
      a1 = warp_sum(a1);
      a2 = warp_sum(a2);
    }
    if (lane == 0) {
      double *o = ck.w < 0 ? target + (long long)ck.x * NMAP : partial + (long long)ck.w * NMAP;
      o[0] = a0;
      if (NMAP == 3) {
        o[1] = a1;
        o[2] = a2;
      }
    }
  }
}

// multi-chunk pixels: {pixel, first partial slot, chunks}
template <int NMAP>
__global__ void k_scatter_combine(const int4 *__restrict__ multi, int nmulti,
                                  const double *__restrict__ partial, double *__restrict__ target) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nmulti; i += gridDim.x * blockDim.x) {
    const int4 mp = multi[i];
    double a[3] = {0, 0, 0};
    for (int c = 0; c < mp.z; ++c)
      for (int j = 0; j < NMAP; ++j) a[j] += partial[(long long)(mp.y + c) * NMAP + j];
    for (int j = 0; j < NMAP; ++j) target[(long long)mp.x * NMAP + j] = a[j];
  }
}

// CSR construction: sort key (cross pixel, or nloc_cross for samples the
// scatter skips) for every sample
template <int NNZ>
__global__ void k_csr_keys(const float4 *p4, const int32_t *pc, long long n, SampleMap sm,
                           const double *bw, int nloc, int deg_shift, int sentinel, int *keys,
                           uint32_t *vals, unsigned long long *nvalid) {
  for (long long i0 = blockIdx.x * (long long)blockDim.x; i0 < n;
       i0 += (long long)gridDim.x * blockDim.x) {
    const long long i = i0 + threadIdx.x;
    bool valid = false;
    if (i < n) {
      const long long det = i / sm.nsamp, s = i - det * sm.nsamp;
      const int px = sample_pix<NNZ>(p4, pc, i);
      const long long b = baseline_of(sm, det, s);
      valid = px < nloc && bw[b] != 0.0;
      keys[i] = valid ? (px >> deg_shift) : sentinel;
      vals[i] = (uint32_t)i;
    }
    const unsigned ball = __ballot_sync(0xffffffffu, valid);
    if ((threadIdx.x & 31) == 0 && ball) atomicAdd(nvalid, (unsigned long long)__popc(ball));
  }
}

template <int NNZ>
__global__ void k_csr_fill(const int *keys, const uint32_t *idx, long long nvalid,
                           const float4 *p4, SampleMap sm, float4 *sp4, int2 *sp2, int *off) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nvalid;
       i += (long long)gridDim.x * blockDim.x) {
    const long long src = idx[i];
    const long long det = src / sm.nsamp, s = src - det * sm.nsamp;
    const int b = (int)baseline_of(sm, det, s);
    if (NNZ == 3) {
      const float4 q = p4[src];
      sp4[i] = make_float4(q.x, q.y, q.z, __int_as_float(b));
    } else {
      sp2[i] = make_int2(b, 0);
    }
    const int key = keys[i];
    const int prev = i == 0 ? -1 : keys[i - 1];
    for (int p = prev + 1; p <= key; ++p) off[p] = (int)i;
  }
}

// dst[i] = src[idx[i]]
__global__ void k_take(const double *src, const uint32_t *idx, long long n, double *dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = src[idx[i]];
}

__global__ void k_fill_int(int *a, long long n, int v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    a[i] = v;
}

// ------------------------------------------------------- filter spectra --
// The noise filter's spectra (build_filter, noise_routines.f90:367-739) on
// the device: one thread per (PSD, frequency bin i < nof/2 + 1).  A PSD's
// table is its frequencies and values with their logarithms (taken on the
// host, as interpolate_psd takes them), `first` its first nonzero frequency.
struct FiltTask {
  int off, nin, first;
  double plateau;  // white-noise level subtracted from the spectrum
  double sigma;    // the detector's sigma before this filter (the inversion cut)
};

// interpolate_psd (noise_routines.f90:130-190) at one target: the bracket is
// where the reference's monotone walk over ascending targets ends, i.e. the
// last index j in [first, nin - 2] below which every frequency past `first`
// is under the target (found by bisection: the frequencies are ascending).
// The arithmetic is the host's, operation by operation; log and exp are
// CUDA's.
__device__ __forceinline__ double filt_interp(const FiltTask &T, const double *fr,
                                              const double *ps, const double *lf,
                                              const double *lp, double target) {
  if (target == 0) return 0.0;
  const double flog = log(target);
  const int nin = T.nin;
  int j = T.first;
  if (j < nin - 2) {
    // smallest k in [first + 1, nin - 2] with lf[k] >= flog; j = k - 1
    int lo = j + 1, hi = nin - 2;
    if (lf[T.off + hi] < flog) {
      j = nin - 2;
    } else {
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (lf[T.off + mid] < flog) lo = mid + 1;
        else hi = mid;
      }
      j = lo - 1;
    }
  }
  const double p0 = ps[T.off + j], p1 = ps[T.off + j + 1];
  if (p0 > 0 && p1 > 0) {
    const double l0 = lf[T.off + j], l1 = lf[T.off + j + 1];
    const double r = __ddiv_rn(__dsub_rn(flog, l0), __dsub_rn(l1, l0));
    return exp(__dadd_rn(__dmul_rn(lp[T.off + j], __dsub_rn(1.0, r)),
                         __dmul_rn(lp[T.off + j + 1], r)));
  }
  const double f0 = fr[T.off + j], f1 = fr[T.off + j + 1];
  const double r = __ddiv_rn(__dsub_rn(target, f0), __dsub_rn(f1, f0));
  return __dadd_rn(__dmul_rn(p0, __dsub_rn(1.0, r)), __dmul_rn(p1, r));
}

// One aliased term of bin j at alias k: spectrum minus the plateau (or its
// margin-th part), times the sinc^2 window.  Sets bit 0 of *flag for a
// spectrum value that is not positive (the reference then fills it from its
// neighbours, which the host does).
__device__ __forceinline__ double filt_term(const FiltTask &T, const double *fr, const double *ps,
                                            const double *lf, const double *lp, int k, long j,
                                            long nof, double fa, double margin, int *flag) {
  const double f = __dadd_rn(__dmul_rn((double)k, fa), __ddiv_rn(__dmul_rn((double)j, fa),
                                                                 (double)nof));
  double sp = filt_interp(T, fr, ps, lf, lp, f);
  sp = (sp > __dmul_rn(T.plateau, __dadd_rn(1.0, margin))) ? __dsub_rn(sp, T.plateau)
                                                           : __dmul_rn(sp, margin);
  if (k == 0 && j == 0) sp = 0.0;  // f[0] == 0: the mean carries no noise
  else if (sp <= 0) atomicOr(flag, 1);
  const double kPi = 3.141592653589793238462643383279502884197;
  const double x = __ddiv_rn(__dmul_rn(kPi, f), fa);
  const double sx = sin(x);
  const double g = (x < (double)1e-30f) ? 1.0 : __ddiv_rn(__dmul_rn(sx, sx), __dmul_rn(x, x));
  return __dmul_rn(sp, g);
}

__global__ void k_filter_spectra(const FiltTask *tasks, const double *fr, const double *ps,
                                 const double *lf, const double *lp, long nof, long nh, double fa,
                                 double margin, double *fcov, int *flag) {
  const FiltTask T = tasks[blockIdx.y];
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nh;
       i += (long)gridDim.x * blockDim.x) {
    double a = 0.0;
    for (int k = 0; k <= 2; ++k) {
      if (i == 0) {
        const double t0 = filt_term(T, fr, ps, lf, lp, k, 0, nof, fa, margin, flag);
        // aspec[0] = spec[0] at k = 0, then += 2 spec[0] g[0]; t0 = spec * g
        // with g[0] = 1 at k = 0
        a = (k == 0) ? t0 : __dadd_rn(a, __dmul_rn(2.0, t0));
      } else {
        const double t1 = filt_term(T, fr, ps, lf, lp, k, i, nof, fa, margin, flag);
        const double t2 = filt_term(T, fr, ps, lf, lp, k, nof - i, nof, fa, margin, flag);
        a = __dadd_rn(__dadd_rn(a, t1), t2);
      }
    }
    double v = (fabs(a) > __dmul_rn(T.sigma, (double)1e-30f)) ? __ddiv_rn(1.0, __dmul_rn(fa, a))
                                                               : 0.0;
    if (i == 0) v = 0.0;
    if (isnan(v)) atomicOr(flag, 2);
    fcov[(long)blockIdx.y * nh + i] = v;
  }
}

// The Fourier-domain preconditioner 1 / (nshort w + fcov) per PSD and bin
// (construct_preconditioner, noise_routines.f90:920-1153).
__global__ void k_fprec(const double *fcov, const double *w, long nh, long npsd, double nshort,
                        double *fp) {
  const long n = nh * npsd;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    fp[i] = __ddiv_rn(1.0, __dadd_rn(__dmul_rn(nshort, w[i / nh]), fcov[i]));
}

// Power of each PSD's inverse-covariance kernel, summed in the host's order
// (construct_preconditioner, noise_routines.f90:1039-1060): ptot =
// sum_{k < nof/2} icv_k^2 and the running sums pre[k] = sum_{k' <= k}
// icv_k'^2 for k < W, from which the band width is chosen.  One CTA per PSD:
// the other warps stage the squares of the next 2048 values in shared
// memory while thread 0 adds the current ones one after the other (the
// additions stay sequential, so the sums are the host's to the bit).
constexpr int kPowTile = 2048;
__global__ void __launch_bounds__(256) k_invcov_power(const double *icv, long nof, long W,
                                                      double *ptot, double *pre) {
  __shared__ double sq[2][kPowTile];
  const long ip = blockIdx.x;
  const double *c = icv + ip * nof;
  const long nsum = nof / 2, nk = max(nsum, W);
  const long ntile = (nk + kPowTile - 1) / kPowTile;
  auto stage = [&](long t, int buf, int t0, int stride) {
    for (int i = t0; i < kPowTile; i += stride) {
      const long k = t * kPowTile + i;
      sq[buf][i] = k < nk ? __dmul_rn(c[k], c[k]) : 0.0;
    }
  };
  stage(0, 0, threadIdx.x, blockDim.x);
  __syncthreads();
  double s = 0.0;
  for (long t = 0; t < ntile; ++t) {
    const int buf = (int)(t & 1);
    if (threadIdx.x >= 32) {
      if (t + 1 < ntile) stage(t + 1, buf ^ 1, threadIdx.x - 32, blockDim.x - 32);
    } else if (threadIdx.x == 0) {
      const long k0 = t * kPowTile;
      const int m = (int)min((long)kPowTile, nk - k0);
      for (int i = 0; i < m; ++i) {
        s = __dadd_rn(s, sq[buf][i]);
        const long k = k0 + i;
        if (k < W) pre[ip * W + k] = s;
        if (k == nsum - 1) ptot[ip] = s;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && nsum == 0) ptot[ip] = 0.0;
}

__global__ void k_iota(int *a, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    a[i] = (int)i;
}

// Scatter chunks of the pixel-sorted pointing: pixel p's entries
// off[p]..off[p+1] cut into ceil(n / K) chunks (one for an empty pixel).
// Pass 0 counts per pixel (chunks, partial-sum slots: the chunks of a pixel
// cut in several, pixels cut in several); pass 1 writes the chunks
// (pixel, first entry, count, slot or -1) and the multi-chunk pixels (pixel,
// first slot, chunks, 0) at the exclusive prefix sums of those counts.
__global__ void k_scatter_chunk_count(const int *off, int npix, int K, int *nck, int *nslot,
                                      int *nmulti) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
    const int n = off[p + 1] - off[p];
    const int nc = max(1, (n + K - 1) / K);
    nck[p] = nc;
    nslot[p] = nc > 1 ? nc : 0;
    nmulti[p] = nc > 1 ? 1 : 0;
  }
}

__global__ void k_scatter_chunk_fill(const int *off, int npix, int K, const int *ck_off,
                                     const int *slot_off, const int *multi_off, int4 *ck,
                                     int4 *multi) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
    const int e0 = off[p], n = off[p + 1] - off[p];
    const int nc = max(1, (n + K - 1) / K);
    const int c0 = ck_off[p];
    if (nc == 1) {
      ck[c0] = make_int4(p, e0, n, -1);
      continue;
    }
    const int s0 = slot_off[p];
    multi[multi_off[p]] = make_int4(p, s0, nc, 0);
    for (int c = 0; c < nc; ++c)
      ck[c0 + c] = make_int4(p, e0 + c * K, min(K, n - c * K), s0 + c);
  }
}

// masked dot products sum_i mask_i a_i b_i for up to 3 pairs
__global__ void k_dots(const double *a0, const double *b0, const double *a1, const double *b1,
                       const double *a2, const double *b2, int nd, const uint8_t *mask,
                       long long n, double *part) {
  double v[3] = {0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (!mask[i]) continue;
    v[0] += a0[i] * b0[i];
    if (nd > 1) v[1] += a1[i] * b1[i];
    if (nd > 2) v[2] += a2[i] * b2[i];
  }
  block_sum<3>(v);
  if (threadIdx.x == 0)
    for (int j = 0; j < 3; ++j) part[j * gridDim.x + blockIdx.x] = v[j];
}

// deterministic final sums; mode 0: scal[slots] = sums
// mode 1 (pap): scal[S_PAP] = s0, scal[S_ALPHA] = rz / pap
// mode 2 (rz, rz2, rr): rzo = rz, then beta = (rz - rz2) / rzo
__global__ void k_finish(const double *part, int nblk, int nd, double *scal, int mode,
                         int slot0) {
  double v[3] = {0, 0, 0};
  for (int j = 0; j < nd; ++j)
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) v[j] += part[j * nblk + i];
  block_sum<3>(v);
  if (threadIdx.x != 0) return;
  if (mode == 0) {
    for (int j = 0; j < nd; ++j) scal[slot0 + j] = v[j];
  } else if (mode == 1) {
    scal[S_PAP] = v[0];
    scal[S_ALPHA] = scal[S_RZ] / v[0];
  } else {
    // mode 2: a new residual; mode 3: the same step's residual replaced (a
    // reliable update), so rz of the previous step stays where it is
    if (mode == 2) scal[S_RZO] = scal[S_RZ];
    scal[S_RZ] = v[0];
    scal[S_RZ2] = v[1];
    scal[S_RR] = v[2];
    scal[S_BETA] = (v[0] - v[1]) / scal[S_RZO];
  }
}

// device copy of a pinned (page-locked, device-mapped) host buffer read
// over the bus by the SMs, so that the copy engine stays free for the
// setup's small transfers; 16-byte loads, four in flight per thread
__global__ void __launch_bounds__(256) k_fetch_host(const double *src, double *dst,
                                                    long long n) {
  const long long n2 = n / 2;
  const double2 *s2 = (const double2 *)src;
  double2 *d2 = (double2 *)dst;
  const long long stride = (long long)gridDim.x * blockDim.x;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (; i + 3 * stride < n2; i += 4 * stride) {
    const double2 a = s2[i], b = s2[i + stride], c = s2[i + 2 * stride], d = s2[i + 3 * stride];
    d2[i] = a;
    d2[i + stride] = b;
    d2[i + 2 * stride] = c;
    d2[i + 3 * stride] = d;
  }
  for (; i < n2; i += stride) d2[i] = s2[i];
  if (blockIdx.x == 0 && threadIdx.x == 0 && (n & 1)) dst[n - 1] = src[n - 1];
}

// zero the cross-resolution pixel matrices of the pixels the input mask drops
__global__ void k_apply_inmask(double *cca, long long n, int ncc, const uint8_t *mask) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x)
    if (!mask[p])
      for (int j = 0; j < ncc; ++j) cca[p * ncc + j] = 0.0;
}

// k_finish's CG scalars from inner products already summed over the ranks
// of a sharded run (scal[src .. src + 2])
__global__ void k_finish_apply(double *scal, int mode, int src) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double v0 = scal[src], v1 = scal[src + 1], v2 = scal[src + 2];
  if (mode == 1) {
    scal[S_PAP] = v0;
    scal[S_ALPHA] = scal[S_RZ] / v0;
  } else {
    if (mode == 2) scal[S_RZO] = scal[S_RZ];
    scal[S_RZ] = v0;
    scal[S_RZ2] = v1;
    scal[S_RR] = v2;
    scal[S_BETA] = (v0 - v1) / scal[S_RZO];
  }
}

// aa += alpha p; ro = r; r -= alpha ap (smadam_routines.f90:882-889)
__global__ void k_update_ar(double *aa, double *r, double *ro, const double *p, const double *ap,
                            long long n, const double *scal) {
  const double alpha = scal[S_ALPHA];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    aa[i] = aa[i] + alpha * p[i];
    const double ri = r[i];
    ro[i] = ri;
    r[i] = ri - alpha * ap[i];
  }
}

// p = z + beta p (922); pw = p * detw for the next scatter
__global__ void k_update_p(double *p, const double *z, double *pw, const double *bw, long long n,
                           const double *scal, int first) {
  const double beta = first ? 0.0 : scal[S_BETA];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = first ? z[i] : z[i] + beta * p[i];
    p[i] = v;
    pw[i] = v * bw[i];
  }
}

__global__ void k_scale_neg(const double *a, const double *bw, double *out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = -(a[i] * bw[i]);
}

// ---------------------------------------------------- serving stepper --
// The vector algebra of several PCG jobs in one launch each (grid.y: job);
// per job the arithmetic of k_update_ar, k_dots + k_finish (mode 2) and
// k_update_p.
__global__ void k_pcg_update_ar_j(const PcgJob *tab) {
  const PcgJob j = tab[blockIdx.y];
  if (!j.active) return;
  const double alpha = j.scal[S_ALPHA];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < j.nb;
       i += (long long)gridDim.x * blockDim.x) {
    j.aa[i] = j.aa[i] + alpha * j.p[i];
    const double ri = j.r[i];
    j.ro[i] = ri;
    j.r[i] = ri - alpha * j.ap[i];
  }
}

__global__ void k_pcg_dots_j(const PcgJob *tab) {
  const PcgJob j = tab[blockIdx.y];
  if (!j.active) return;
  double v[3] = {0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < j.nb;
       i += (long long)gridDim.x * blockDim.x) {
    if (!j.rmask[i]) continue;
    v[0] += j.r[i] * j.z[i];
    v[1] += j.ro[i] * j.z[i];
    v[2] += j.r[i] * j.r[i];
  }
  block_sum<3>(v);
  if (threadIdx.x == 0)
    for (int q = 0; q < 3; ++q) j.part[q * gridDim.x + blockIdx.x] = v[q];
}

__global__ void k_pcg_finish_j(const PcgJob *tab, int nblk, double *out) {
  const PcgJob j = tab[blockIdx.x];
  if (!j.active) return;
  double v[3] = {0, 0, 0};
  for (int q = 0; q < 3; ++q)
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) v[q] += j.part[q * nblk + i];
  block_sum<3>(v);
  if (threadIdx.x != 0) return;
  double *sc = j.scal;
  sc[S_RZO] = sc[S_RZ];
  sc[S_RZ] = v[0];
  sc[S_RZ2] = v[1];
  sc[S_RR] = v[2];
  sc[S_BETA] = (v[0] - v[1]) / sc[S_RZO];
  out[2 * blockIdx.x] = v[0];
  out[2 * blockIdx.x + 1] = v[2];
}

__global__ void k_pcg_update_p_j(const PcgJob *tab) {
  const PcgJob j = tab[blockIdx.y];
  if (!j.active) return;
  const double beta = j.scal[S_BETA];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < j.nb;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = j.z[i] + beta * j.p[i];
    j.p[i] = v;
    j.pw[i] = v * j.bw[i];
  }
}

// NaN count of n values (checknan diagnostics)
template <typename T>
__global__ void k_count_nan(const T *v, long long n, unsigned long long *out) {
  unsigned long long c = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    c += isnan(v[i]) ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

// r = b - ax (the true residual of a reliable update)
__global__ void k_residual(double *r, const double *b, const double *ax, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    r[i] = b[i] - ax[i];
}

__global__ void k_mul(double *z, const double *r, const double *d, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    z[i] = r[i] * d[i];
}

__global__ void k_diagfilter(double *ap, const double *nna, const double *p, double f,
                             long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    ap[i] = nna[i] * p[i] * f;
}

__global__ void k_add(double *a, const double *b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    a[i] = a[i] + b[i];
}

// clean_tod (smadam_routines.f90:1545-1585): every sample, no pixel test
__global__ void k_clean_tod(double *tod, long long n, SampleMap sm, const double *aa) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long det = i / sm.nsamp, s = i - det * sm.nsamp;
    tod[i] = tod[i] - 1.0 * aa[baseline_of(sm, det, s)];
  }
}

// restore_pixels (pointing.f90:168-191) and the list of samples whose value
// differs from the caller's input
__global__ void k_restore(const int32_t *pixc, const int32_t *orig, long long n, const int *sub2,
                          int nosubpix, int32_t *final_pix, long long *idx, int32_t *val,
                          unsigned long long *count, long long cap) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = pixc[i];
    const int v = c + sub2[c / nosubpix] * nosubpix;
    if (final_pix) final_pix[i] = v;
    if (orig && v != orig[i]) {
      const unsigned long long o = atomicAdd(count, 1ull);
      if ((long long)o < cap) {
        idx[o] = i;
        val[o] = v;
      }
    }
  }
}

__global__ void k_monopole(const double *map, const int *mask, long long n, int nmap,
                           double *part) {
  double v[2] = {0, 0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    v[0] += map[p * nmap];
    v[1] += mask[p] > 0 ? 1.0 : 0.0;
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = v[0];
    part[gridDim.x + blockIdx.x] = v[1];
  }
}

__global__ void k_sub_monopole(double *map, const int *mask, long long n, int nmap,
                               const double *scal) {
  const double cover = scal[1];
  if (cover == 0) return;
  const double mono = scal[0] / cover;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x)
    if (mask[p] > 0) map[p * nmap] -= mono;
}

// --- CG fallback preconditioner (apply_CG_preconditioner,
// noise_routines.f90:1305-1409), one CTA per segment
struct CgpSeg {
  long long k0;
  int n;
  int spec;
};

__global__ void k_cgp_init(const CgpSeg *segs, const double *r, double *x, double *resid,
                           double *prop, double *zres, double *prec, const double *nna,
                           const double *invcov, long long nof, double *st, int *done) {
  const CgpSeg g = segs[blockIdx.x];
  const double ic0 = invcov[(long long)g.spec * nof];
  double v[2] = {0, 0};
  for (int i = threadIdx.x; i < g.n; i += blockDim.x) {
    const long long k = g.k0 + i;
    x[k] = 0;
    const double rr = r[k];
    resid[k] = rr;
    double pc = nna[k] + ic0;
    if (pc != 0) pc = 1 / pc;
    prec[k] = pc;
    const double zz = pc * rr;
    zres[k] = zz;
    prop[k] = zz;
    v[0] += rr * rr;
    v[1] += rr * zz;
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    st[4 * blockIdx.x + 0] = v[0];  // rr
    st[4 * blockIdx.x + 1] = v[0];  // rr0
    st[4 * blockIdx.x + 2] = v[1];  // rz
    done[blockIdx.x] = (v[0] == 0);
  }
}

__global__ void k_cgp_step(const CgpSeg *segs, double *x, double *resid, double *prop,
                           double *aprop, double *zres, const double *prec, const double *nna,
                           double *st, int *done, int iter, int *active) {
  if (done[blockIdx.x]) return;
  const CgpSeg g = segs[blockIdx.x];
  __shared__ double sh[2];
  double v[2] = {0, 0};
  for (int i = threadIdx.x; i < g.n; i += blockDim.x) {
    const long long k = g.k0 + i;
    const double a = aprop[k] + nna[k] * prop[k];
    aprop[k] = a;
    v[0] += prop[k] * a;
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) sh[0] = st[4 * blockIdx.x + 2] / v[0];
  __syncthreads();
  const double alpha = sh[0];
  v[0] = 0;
  for (int i = threadIdx.x; i < g.n; i += blockDim.x) {
    const long long k = g.k0 + i;
    x[k] = x[k] + alpha * prop[k];
    const double rs = resid[k] - alpha * aprop[k];
    resid[k] = rs;
    v[0] += rs * rs;
  }
  v[1] = 0;
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    st[4 * blockIdx.x + 0] = v[0];
    const bool fin = (v[0] / st[4 * blockIdx.x + 1] < fsp(1e-6f)) || iter == 100;
    done[blockIdx.x] = fin;
    sh[1] = fin;
  }
  __syncthreads();
  if (sh[1] != 0) return;
  v[0] = 0;
  v[1] = 0;
  for (int i = threadIdx.x; i < g.n; i += blockDim.x) {
    const long long k = g.k0 + i;
    const double zz = prec[k] * resid[k];
    zres[k] = zz;
    v[0] += resid[k] * zz;
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    const double rz_old = st[4 * blockIdx.x + 2];
    st[4 * blockIdx.x + 2] = v[0];
    sh[0] = v[0] / rz_old;
    atomicAdd(active, 1);
  }
  __syncthreads();
  const double beta = sh[0];
  for (int i = threadIdx.x; i < g.n; i += blockDim.x) {
    const long long k = g.k0 + i;
    prop[k] = zres[k] + beta * prop[k];
  }
}

__global__ void k_copy_seg(const CgpSeg *segs, const double *x, double *z) {
  const CgpSeg g = segs[blockIdx.x];
  for (int i = threadIdx.x; i < g.n; i += blockDim.x) z[g.k0 + i] = x[g.k0 + i];
}

unsigned grid_for(long long n, int block = 256) {
  long long g = (n + block - 1) / block;
  return (unsigned)std::max(1LL, std::min(g, 148LL * 32));
}

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

#include "batch_kernels.inl"
#include "pair_kernels.inl"
#include "engine_host.inl"
#include "engine_batch.inl"
#include "subsets.inl"
#include "basis.inl"
#include "covmat.inl"

}  // namespace madam
