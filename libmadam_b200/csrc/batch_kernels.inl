// Multi-right-hand-side kernels of the batched Monte-Carlo solve
// (madam_b200_destripe_with_cache_batch).  The R realisations share the
// pointing, the pixel matrices, the filter and the preconditioner, so one
// pass over the pointing serves a group of right-hand sides.  Baseline
// vectors are stored right-hand-side major ([R][nb]); the projections work
// on right-hand-side-minor copies (below).  For every right-hand side the
// arithmetic of the projections and its order are those of the single-RHS
// kernels.  `act[r]` is 0 for right-hand sides whose PCG has stopped.

// baseline_to_map for right-hand sides [r0, r0 + nr), nr <= RB
template <int NMAP, int RB>
__global__ void __launch_bounds__(256) k_scatter_chunks_b(
    const int4 *__restrict__ chunks, long long nchunks, const float4 *__restrict__ sp4,
    const int2 *__restrict__ sp2, const double *__restrict__ pw, long long nb, int r0, int nr,
    double *__restrict__ target, long long tstride, double *__restrict__ partial,
    long long pstride) {
  const int lane = threadIdx.x & 31;
  const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  constexpr int U = kScatterChunk / 32;
  for (long long c = w0; c < nchunks; c += nwarps) {
    const int4 ck = chunks[c];
    float4 q[U];
    int k[U];
#pragma unroll
    for (int r = 0; r < U; ++r) {
      const int i = r * 32 + lane;
      if (NMAP == 3) {
        q[r] = i < ck.z ? __ldcs(sp4 + ck.y + i) : make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
        k[r] = __float_as_int(q[r].w);
      } else {
        k[r] = i < ck.z ? __ldcs(&sp2[ck.y + i].x) : -1;
      }
    }
    double a[RB][NMAP];
#pragma unroll
    for (int j = 0; j < RB; ++j) {
#pragma unroll
      for (int e = 0; e < NMAP; ++e) a[j][e] = 0.0;
      if (j < nr) {
        const double *pj = pw + (long long)(r0 + j) * nb;
        double wv[U];
#pragma unroll
        for (int r = 0; r < U; ++r) wv[r] = k[r] >= 0 ? pj[k[r]] : 0.0;
#pragma unroll
        for (int r = 0; r < U; ++r) {
          if (NMAP == 3) {
            a[j][0] += (double)q[r].x * wv[r];
            a[j][1] += (double)q[r].y * wv[r];
            a[j][2] += (double)q[r].z * wv[r];
          } else {
            a[j][0] += wv[r];
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < RB; ++j) {
      if (j >= nr) break;
#pragma unroll
      for (int e = 0; e < NMAP; ++e) a[j][e] = warp_sum(a[j][e]);
      if (lane == 0) {
        double *o = ck.w < 0 ? target + (long long)(r0 + j) * tstride + (long long)ck.x * NMAP
                             : partial + (long long)(r0 + j) * pstride + (long long)ck.w * NMAP;
#pragma unroll
        for (int e = 0; e < NMAP; ++e) o[e] = a[j][e];
      }
    }
  }
}

// blockIdx.y = right-hand side
template <int NMAP>
__global__ void k_scatter_combine_b(const int4 *__restrict__ multi, int nmulti,
                                    const double *__restrict__ partial, long long pstride,
                                    double *__restrict__ target, long long tstride) {
  const double *pr = partial + (long long)blockIdx.y * pstride;
  double *tr = target + (long long)blockIdx.y * tstride;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nmulti; i += gridDim.x * blockDim.x) {
    const int4 mp = multi[i];
    double a[3] = {0, 0, 0};
    for (int c = 0; c < mp.z; ++c)
      for (int j = 0; j < NMAP; ++j) a[j] += pr[(long long)(mp.y + c) * NMAP + j];
    for (int j = 0; j < NMAP; ++j) tr[(long long)mp.x * NMAP + j] = a[j];
  }
}

template <int NMAP>
__global__ void k_ccmult_b(const double *cc, double *m, long long n) {
  double *mr = m + (long long)blockIdx.y * n * NMAP;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    if (NMAP == 1) {
      const double c = cc[p];
      mr[p] = (c == 0) ? 0.0 : c * mr[p];
    } else {
      const double *c = cc + p * 6;
      double *v = mr + p * 3;
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

// masked dots for every active right-hand side: blockIdx.y = r, part
// [R][3][kRedBlocks]
__global__ void k_dots_b(const double *a0, const double *b0, const double *a1, const double *b1,
                         const double *a2, const double *b2, int nd, const uint8_t *mask,
                         long long n, const int *act, double *part) {
  const int rr = blockIdx.y;
  if (!act[rr]) return;
  const long long o = (long long)rr * n;
  double v[3] = {0, 0, 0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (!mask[i]) continue;
    v[0] += a0[o + i] * b0[o + i];
    if (nd > 1) v[1] += a1[o + i] * b1[o + i];
    if (nd > 2) v[2] += a2[o + i] * b2[o + i];
  }
  block_sum<3>(v);
  double *pr = part + (long long)rr * 3 * kRedBlocks;
  if (threadIdx.x == 0)
    for (int j = 0; j < 3; ++j) pr[j * gridDim.x + blockIdx.x] = v[j];
}

// k_finish per right-hand side: blockIdx.x = r, scal [R][S_NSCAL]
__global__ void k_finish_b(const double *part, int nblk, int nd, double *scal, int mode,
                           int slot0, const int *act) {
  const int rr = blockIdx.x;
  if (!act[rr]) return;
  const double *pr = part + (long long)rr * 3 * kRedBlocks;
  double *sc = scal + (long long)rr * S_NSCAL;
  double v[3] = {0, 0, 0};
  for (int j = 0; j < nd; ++j)
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) v[j] += pr[j * nblk + i];
  block_sum<3>(v);
  if (threadIdx.x != 0) return;
  if (mode == 0) {
    for (int j = 0; j < nd; ++j) sc[slot0 + j] = v[j];
  } else if (mode == 1) {
    sc[S_PAP] = v[0];
    sc[S_ALPHA] = sc[S_RZ] / v[0];
  } else {
    if (mode == 2) sc[S_RZO] = sc[S_RZ];  // mode 3: a reliable update's redo
    sc[S_RZ] = v[0];
    sc[S_RZ2] = v[1];
    sc[S_RR] = v[2];
    sc[S_BETA] = (v[0] - v[1]) / sc[S_RZO];
  }
}

__global__ void k_update_ar_b(double *aa, double *r, double *ro, const double *p,
                              const double *ap, long long n, const double *scal, const int *act) {
  const int rr = blockIdx.y;
  if (!act[rr]) return;
  const double alpha = scal[(long long)rr * S_NSCAL + S_ALPHA];
  const long long o = (long long)rr * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    aa[o + i] = aa[o + i] + alpha * p[o + i];
    const double ri = r[o + i];
    ro[o + i] = ri;
    r[o + i] = ri - alpha * ap[o + i];
  }
}

__global__ void k_update_p_b(double *p, const double *z, double *pw, const double *bw,
                             long long n, const double *scal, int first, const int *act) {
  const int rr = blockIdx.y;
  if (!act[rr]) return;
  const double beta = first ? 0.0 : scal[(long long)rr * S_NSCAL + S_BETA];
  const long long o = (long long)rr * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = first ? z[o + i] : z[o + i] + beta * p[o + i];
    p[o + i] = v;
    pw[o + i] = v * bw[i];
  }
}

// ---------------------------------------------------------------------------
// Right-hand-side-minor projections.  For a group of up to 32 G right-hand
// sides, p.detw and the map are stored transposed, [baseline][32 G] and
// [pixel][nmap][32 G], so that the lanes of a warp hold 32 G right-hand
// sides of ONE sample: a pointing record is read once (a shared-memory
// broadcast) and its lookups are coalesced 256-byte rows instead of one
// scattered 8-byte load per sample and right-hand side.  Each right-hand
// side sees the arithmetic of k_scatter_chunks / k_gather_chunks in the same
// order, so its map and baseline sums equal theirs to the bit.

// [R][nb] (right-hand sides r0 .. r0 + nr) -> [nb][32 G], zero padded; T =
// float in the FP32-TOD form
template <int G, class T>
__global__ void k_transpose_rhs(const double *__restrict__ src, long long nb, int r0, int nr,
                                T *__restrict__ dst) {
  constexpr int GW = 32 * G;
  __shared__ double t[32][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  const int g = blockIdx.y;
  for (long long b0 = (long long)blockIdx.x * 32; b0 < nb; b0 += (long long)gridDim.x * 32) {
    for (int rr = ty; rr < 32; rr += 8) {
      const int r = g * 32 + rr;
      const long long b = b0 + tx;
      t[rr][tx] = (r < nr && b < nb) ? src[(long long)(r0 + r) * nb + b] : 0.0;
    }
    __syncthreads();
    for (int bb = ty; bb < 32; bb += 8) {
      const long long b = b0 + bb;
      if (b < nb) dst[b * GW + g * 32 + tx] = (T)t[tx][bb];
    }
    __syncthreads();
  }
}

__host__ __device__ constexpr int cpopc5(int x) {
  return (x & 1) + ((x >> 1) & 1) + ((x >> 2) & 1) + ((x >> 3) & 1) + ((x >> 4) & 1);
}
__host__ __device__ constexpr int ctrail1(int x) { return (x & 1) ? 1 + ctrail1(x >> 1) : 0; }
__host__ __device__ constexpr int cbrev5(int x) {
  return ((x & 1) << 4) | ((x & 2) << 2) | (x & 4) | ((x & 8) >> 2) | ((x & 16) >> 4);
}

// baseline_to_map over the pixel-sorted chunks of k_scatter_chunks.  There,
// lane L adds entries L, L + 32, ... and a xor butterfly adds the 32 lane
// sums; the butterfly's association (as lane 0 holds it) is a balanced
// binary tree over the lane sums in bit-reversed lane order.  Here lane r
// forms right-hand side r's lane sums one column at a time in that order:
// four subtrees of 8 columns each (unrolled, on a binary-counter stack),
// then ((X0 + X1) + (X2 + X3)) - the same tree.  Keeping the unrolled part
// to 8 columns keeps the kernel's code small enough for the instruction
// cache.  One launch covers the 32 right-hand sides g0 .. g0 + 31 of rows
// of GW.
template <int NMAP, int GW, class TW>
__global__ void __launch_bounds__(256) k_scatter_T(
    const int4 *__restrict__ chunks, long long nchunks, const float4 *__restrict__ sp4,
    const int2 *__restrict__ sp2, const TW *__restrict__ pwT, int g0,
    double *__restrict__ target, double *__restrict__ partial) {
  constexpr int G = 1;
  constexpr int U = kScatterChunk / 32;
  __shared__ float4 rec[8][kScatterChunk];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  float4 *rw = rec[wid];
  for (long long c = w0; c < nchunks; c += nwarps) {
    const int4 ck = chunks[c];  // {pixel, first entry, entries, partial slot or -1}
#pragma unroll
    for (int r = 0; r < U; ++r) {
      const int i = r * 32 + lane;
      if (i < ck.z)
        rw[i] = NMAP == 3 ? __ldcs(sp4 + ck.y + i)
                          : make_float4(1.f, 0.f, 0.f, __int_as_float(__ldcs(&sp2[ck.y + i].x)));
    }
    __syncwarp();
    double B0[G][NMAP], B1[G][NMAP];
#pragma unroll 1
    for (int o = 0; o < 4; ++o) {
      // columns i = 8 o + j, lanes L = bitrev5(i) = 4 bitrev3(j) + bitrev2(o)
      const int lo2 = ((o & 1) << 1) | (o >> 1);
      double S[4][G][NMAP];
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) {
        const int L = (cbrev5(jj) >> 0) + lo2;  // cbrev5(jj) = 4 bitrev3(jj) for jj < 8
        double P[G][NMAP];
#pragma unroll
        for (int g = 0; g < G; ++g)
#pragma unroll
          for (int e = 0; e < NMAP; ++e) P[g][e] = 0.0;
#pragma unroll
        for (int r = 0; r < U; ++r) {
          const int e0 = r * 32 + L;
          if (e0 < ck.z) {
            const float4 q = rw[e0];
            const TW *pk = pwT + (long long)__float_as_int(q.w) * GW + g0 + lane;
#pragma unroll
            for (int g = 0; g < G; ++g) {
              const double wv = (double)__ldg(pk + g * 32);
              if (NMAP == 3) {
                P[g][0] = fma((double)q.x, wv, P[g][0]);
                P[g][1] = fma((double)q.y, wv, P[g][1]);
                P[g][2] = fma((double)q.z, wv, P[g][2]);
              } else {
                P[g][0] += wv;
              }
            }
          }
        }
        // push column jj's sum, then carry as a binary counter does
        const int pos = cpopc5(jj);
#pragma unroll
        for (int g = 0; g < G; ++g)
#pragma unroll
          for (int e = 0; e < NMAP; ++e) S[pos][g][e] = P[g][e];
        const int t = ctrail1(jj);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          if (k < t) {
            const int lv = pos - 1 - k;
#pragma unroll
            for (int g = 0; g < G; ++g)
#pragma unroll
              for (int e = 0; e < NMAP; ++e) S[lv][g][e] = S[lv][g][e] + S[lv + 1][g][e];
          }
        }
      }
#pragma unroll
      for (int g = 0; g < G; ++g)
#pragma unroll
        for (int e = 0; e < NMAP; ++e) {
          const double x = S[0][g][e];
          if (o == 0) B0[g][e] = x;
          else if (o == 1) B0[g][e] = B0[g][e] + x;
          else if (o == 2) B1[g][e] = x;
          else B1[g][e] = B1[g][e] + x;
        }
    }
    double *out = ck.w < 0 ? target + (long long)ck.x * NMAP * GW
                           : partial + (long long)ck.w * NMAP * GW;
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int e = 0; e < NMAP; ++e) out[e * GW + g0 + g * 32 + lane] = B0[g][e] + B1[g][e];
    __syncwarp();
  }
}

// The FP32-TOD batch's baseline_to_map over the same chunks: lane j holds
// right-hand sides j, j + 32, ... (all GW of a row in one launch) and adds a
// chunk's entries in entry order.  The float32 p.detw already sets this
// form's precision, so the single solve's summation tree is not rebuilt.
template <int NMAP, int GW>
__global__ void __launch_bounds__(256) k_scatter_T_seq(
    const int4 *__restrict__ chunks, long long nchunks, const float4 *__restrict__ sp4,
    const int2 *__restrict__ sp2, const float *__restrict__ pwT, double *__restrict__ target,
    double *__restrict__ partial) {
  constexpr int G = GW / 32;
  constexpr int U = kScatterChunk / 32;
  __shared__ float4 rec[8][kScatterChunk];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  float4 *rw = rec[wid];
  for (long long c = w0; c < nchunks; c += nwarps) {
    const int4 ck = chunks[c];  // {pixel, first entry, entries, partial slot or -1}
#pragma unroll
    for (int r = 0; r < U; ++r) {
      const int i = r * 32 + lane;
      if (i < ck.z)
        rw[i] = NMAP == 3 ? __ldcs(sp4 + ck.y + i)
                          : make_float4(1.f, 0.f, 0.f, __int_as_float(__ldcs(&sp2[ck.y + i].x)));
    }
    __syncwarp();
    double P[G][NMAP];
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int e = 0; e < NMAP; ++e) P[g][e] = 0.0;
#pragma unroll 8
    for (int i = 0; i < ck.z; ++i) {
      const float4 q = rw[i];
      const float *pk = pwT + (long long)__float_as_int(q.w) * GW + lane;
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const double wv = (double)__ldg(pk + g * 32);
        if (NMAP == 3) {
          P[g][0] = fma((double)q.x, wv, P[g][0]);
          P[g][1] = fma((double)q.y, wv, P[g][1]);
          P[g][2] = fma((double)q.z, wv, P[g][2]);
        } else {
          P[g][0] += wv;
        }
      }
    }
    double *out = ck.w < 0 ? target + (long long)ck.x * NMAP * GW
                           : partial + (long long)ck.w * NMAP * GW;
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int e = 0; e < NMAP; ++e) out[e * GW + g * 32 + lane] = P[g][e];
    __syncwarp();
  }
}

// multi-chunk pixels {pixel, first partial slot, chunks}: partial sums added
// in chunk order; thread per (pixel, component, right-hand side)
template <int NMAP, int G>
__global__ void k_scatter_combine_T(const int4 *__restrict__ multi, int nmulti,
                                    const double *__restrict__ partial,
                                    double *__restrict__ target) {
  constexpr int GW = 32 * G;
  const long long total = (long long)nmulti * NMAP * GW;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / (NMAP * GW));
    const int ce = (int)(t - (long long)i * NMAP * GW);
    const int4 mp = multi[i];
    double a = 0.0;
    for (int c = 0; c < mp.z; ++c) a += partial[(long long)(mp.y + c) * NMAP * GW + ce];
    target[(long long)mp.x * NMAP * GW + ce] = a;
  }
}

// ccmultiply on the transposed map; thread per (pixel, right-hand side)
// (and, in the FP32-TOD form, a float32 copy mf for the gather)
template <int NMAP, int G>
__global__ void k_ccmult_T(const double *__restrict__ cc, double *__restrict__ m, long long n,
                           float *__restrict__ mf) {
  constexpr int GW = 32 * G;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n * GW;
       t += (long long)gridDim.x * blockDim.x) {
    const long long p = t / GW;
    const int r = (int)(t - p * GW);
    double *v = m + p * NMAP * GW + r;
    if (NMAP == 1) {
      const double c = cc[p];
      v[0] = (c == 0) ? 0.0 : c * v[0];
    } else {
      const double *c = cc + p * 6;
      if (c[0] == 0) {
        v[0] = v[GW] = v[2 * GW] = 0;
      } else {
        const double a = v[0], b = v[GW], d = v[2 * GW];
        v[0] = fma(c[2], d, fma(c[1], b, c[0] * a));
        v[GW] = fma(c[4], d, fma(c[3], b, c[1] * a));
        v[2 * GW] = fma(c[5], d, fma(c[4], b, c[2] * a));
      }
    }
    if (mf) {
      float *f = mf + p * NMAP * GW + r;
#pragma unroll
      for (int e = 0; e < NMAP; ++e) f[e * GW] = (float)v[e * GW];
    }
  }
}

// map_to_baseline sums per baseline and right-hand side, in time order as
// lane j of k_gather_chunks adds baseline j: apnT[b][r] = sum_s w_s . m_r[p_s]
template <int NMAP, int G, class TM>
__global__ void __launch_bounds__(256) k_gather_T(
    const int2 *__restrict__ chunks, long long nchunks, const float4 *__restrict__ p4,
    const int32_t *__restrict__ pc, const uint32_t *__restrict__ bstart, long noba,
    long long nsamp, const TM *__restrict__ mT, int deg_shift, int nloc,
    double *__restrict__ apnT) {
  constexpr int GW = 32 * G;
  constexpr int U = kGatherChunk / 32;
  __shared__ float4 rec[8][kGatherChunk];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  float4 *rw = rec[wid];
  for (long long c = w0; c < nchunks; c += nwarps) {
    const int2 ck = chunks[c];
    const long long det = ck.x / noba, k0 = ck.x - det * noba;
    const int s0 = (int)bstart[k0];
    const int n = (int)(bstart[k0 + ck.y] - s0);
    const long long base = det * nsamp + s0;
#pragma unroll
    for (int r = 0; r < U; ++r) {
      const int i = r * 32 + lane;
      if (i < n)
        rw[i] = NMAP == 3 ? __ldcs(p4 + base + i)
                          : make_float4(0.f, 0.f, 0.f, __int_as_float(__ldcs(pc + base + i)));
    }
    __syncwarp();
    int a1 = 0;
    for (int j = 0; j < ck.y; ++j) {
      const int a0 = a1;
      a1 = (int)(bstart[k0 + j + 1] - s0);
      double apn[G];
#pragma unroll
      for (int g = 0; g < G; ++g) apn[g] = 0.0;
#pragma unroll 4
      for (int s = a0; s < a1; ++s) {
        const float4 q = rw[s];
        const int px = __float_as_int(q.w);
        if (px < nloc) {
          const TM *mm = mT + (long long)(px >> deg_shift) * NMAP * GW + lane;
#pragma unroll
          for (int g = 0; g < G; ++g) {
            if (NMAP == 3) {
              const double m0 = (double)__ldg(mm + g * 32), m1 = (double)__ldg(mm + GW + g * 32),
                           m2 = (double)__ldg(mm + 2 * GW + g * 32);
              apn[g] += fma((double)q.z, m2, fma((double)q.y, m1, (double)q.x * m0));
            } else {
              apn[g] += (double)__ldg(mm + g * 32);
            }
          }
        } else {
#pragma unroll
          for (int g = 0; g < G; ++g) apn[g] += 0.0;
        }
      }
#pragma unroll
      for (int g = 0; g < G; ++g) apnT[(long long)(ck.x + j) * GW + g * 32 + lane] = apn[g];
    }
    __syncwarp();
  }
}

// The FP32-TOD batch's map_to_baseline over pointing pairs (as
// k_gather_pairs): chunks {first baseline, baselines, first pair, pairs},
// per-baseline pair offsets poff, pair records {sum w, cross pixel (-1:
// none)}; lane j holds right-hand sides j, j + 32, ... and sums each
// baseline's pairs in time order from the float32 map rows.
template <int G>
__global__ void __launch_bounds__(256) k_gather_T_pairs(
    const int4 *__restrict__ chunks, long long nchunks, const float4 *__restrict__ gp4,
    const int *__restrict__ poff, const float *__restrict__ mT, double *__restrict__ apnT) {
  constexpr int GW = 32 * G;
  constexpr int U = kGatherChunk / 32;
  __shared__ float4 rec[8][kGatherChunk];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  float4 *rw = rec[wid];
  for (long long c = w0; c < nchunks; c += nwarps) {
    const int4 ck = chunks[c];
#pragma unroll
    for (int r = 0; r < U; ++r) {
      const int i = r * 32 + lane;
      if (i < ck.w) rw[i] = __ldcs(gp4 + (long long)ck.z + i);
    }
    __syncwarp();
    int a1 = poff[ck.x] - ck.z;
    for (int j = 0; j < ck.y; ++j) {
      const int a0 = a1;
      a1 = poff[ck.x + j + 1] - ck.z;
      double apn[G];
#pragma unroll
      for (int g = 0; g < G; ++g) apn[g] = 0.0;
#pragma unroll 4
      for (int s = a0; s < a1; ++s) {
        const float4 q = rw[s];
        const int px = __float_as_int(q.w);
        if (px >= 0) {
          const float *mm = mT + (long long)px * 3 * GW + lane;
#pragma unroll
          for (int g = 0; g < G; ++g) {
            const double m0 = (double)__ldg(mm + g * 32), m1 = (double)__ldg(mm + GW + g * 32),
                         m2 = (double)__ldg(mm + 2 * GW + g * 32);
            apn[g] += fma((double)q.z, m2, fma((double)q.y, m1, (double)q.x * m0));
          }
        }
      }
#pragma unroll
      for (int g = 0; g < G; ++g) apnT[(long long)(ck.x + j) * GW + g * 32 + lane] = apn[g];
    }
    __syncwarp();
  }
}

// ap[r][b] = ap + (nna p - apn detw) for the group's right-hand sides and the
// p.ap partial sums per block; a block transposes tiles of 32 baselines
template <int G>
__global__ void __launch_bounds__(256) k_gather_finish_T(
    const double *__restrict__ apnT, long long nb, const double *__restrict__ bw,
    const double *__restrict__ nna, const uint8_t *__restrict__ rmask,
    const double *__restrict__ p, double *__restrict__ ap, int r0, int nr,
    double *__restrict__ part) {
  constexpr int GW = 32 * G;
  constexpr int RPW = GW / 8;  // right-hand sides per warp
  __shared__ double t[32][GW + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double pap[RPW];
#pragma unroll
  for (int k = 0; k < RPW; ++k) pap[k] = 0.0;
  for (long long b0 = (long long)blockIdx.x * 32; b0 < nb; b0 += (long long)gridDim.x * 32) {
    for (int idx = threadIdx.x; idx < 32 * GW; idx += blockDim.x) {
      const int bl = idx / GW, r = idx - bl * GW;
      t[bl][r] = b0 + bl < nb ? apnT[(b0 + bl) * GW + r] : 0.0;
    }
    __syncthreads();
    const long long b = b0 + lane;
    if (b < nb) {
      const double detw = bw[b], nn = nna[b];
      const bool rm = rmask[b] != 0;
#pragma unroll
      for (int k = 0; k < RPW; ++k) {
        const int r = wid + 8 * k;
        if (r < nr) {
          const long long o = (long long)(r0 + r) * nb + b;
          const double pb = p[o], apb = ap[o];
          if (detw == 0) {
            if (rm) pap[k] += pb * apb;
          } else {
            const double val = apb + fma(-t[lane][r], detw, nn * pb);
            ap[o] = val;
            if (rm) pap[k] += pb * val;
          }
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < RPW; ++k) {
    const int r = wid + 8 * k;
    const double s = warp_sum(pap[k]);
    if (lane == 0 && r < nr) part[(long long)(r0 + r) * 3 * kRedBlocks + blockIdx.x] = s;
  }
}
