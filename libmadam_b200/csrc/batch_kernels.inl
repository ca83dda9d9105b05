// Multi-right-hand-side kernels of the batched Monte-Carlo solve
// (madam_b200_destripe_with_cache_batch).  The R realisations share the
// pointing, the pixel matrices, the filter and the preconditioner, so one
// pass over the pointing serves a group of RB right-hand sides.  Vectors are
// stored right-hand-side major ([R][nb] baseline vectors, [R][npix][nmap]
// maps).  For every right-hand side the arithmetic and its order are those
// of the single-RHS kernels (same chunking, same per-lane sums, same warp
// trees), so a batched solve repeats the single solves to the last bit.
// `act[r]` is 0 for right-hand sides whose PCG has stopped.

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

// map_to_baseline for right-hand sides [r0, r0 + nr), nr <= RB; the warps'
// staging slices are [RB][kGatherChunk] doubles of dynamic shared memory
template <int NMAP, int RB>
__global__ void __launch_bounds__(256) k_gather_chunks_b(
    const int2 *__restrict__ chunks, long long nchunks, const float4 *__restrict__ p4,
    const int32_t *__restrict__ pc, const uint32_t *__restrict__ bstart, long noba,
    long long nsamp, const double *__restrict__ bw, const double *__restrict__ p, long long nb,
    const double *__restrict__ nna, const double *__restrict__ m, long long mstride,
    int deg_shift, int nloc, const uint8_t *__restrict__ rmask, double *__restrict__ ap,
    int r0, int nr, double *__restrict__ part) {
  extern __shared__ double gvb[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double *vb = gvb + (size_t)wid * RB * kGatherChunk;
  const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  constexpr int U = kGatherChunk / 32;
  double pap[RB];
#pragma unroll
  for (int j = 0; j < RB; ++j) pap[j] = 0.0;
  for (long long c = w0; c < nchunks; c += nwarps) {
    const int2 ck = chunks[c];
    const long long det = ck.x / noba, k0 = ck.x - det * noba;
    const int s0 = (int)bstart[k0];
    const int n = (int)(bstart[k0 + ck.y] - s0);
    const long long base = det * nsamp + s0;
    double detw = 0;
    double pb[RB], apb[RB], npb[RB];
    int a0 = 0, a1 = 0;
    bool rm = false;
    if (lane < ck.y) {
      const long long b = ck.x + lane;
      detw = bw[b];
      const double nn = nna[b];
#pragma unroll
      for (int j = 0; j < RB; ++j) {
        if (j < nr) {
          pb[j] = p[(long long)(r0 + j) * nb + b];
          apb[j] = ap[(long long)(r0 + j) * nb + b];
          npb[j] = nn * pb[j];
        }
      }
      rm = rmask[b] != 0;
      a0 = (int)(bstart[k0 + lane] - s0);
      a1 = (int)(bstart[k0 + lane + 1] - s0);
    }
    if (NMAP == 3) {
      float4 q[U];
#pragma unroll
      for (int r = 0; r < U; ++r) {
        const int i = r * 32 + lane;
        q[r] = i < n ? __ldcs(p4 + base + i) : make_float4(0.f, 0.f, 0.f, __int_as_float(nloc));
      }
#pragma unroll
      for (int j = 0; j < RB; ++j) {
        if (j >= nr) break;
        const double *mj = m + (long long)(r0 + j) * mstride;
#pragma unroll
        for (int r = 0; r < U; ++r) {
          const int px = point_pix(q[r]);
          double v = 0.0;
          if (px < nloc) {
            const double *mm = mj + (long long)(px >> deg_shift) * 3;
            v = (double)q[r].x * mm[0] + (double)q[r].y * mm[1] + (double)q[r].z * mm[2];
          }
          vb[j * kGatherChunk + r * 32 + lane] = v;
        }
      }
    } else {
      int px[U];
#pragma unroll
      for (int r = 0; r < U; ++r) {
        const int i = r * 32 + lane;
        px[r] = i < n ? __ldcs(pc + base + i) : nloc;
      }
#pragma unroll
      for (int j = 0; j < RB; ++j) {
        if (j >= nr) break;
        const double *mj = m + (long long)(r0 + j) * mstride;
#pragma unroll
        for (int r = 0; r < U; ++r)
          vb[j * kGatherChunk + r * 32 + lane] = px[r] < nloc ? mj[px[r] >> deg_shift] : 0.0;
      }
    }
    __syncwarp();
    if (lane < ck.y) {
      const long long b = ck.x + lane;
#pragma unroll
      for (int j = 0; j < RB; ++j) {
        if (j >= nr) break;
        if (detw == 0) {
          if (rm) pap[j] += pb[j] * apb[j];
        } else {
          double apn = 0;
          for (int i = a0; i < a1; ++i) apn += vb[j * kGatherChunk + i];
          const double val = apb[j] + (npb[j] - apn * detw);
          ap[(long long)(r0 + j) * nb + b] = val;
          if (rm) pap[j] += pb[j] * val;
        }
      }
    }
    __syncwarp();
  }
  block_sum<RB>(pap);
  if (threadIdx.x == 0)
    for (int j = 0; j < nr; ++j) part[(long long)(r0 + j) * 3 * kRedBlocks + blockIdx.x] = pap[j];
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
    sc[S_RZO] = sc[S_RZ];
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
