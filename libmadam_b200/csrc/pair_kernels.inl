// Pointing pairs of the FP32-TOD precision form (madam_b200_destripe_fp32).
//
// Consecutive valid samples of one baseline that fall in one cross pixel
// form a pair {sum w_I, sum w_Q, sum w_U, cross pixel} (sums in double,
// stored as float).  A sample is valid when it has a map pixel (< nloc) and
// its baseline a nonzero weight.  Both PCG products need only these sums:
// sum_s w_s . m[p_s] = sum_pairs (sum w) . m[p] (map_to_baseline) and
// sum_{s in p} w_s a_b(s) = sum_{pairs in p} (sum w) a_b (baseline_to_map),
// so each PCG iteration streams the pairs (about two samples each on a ring
// scan) instead of the samples.  Rounding the sums to float moves the
// solution by ~1e-7 relative in well-conditioned systems, inside the form's
// 1e-4 tolerance; the FP64 path keeps the samples.

// head[i] = 1 where a pair starts: sample i is valid and starts its
// baseline, or follows an invalid sample or one in another cross pixel
__global__ void k_pair_heads(const float4 *p4, long long n, SampleMap sm, const double *bw,
                             int nloc, int deg_shift, int *head) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long det = i / sm.nsamp, s = i - det * sm.nsamp;
    const int px = point_pix(p4[i]);
    int h = 0;
    if (px < nloc) {
      const long long b = baseline_of(sm, det, s);
      if (bw[b] != 0.0) {
        if (s == 0) {
          h = 1;
        } else {
          const int pp = point_pix(p4[i - 1]);
          h = (pp >= nloc || (pp >> deg_shift) != (px >> deg_shift) ||
               baseline_of(sm, det, s - 1) != b)
                  ? 1
                  : 0;
        }
      }
    }
    head[i] = h;
  }
}

// one thread per pair head: the pair's weight sums (time order) and its
// global baseline
__global__ void k_pair_fill(const float4 *p4, long long n, SampleMap sm, const uint32_t *bstart,
                            int nloc, int deg_shift, const int *head, const int *pidx,
                            float4 *gp4, int *pbase) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (!head[i]) continue;
    const long long det = i / sm.nsamp, s = i - det * sm.nsamp;
    const long long b = baseline_of(sm, det, s);
    const long long k = b - det * sm.noba_short;
    const long long end = det * sm.nsamp + bstart[k + 1];
    const int cross = point_pix(p4[i]) >> deg_shift;
    double w0 = 0, w1 = 0, w2 = 0;
    for (long long j = i; j < end; ++j) {
      const float4 q = p4[j];
      if (j > i) {
        const int pj = point_pix(q);
        if (pj >= nloc || (pj >> deg_shift) != cross) break;
      }
      w0 += q.x;
      w1 += q.y;
      w2 += q.z;
    }
    const int o = pidx[i];
    gp4[o] = make_float4((float)w0, (float)w1, (float)w2, __int_as_float(cross));
    pbase[o] = (int)b;
  }
}

// poff[b] = first pair of baseline b (pairs before its first sample);
// poff[nb] = number of pairs
__global__ void k_pair_offsets(const int *pidx, const uint32_t *bstart, long long nsamp,
                               long noba, long long nb, long long n, int total, int *poff) {
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b <= nb;
       b += (long long)gridDim.x * blockDim.x) {
    if (b == nb) {
      poff[b] = total;
      continue;
    }
    const long long det = b / noba, k = b - det * noba;
    const long long i = det * nsamp + bstart[k];
    poff[b] = i < n ? pidx[i] : total;
  }
}

__global__ void k_pair_keys(const float4 *gp4, int npair, int *keys, uint32_t *vals) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npair; i += gridDim.x * blockDim.x) {
    keys[i] = __float_as_int(gp4[i].w);
    vals[i] = (uint32_t)i;
  }
}

// pixel-sorted pairs {sum w, global baseline} and the CSR offsets
__global__ void k_pair_csr_fill(const int *keys, const uint32_t *idx, int npair,
                                const float4 *gp4, const int *pbase, float4 *sp4, int *off) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npair; i += gridDim.x * blockDim.x) {
    const int src = (int)idx[i];
    const float4 q = gp4[src];
    sp4[i] = make_float4(q.x, q.y, q.z, __int_as_float(pbase[src]));
    const int key = keys[i];
    const int prev = i == 0 ? -1 : keys[i - 1];
    for (int p = prev + 1; p <= key; ++p) off[p] = i;
  }
}

// map_to_baseline over pairs: warp chunks {first baseline, baselines, first
// pair, pairs} of <= kGatherChunk pairs and <= 32 baselines.  A lane loads
// its 8 pairs (coalesced) with their float32 map values in flight, stages
// w.m in the warp's shared-memory slice, and chunk_baseline_sums adds every
// baseline of the chunk at once (a pair chunk holds few long baselines);
// fused with the p.ap partial sums.
__global__ void __launch_bounds__(256) k_gather_pairs(
    const int4 *__restrict__ chunks, long long nchunks, const float4 *__restrict__ gp4,
    const int *__restrict__ poff, const double *__restrict__ bw, const double *__restrict__ p,
    const double *__restrict__ nna, const float4 *__restrict__ mf,
    const uint8_t *__restrict__ rmask, double *__restrict__ ap, double *__restrict__ part) {
  __shared__ double vbuf[8][kGatherChunk + kGatherChunk / 8];
  __shared__ ChunkSmem csm[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double *vb = vbuf[wid];
  ChunkSmem &cs = csm[wid];
  const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  constexpr int U = kGatherChunk / 32;
  double pap = 0;
  for (long long c = w0; c < nchunks; c += nwarps) {
    const int4 ck = chunks[c];
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
      a0 = poff[b] - ck.z;
      a1 = poff[b + 1] - ck.z;
    }
    float4 q[U];
#pragma unroll
    for (int r = 0; r < U; ++r) {
      const int i = r * 32 + lane;
      q[r] = i < ck.w ? __ldcs(gp4 + (long long)ck.z + i)
                      : make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
    }
#pragma unroll
    for (int r = 0; r < U; ++r) {
      const int px = __float_as_int(q[r].w);
      vb[r * 36 + lane + (lane >> 3)] = px >= 0 ? map_dot(mf, px, q[r]) : 0.0;
    }
    __syncwarp();
    chunk_baseline_sums(vb, ck.y, a0, a1, cs, lane);
    if (lane < ck.y) {
      const long long b = ck.x + lane;
      if (detw == 0) {
        if (rm) pap += pb * apb;
      } else {
        const double val = apb + fma(-cs.bsum[lane], detw, npb);
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

__global__ void k_f32_to_f64(const float *a, double *b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = (double)a[i];
}

__global__ void k_f64_to_f32(const double *a, float *b, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}
