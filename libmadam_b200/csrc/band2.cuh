// Deduplicated band Cholesky factor and chunk-parallel solve (band2.cu).
#pragma once

#include <cuda_runtime.h>

namespace madam {

// One factored segment.  row_off / run_off locate its distinct rows and runs.
struct PSeg {
  long long k0;       // first baseline of the segment
  long long row_off;  // offset (doubles) of its row table
  int n;              // rows
  int nb;             // band width (w + 1)
  int run_off;        // first run
  int nrun;           // runs
  int ch_off;         // first chunk
  int nch;            // chunks
};

// Rows [start, next run's start) share the distinct row at row_off.
struct PRun {
  int start;
  int pad;
  long long row_off;
};

// A chunk of rows [a, b) of segment seg.
struct PChunk {
  int seg, a, b;
  int run;     // run containing row a
  int run_hi;  // run containing row min(b + w, n) - 1
  int first, last;
  int tf, tb;  // offsets (doubles) of the forward / backward transfer matrices
};

struct PTrans {
  int chunk;       // representative chunk
  int dir;         // 0 forward, 1 backward
  long long off;   // offset of the w x w matrix
};

constexpr int kBand2MaxWidth = 128;
constexpr int kBand2Chunk = 256;

void band2_factor(cudaStream_t st, const PSeg *segs, int nseg, const int *spec,
                  const double *invcov, long long nof, const double *nna, double *urows,
                  PRun *runs, int *status, int *nunique, int *nruns);
void band2_transfer(cudaStream_t st, const PSeg *segs, const PChunk *ch, const PTrans *tr, int ntr,
                    const PRun *runs, const double *urows, double *T);
void band2_solve(cudaStream_t st, const PSeg *segs, int nseg, const PChunk *ch, int nch,
                 const PRun *runs, const double *urows, const double *T, const double *r,
                 double *z, double *work_p, double *work_s);

}  // namespace madam
