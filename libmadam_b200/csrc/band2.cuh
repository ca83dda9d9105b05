// Deduplicated band Cholesky factor and chunk-parallel solve (band2.cu).
#pragma once

#include <cuda_runtime.h>

namespace madam {

// One factored segment of n baselines with band width nb = w + 1.
// Coefficient entries are nb + 1 doubles: the nb band values and the
// reciprocal of the first one.
struct PSeg {
  long long k0;       // first baseline of the segment
  long long row_off;  // offset (doubles) of its entry table while factoring
  int n;              // rows
  int nb;             // band width (w + 1)
  int run_off, nrun;  // forward runs (rows of L, position p = row j)
  int crun_off, ncrun;  // backward runs (columns of L, position p = n - 1 - j)
  int ch_off, nch;    // chunks
};

// Positions [start, next run's start) of one direction share the entry at
// off.  fill = 1 marks a backward entry that a kernel assembles from rows.
struct PRun {
  int start;
  int fill;
  long long off;
};

// Rows [a, b) of segment seg; the forward pass visits them ascending, the
// backward pass descending.
struct PChunk {
  int seg, a, b;
  int run_f;   // forward run containing row a
  int run_b;   // backward run containing position n - b (row b - 1)
  int first, last;
  int tf, tb;  // offsets (doubles) of the forward / backward transfer matrices
};

struct PTrans {
  int chunk;  // representative chunk
  int dir;    // 0 forward, 1 backward
  long long off;  // offset of the w x w matrix
};

// A chunk of the guarded solve: rows [a, b) of segment seg.  The forward
// recurrence starts from a zero state at row ga <= a (in forward run run_fg)
// and writes rows a .. b-1; the backward one starts at backward position
// gp <= n - b (in backward run run_bg) and writes positions n-b .. n-a-1
// (rows b-1 .. a).  The guard (a - ga, n - b - gp positions) is checked at
// set-up: the response of the first written position's state to a unit
// state at the guard start is below kBand2GuardTol in every entry, so the
// zero start differs from the true state by less than that relative amount.
struct GChunk {
  int seg, a, b;
  int ga, run_fg, run_fa;  // forward guard start, runs containing ga and a
  int gp, run_bg, run_bb;  // backward guard start, runs containing gp and n - b
};
constexpr double kBand2GuardTol = 1e-20;

constexpr int kBand2MaxWidth = 128;
constexpr int kBand2State = 128;  // doubles per chunk state slot (>= w)

// Factor one segment per warp; rows: worst case n * (nb + 1) doubles at
// seg.row_off, runs: worst case n at seg.run_off.
void band2_factor(cudaStream_t st, const PSeg *segs, int nseg, const int *spec,
                  const double *invcov, long long nof, const double *nna, double *rows,
                  PRun *runs, int *status, int *nunique, int *nruns);
// Assemble the backward entries flagged in the column runs.
void band2_columns(cudaStream_t st, const PSeg *segs, int nseg, int max_ncrun, const PRun *runs,
                   const PRun *cruns, double *tab);
// Transfer matrices; tcls_begin: transfer ranges of the width classes.
void band2_transfer(cudaStream_t st, const PSeg *segs, const PChunk *ch, const PTrans *tr,
                    const int *cls_w, const int *tcls_begin, int ncls, const PRun *runs,
                    const PRun *cruns, const double *tab, double *T);
// Solve L L^T z = r on every factored segment.  Width class i: chunks
// [cls_begin[i], cls_begin[i + 1]) of segments [cls_seg[i], cls_seg[i + 1])
// with w <= cls_w[i] (host arrays).
// toff_f / toff_b: the chunks' forward / backward transfer offsets (device).
void band2_solve(cudaStream_t st, const PSeg *segs, int nseg, const PChunk *ch, int nch,
                 const int *toff_f, const int *toff_b, const int *cls_w, const int *cls_begin,
                 const int *cls_seg, int ncls, const PRun *runs, const PRun *cruns,
                 const double *tab, const double *T, const double *r, double *z, double *work_p,
                 double *work_s);
// Smallest compiled register width >= w (0 when w needs the generic path).
int band2_class_width(int w);

// Guard check: worst[c] = the largest entry, over both directions, of the
// response at guarded chunk c's first written position to a unit state at its
// guard start (0 for chunks without a guard).  Width class i: guarded chunks
// [gcls_begin[i], gcls_begin[i + 1]) with w <= cls_w[i] (host arrays).
void band2_guard_check(cudaStream_t st, const PSeg *segs, const GChunk *gc, const int *cls_w,
                       const int *gcls_begin, int ncls, const PRun *runs, const PRun *cruns,
                       const double *tab, double *worst);
// Solve L L^T z = r on every factored segment with the guarded chunks: one
// forward launch (r -> y) and one backward launch (y -> z) per width class;
// no state propagation.  Register widths only (cls_w[i] > 0).  *err (device)
// becomes nonzero if a staging wait ran out (the result is then invalid).
void band2_solve_guarded(cudaStream_t st, const PSeg *segs, const GChunk *gc, const int *cls_w,
                         const int *gcls_begin, int ncls, const PRun *runs, const PRun *cruns,
                         const double *tab, const double *r, double *y, double *z, int *err);

}  // namespace madam
