// Communicators of runs sharded over several ranks (one process per GPU),
// standing in for the reference's MPI communicator (mpi_wrappers.f90).
//
// Every rank holds its own share of the TOD (detectors and/or time spans)
// and the whole map; the reference's reductions (collect_map, collect_cc,
// collect_hits, sum_mpi of inner products and counts) become in-place
// all-reduces of device buffers on the engine's stream.  Two kinds:
//   NCCL  device all-reduce over NVLink / NVSwitch (libnccl.so.2, loaded on
//         first use), one rank per GPU;
//   host  the caller's function all-reduces a host buffer (the engine copies
//         the device buffer out and back); used with a CPU process group,
//         e.g. to run the sharded path with several ranks on one GPU.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace madam {

typedef void (*HostAllreduce)(double *buf, long n, int op);  // op 0 sum, 1 max

class Comm {
 public:
  virtual ~Comm() {}
  int rank = 0, nranks = 1;
  // in place, op 0 = sum, 1 = max, ordered on stream st
  virtual void allreduce(double *dev, size_t n, int op, cudaStream_t st) = 0;
  virtual void allreduce(int *dev, size_t n, int op, cudaStream_t st) = 0;
};

// The communicator registered under handle (madam_b200_comm_init_*), or
// nullptr: handle 0 and unknown handles mean a single rank.
Comm *comm_lookup(int handle);

}  // namespace madam
