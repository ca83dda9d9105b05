// Communicators of sharded runs (comm.h) and their C-ABI.
#include "comm.h"

#include <dlfcn.h>
#include <nccl.h>

#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "params.h"

namespace madam {
namespace {

// NCCL entry points, resolved from libnccl.so.2 on first use so that single-
// GPU runs do not depend on it
struct NcclApi {
  ncclResult_t (*get_unique_id)(ncclUniqueId *) = nullptr;
  ncclResult_t (*comm_init_rank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*all_reduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t,
                             ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
  const char *(*error_string)(ncclResult_t) = nullptr;
};

const NcclApi &nccl() {
  static NcclApi api;
  static std::once_flag once;
  static std::string err;
  std::call_once(once, [] {
    void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
    if (!h) {
      err = std::string("cannot load libnccl.so.2: ") + dlerror();
      return;
    }
    api.get_unique_id = (decltype(api.get_unique_id))dlsym(h, "ncclGetUniqueId");
    api.comm_init_rank = (decltype(api.comm_init_rank))dlsym(h, "ncclCommInitRank");
    api.all_reduce = (decltype(api.all_reduce))dlsym(h, "ncclAllReduce");
    api.comm_destroy = (decltype(api.comm_destroy))dlsym(h, "ncclCommDestroy");
    api.error_string = (decltype(api.error_string))dlsym(h, "ncclGetErrorString");
    if (!api.get_unique_id || !api.comm_init_rank || !api.all_reduce || !api.comm_destroy ||
        !api.error_string) {
      api = NcclApi();
      err = "libnccl.so.2 lacks an entry point";
    }
  });
  if (!api.all_reduce) fail(err);
  return api;
}

void nccl_check(ncclResult_t r, const char *what) {
  if (r != ncclSuccess) fail(std::string(what) + ": " + nccl().error_string(r));
}

class NcclComm : public Comm {
 public:
  NcclComm(int r, int n, const ncclUniqueId &id) {
    rank = r;
    nranks = n;
    nccl_check(nccl().comm_init_rank(&comm_, n, id, r), "ncclCommInitRank");
  }
  ~NcclComm() override {
    if (comm_) nccl().comm_destroy(comm_);
  }
  void allreduce(double *dev, size_t n, int op, cudaStream_t st) override {
    if (n == 0) return;
    nccl_check(nccl().all_reduce(dev, dev, n, ncclFloat64, op ? ncclMax : ncclSum, comm_, st),
               "ncclAllReduce");
  }
  void allreduce(int *dev, size_t n, int op, cudaStream_t st) override {
    if (n == 0) return;
    nccl_check(nccl().all_reduce(dev, dev, n, ncclInt32, op ? ncclMax : ncclSum, comm_, st),
               "ncclAllReduce");
  }

 private:
  ncclComm_t comm_ = nullptr;
};

class HostComm : public Comm {
 public:
  HostComm(int r, int n, HostAllreduce fn) : fn_(fn) {
    rank = r;
    nranks = n;
  }
  void allreduce(double *dev, size_t n, int op, cudaStream_t st) override {
    if (n == 0) return;
    buf_.resize(n);
    MADAM_CUDA(cudaMemcpyAsync(buf_.data(), dev, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    MADAM_CUDA(cudaStreamSynchronize(st));
    fn_(buf_.data(), (long)n, op);
    MADAM_CUDA(cudaMemcpyAsync(dev, buf_.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    MADAM_CUDA(cudaStreamSynchronize(st));
  }
  void allreduce(int *dev, size_t n, int op, cudaStream_t st) override {
    if (n == 0) return;
    std::vector<int> iv(n);
    MADAM_CUDA(cudaMemcpyAsync(iv.data(), dev, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    MADAM_CUDA(cudaStreamSynchronize(st));
    buf_.assign(iv.begin(), iv.end());  // counts are exact in double
    fn_(buf_.data(), (long)n, op);
    for (size_t i = 0; i < n; ++i) iv[i] = (int)buf_[i];
    MADAM_CUDA(cudaMemcpyAsync(dev, iv.data(), n * sizeof(int), cudaMemcpyHostToDevice, st));
    MADAM_CUDA(cudaStreamSynchronize(st));
  }

 private:
  HostAllreduce fn_;
  std::vector<double> buf_;
};

std::mutex g_comm_mu;
std::map<int, std::unique_ptr<Comm>> g_comms;
// Library handles start far from the values MPI libraries give Fortran
// communicator handles (Open MPI: small table indices, MPI_COMM_WORLD = 0,
// MPI_COMM_SELF = 1; MPICH: bit patterns 0x44000000 and up for the built-in
// communicators, negative as int for created ones), so an MPI handle passed
// as `comm` is never taken for one of this library's communicators.
constexpr int kFirstHandle = 0x2D420001;
int g_next_handle = kFirstHandle;
std::string g_comm_err;

int add(Comm *c) {
  std::lock_guard<std::mutex> lk(g_comm_mu);
  const int h = g_next_handle++;
  g_comms[h].reset(c);
  return h;
}

}  // namespace

Comm *comm_lookup(int handle) {
  std::lock_guard<std::mutex> lk(g_comm_mu);
  auto it = g_comms.find(handle);
  return it == g_comms.end() ? nullptr : it->second.get();
}

}  // namespace madam

extern "C" {

int madam_b200_comm_error(char *buf, long len) {
  if (buf && len > 0) {
    std::strncpy(buf, madam::g_comm_err.c_str(), (size_t)len - 1);
    buf[len - 1] = '\0';
  }
  return madam::g_comm_err.empty() ? 0 : 1;
}

int madam_b200_comm_nccl_id(char *id) {
  try {
    ncclUniqueId u;
    madam::nccl_check(madam::nccl().get_unique_id(&u), "ncclGetUniqueId");
    std::memcpy(id, u.internal, sizeof u.internal);
    madam::g_comm_err.clear();
    return 0;
  } catch (const std::exception &e) {
    madam::g_comm_err = e.what();
    return 1;
  }
}

int madam_b200_comm_init_nccl(int rank, int nranks, const char *id) {
  try {
    if (nranks < 1 || rank < 0 || rank >= nranks) madam::fail("invalid rank / nranks");
    ncclUniqueId u;
    std::memcpy(u.internal, id, sizeof u.internal);
    madam::g_comm_err.clear();
    return madam::add(new madam::NcclComm(rank, nranks, u));
  } catch (const std::exception &e) {
    madam::g_comm_err = e.what();
    return -1;
  }
}

int madam_b200_comm_init_host(int rank, int nranks, madam::HostAllreduce fn) {
  if (!fn || nranks < 1 || rank < 0 || rank >= nranks) {
    madam::g_comm_err = "invalid rank / nranks or no all-reduce function";
    return -1;
  }
  madam::g_comm_err.clear();
  return madam::add(new madam::HostComm(rank, nranks, fn));
}

int madam_b200_comm_free(int handle) {
  std::lock_guard<std::mutex> lk(madam::g_comm_mu);
  return madam::g_comms.erase(handle) ? 0 : 1;
}

}  // extern "C"
