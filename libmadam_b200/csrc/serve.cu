// Serving: a queue of destriping jobs of uneven sizes on one GPU.
//
// Callers submit complete destripe() jobs (the arguments of the reference
// C-ABI, smadam.F90:64-101; float64 signals, or float32 signals for the
// FP32-TOD form of destripe_fp32) and collect their products later.  A fixed set
// of worker threads each owns an engine with its own CUDA stream, so jobs in
// flight overlap on the device.  A job is admitted when its estimated device
// footprint fits the memory budget next to the jobs already running (the
// first job in flight is always admitted); admission is first come, first
// served, so a large job at the head of the queue holds back smaller ones
// behind it until memory frees up.  Every job runs the kernels of a lone
// destripe() on its own engine, so its products do not depend on what else
// is in flight (up to the rounding-level order effects of the setup's
// atomic sums, which differ between any two runs).  Each job's products (maps, hits, baselines, scalars) are
// copied to host memory when it finishes, and the worker's engine moves on.
// The caller's buffers must stay valid until its job is done; host pixel
// buffers are written back like destripe() does.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"
#include "params.h"

namespace madam {
namespace {

double wall_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Job {
  long id = 0;
  Params par;
  std::vector<Detector> dets;
  long ndet = 0, nsamp = 0, nnz = 0;
  double *ts = nullptr;
  int32_t *pix = nullptr;
  float *w = nullptr;
  double *sig = nullptr;
  std::vector<long> periods;
  bool dev = false;
  bool fp32 = false;  // float32 signal: the FP32-TOD form (destripe_fp32)
  size_t bytes = 0;
  int state = 0;  // 0 queued, 1 running, 2 done, 3 failed
  std::string error;
  double t_submit = 0, t_start = 0, t_end = 0;
  std::map<std::string, std::vector<char>> results;
  double noiter = 0;
};

// device memory of a job, from the engine's buffers per sample / baseline
size_t job_bytes(const Job &j) {
  const double n = (double)j.ndet * j.nsamp;
  const double dn = std::max(1.0, std::min(j.par.dnshort, 1e9));
  const double nb = n / dn + j.ndet;
  const double npix = 12.0 * j.par.nside_map * j.par.nside_map;
  double b = n * (j.dev ? 64.0 : 84.0) + nb * 8.0 * 24 + npix * 8.0 * 24 + (256 << 20);
  if (j.fp32) b += n * (j.dev ? 40.0 : 44.0);  // pairs, their sort and the float32 staging
  return (size_t)b;
}

class Server {
 public:
  int device() const { return device_; }
  Server(int nworkers, double frac) {
    MADAM_CUDA(cudaGetDevice(&device_));
    size_t fr = 0, tot = 0;
    MADAM_CUDA(cudaMemGetInfo(&fr, &tot));
    budget_ = (size_t)(frac * (double)fr);
    for (int i = 0; i < nworkers; ++i) threads_.emplace_back([this] { worker(); });
  }
  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_work_.notify_all();
    for (auto &t : threads_) t.join();
  }
  long submit(std::unique_ptr<Job> j) {
    std::lock_guard<std::mutex> lk(mu_);
    const long id = next_id_++;
    j->id = id;
    j->t_submit = wall_s();
    queue_.push_back(j.get());
    jobs_[id] = std::move(j);
    cv_work_.notify_all();
    return id;
  }
  int wait(long id, double timeout_s) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = jobs_.find(id);
    if (it == jobs_.end()) return -1;
    Job *j = it->second.get();
    auto done = [&] { return j->state >= 2; };
    if (timeout_s < 0) cv_done_.wait(lk, done);
    else cv_done_.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
    return j->state;
  }
  Job *get(long id) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = jobs_.find(id);
    return (it == jobs_.end() || it->second->state < 2) ? nullptr : it->second.get();
  }
  int release(long id) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = jobs_.find(id);
    if (it == jobs_.end() || it->second->state < 2) return 1;
    jobs_.erase(it);
    return 0;
  }
  std::string last_error;

 private:
  void worker() {
    MADAM_CUDA(cudaSetDevice(device_));
    std::unique_ptr<Engine> eng;
    for (;;) {
      Job *j = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_work_.wait(lk, [&] {
          if (stop_) return true;
          if (queue_.empty()) return false;
          const Job *h = queue_.front();
          return running_ == 0 || in_flight_ + h->bytes <= budget_;
        });
        if (stop_) return;
        j = queue_.front();
        queue_.pop_front();
        in_flight_ += j->bytes;
        ++running_;
        j->state = 1;
        j->t_start = wall_s();
      }
      int st = 2;
      std::string err;
      std::map<std::string, std::vector<char>> res;
      double noiter = 0;
      try {
        if (!eng) eng.reset(new Engine());
        eng->set_fp32(j->fp32);
        eng->run(j->par, j->dets, j->ndet, j->nsamp, j->nnz, j->ts, j->pix, j->w, j->sig,
                 (long)j->periods.size(), j->periods.data(), j->dev);
        for (const char *nm : {"map", "binmap", "hits", "mask", "aa", "scalars", "rr_history"}) {
          const long sz = eng->result_size(nm);
          const size_t el = (std::strcmp(nm, "hits") == 0 || std::strcmp(nm, "mask") == 0)
                                ? sizeof(int)
                                : sizeof(double);
          std::vector<char> buf((size_t)std::max<long>(0, sz) * el);
          if (sz > 0) eng->result_copy(nm, buf.data(), (long)buf.size());
          res[nm] = std::move(buf);
        }
        noiter = (double)eng->noiter;
      } catch (const std::exception &e) {
        st = 3;
        err = e.what();
        eng.reset();  // a failed job leaves no state behind
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        j->results = std::move(res);
        j->noiter = noiter;
        j->error = err;
        j->t_end = wall_s();
        j->state = st;
        in_flight_ -= j->bytes;
        --running_;
      }
      cv_done_.notify_all();
      cv_work_.notify_all();
    }
  }

  int device_ = 0;
  size_t budget_ = 0, in_flight_ = 0;
  int running_ = 0;
  long next_id_ = 0;
  bool stop_ = false;
  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_;
  std::deque<Job *> queue_;
  std::map<long, std::unique_ptr<Job>> jobs_;
  std::vector<std::thread> threads_;
};

void set_msg(char *buf, long len, const std::string &m) {
  if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", m.c_str());
}

}  // namespace
}  // namespace madam

using madam::Job;
using madam::Server;

extern "C" {

void *madam_b200_serve_open(int nworkers, double mem_fraction, char *err, long errlen) {
  try {
    if (nworkers < 1 || nworkers > 64) madam::fail("nworkers must be in 1..64");
    if (!(mem_fraction > 0 && mem_fraction <= 1)) madam::fail("mem_fraction must be in (0, 1]");
    return new Server(nworkers, mem_fraction);
  } catch (const std::exception &e) {
    madam::set_msg(err, errlen, e.what());
    return nullptr;
  }
}

static long serve_submit(bool fp32, void *srv, char *parstring, long ndet, char *detstring,
                         double *detweights, long nsamp, long nnz, void *timestamps, void *pix,
                         void *pixweights, void *signal, long nperiod, long *periods, long *npsd,
                         long npsdtot, double *psdstarts, long npsdbin, double *psdfreqs,
                         long npsdval, double *psdvals, char *err, long errlen);

long madam_b200_serve_submit(void *srv, char *parstring, long ndet, char *detstring,
                             double *detweights, long nsamp, long nnz, void *timestamps, void *pix,
                             void *pixweights, void *signal, long nperiod, long *periods,
                             long *npsd, long npsdtot, double *psdstarts, long npsdbin,
                             double *psdfreqs, long npsdval, double *psdvals, char *err,
                             long errlen) {
  return serve_submit(false, srv, parstring, ndet, detstring, detweights, nsamp, nnz, timestamps,
                      pix, pixweights, signal, nperiod, periods, npsd, npsdtot, psdstarts,
                      npsdbin, psdfreqs, npsdval, psdvals, err, errlen);
}

long madam_b200_serve_submit_fp32(void *srv, char *parstring, long ndet, char *detstring,
                                  double *detweights, long nsamp, long nnz, void *timestamps,
                                  void *pix, void *pixweights, float *signal, long nperiod,
                                  long *periods, long *npsd, long npsdtot, double *psdstarts,
                                  long npsdbin, double *psdfreqs, long npsdval, double *psdvals,
                                  char *err, long errlen) {
  return serve_submit(true, srv, parstring, ndet, detstring, detweights, nsamp, nnz, timestamps,
                      pix, pixweights, signal, nperiod, periods, npsd, npsdtot, psdstarts,
                      npsdbin, psdfreqs, npsdval, psdvals, err, errlen);
}

static long serve_submit(bool fp32, void *srv, char *parstring, long ndet, char *detstring,
                         double *detweights, long nsamp, long nnz, void *timestamps, void *pix,
                         void *pixweights, void *signal, long nperiod, long *periods, long *npsd,
                         long npsdtot, double *psdstarts, long npsdbin, double *psdfreqs,
                         long npsdval, double *psdvals, char *err, long errlen) {
  Server *s = (Server *)srv;
  if (!s) return -1;
  try {
    std::unique_ptr<Job> j(new Job());
    j->par = madam::parse_parstring(parstring);
    if (j->par.mcmode) madam::fail("mcmode jobs are not served");
    if (j->par.nsubchunk > 1) madam::fail("nsubchunk > 1 jobs are not served");
    if (j->par.temperature_only && nnz != 1)
      madam::fail("temperature_only=T but pointing weights are polarized");
    if (ndet <= 0 || nsamp <= 0 || nnz <= 0) madam::fail("empty data");
    j->dets = madam::read_detectors(j->par, detstring, ndet, detweights, npsd, npsdtot,
                                    psdstarts, npsdbin, psdfreqs, npsdval, psdvals);
    j->ndet = ndet;
    j->nsamp = nsamp;
    j->nnz = nnz;
    j->ts = (double *)timestamps;
    j->pix = (int32_t *)pix;
    j->w = (float *)pixweights;
    j->sig = (double *)signal;
    j->periods.assign(periods, periods + nperiod);
    j->dev = madam::inputs_on_device(s->device(), {timestamps, pix, pixweights, signal});
    j->fp32 = fp32;
    j->bytes = madam::job_bytes(*j);
    return s->submit(std::move(j));
  } catch (const std::exception &e) {
    madam::set_msg(err, errlen, e.what());
    return -1;
  }
}

int madam_b200_serve_wait(void *srv, long job, double timeout_s) {
  Server *s = (Server *)srv;
  return s ? s->wait(job, timeout_s) : -1;
}

long madam_b200_serve_result_size(void *srv, long job, const char *name) {
  Server *s = (Server *)srv;
  Job *j = s ? s->get(job) : nullptr;
  if (!j || j->state != 2) return -1;
  auto it = j->results.find(name);
  if (it == j->results.end()) return -1;
  const bool ints = std::strcmp(name, "hits") == 0 || std::strcmp(name, "mask") == 0;
  return (long)(it->second.size() / (ints ? sizeof(int) : sizeof(double)));
}

int madam_b200_serve_result_copy(void *srv, long job, const char *name, void *dst, long nbytes) {
  Server *s = (Server *)srv;
  Job *j = s ? s->get(job) : nullptr;
  if (!j || j->state != 2) return 1;
  auto it = j->results.find(name);
  if (it == j->results.end() || (size_t)nbytes < it->second.size()) return 1;
  std::memcpy(dst, it->second.data(), it->second.size());
  return 0;
}

int madam_b200_serve_job_info(void *srv, long job, double *out, long nout) {
  Server *s = (Server *)srv;
  Job *j = s ? s->get(job) : nullptr;
  if (!j || nout < 6) return 1;
  out[0] = j->t_submit;
  out[1] = j->t_start;
  out[2] = j->t_end;
  out[3] = (double)j->ndet * j->nsamp;
  out[4] = j->noiter;
  out[5] = (double)j->bytes;
  return 0;
}

int madam_b200_serve_error(void *srv, long job, char *buf, long buflen) {
  Server *s = (Server *)srv;
  Job *j = s ? s->get(job) : nullptr;
  if (!j) return 1;
  madam::set_msg(buf, buflen, j->error);
  return j->state == 3 ? 1 : 0;
}

int madam_b200_serve_release(void *srv, long job) {
  Server *s = (Server *)srv;
  return s ? s->release(job) : 1;
}

int madam_b200_serve_close(void *srv) {
  delete (Server *)srv;
  return 0;
}

}  // extern "C"
