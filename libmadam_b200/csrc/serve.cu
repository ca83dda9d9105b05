// Serving: a queue of destriping jobs of uneven sizes on one GPU.
//
// Callers submit complete destripe() jobs (the arguments of the reference
// C-ABI, smadam.F90:64-101; float64 signals, or float32 signals for the
// FP32-TOD form of destripe_fp32) and collect their products later.  A fixed
// set of worker threads, the job slots, each owns an engine with its own CUDA
// stream.  A job is admitted when its estimated device footprint fits the
// memory budget next to the jobs already running (the first job in flight is
// always admitted); admission is first come, first served, so a large job at
// the head of the queue holds back smaller ones behind it until memory frees
// up.  A worker runs its job's setup (everything before the PCG) on its
// engine, so the setups of jobs in flight overlap on the device.
//
// Continuous batching of the PCG: the jobs whose setup is done iterate in
// shared rounds driven by one stepper thread.  Per round every job in flight
// takes one PCG iteration: the stepper queues each job's A p (projections,
// filter) and preconditioner on one of a few streams, so the jobs' kernels
// overlap, and runs the CG vector algebra of all jobs in shared launches (one
// kernel each for aa/r/ro, for the inner products, for the CG scalars and for
// p; pcg_shared), then one host synchronisation serves every job's
// convergence test.  Jobs join the rounds when their setup finishes and leave
// when they converge, each with its own CG scalars, iteration count and
// stopping rule.  A job's arithmetic is that of a lone destripe() (same
// kernels, grids and reduction order), so its products do not depend on what
// else is in flight (up to the rounding-level order effects of the setup's
// atomic sums, which differ between any two runs).  Each job's products
// (maps, hits, baselines, scalars) are copied to host memory when it
// finishes, and the worker's engine moves on.  The caller's buffers must stay
// valid until its job is done; host pixel buffers are written back like
// destripe() does.
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
  double setup_ms = 0, iterate_ms = 0, finalize_ms = 0;  // the engine's phases
  bool retried = false;  // requeued once after running out of device memory
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

// A job handed from its worker to the stepper for the PCG rounds.
struct Stepping {
  Engine *eng = nullptr;
  bool done = false, failed = false;
  std::string err;
};

class Server {
 public:
  int device() const { return device_; }
  Server(int nworkers, double frac) {
    MADAM_CUDA(cudaGetDevice(&device_));
    size_t fr = 0, tot = 0;
    MADAM_CUDA(cudaMemGetInfo(&fr, &tot));
    budget_ = (size_t)(frac * (double)fr);
    MADAM_CUDA(cudaStreamCreateWithFlags(&ssm_, cudaStreamNonBlocking));
    MADAM_CUDA(cudaEventCreateWithFlags(&se0_, cudaEventDisableTiming));
    for (int k = 0; k < kStepStreams; ++k) {
      MADAM_CUDA(cudaStreamCreateWithFlags(&ssa_[k], cudaStreamNonBlocking));
      MADAM_CUDA(cudaEventCreateWithFlags(&sek_[k], cudaEventDisableTiming));
    }
    stepper_ = std::thread([this] { stepper(); });
    for (int i = 0; i < nworkers; ++i) threads_.emplace_back([this] { worker(); });
  }
  // rounds, job-rounds (jobs summed over rounds), most jobs in one round
  void stats(double *out) {
    std::lock_guard<std::mutex> lk(smu_);
    out[0] = (double)rounds_;
    out[1] = (double)job_rounds_;
    out[2] = (double)max_round_;
  }
  ~Server() {
    // the workers finish their jobs (whose PCG needs the stepper), then the
    // stepper stops
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_work_.notify_all();
    for (auto &t : threads_) t.join();
    {
      std::lock_guard<std::mutex> lk(smu_);
      sstop_ = true;
    }
    scv_in_.notify_all();
    stepper_.join();
    for (int k = 0; k < kStepStreams; ++k) {
      cudaEventDestroy(sek_[k]);
      cudaStreamDestroy(ssa_[k]);
    }
    cudaEventDestroy(se0_);
    cudaStreamDestroy(ssm_);
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
      Timings tm;
      try {
        if (!eng) eng.reset(new Engine());
        eng->set_fp32(j->fp32);
        eng->run_setup(j->par, j->dets, j->ndet, j->nsamp, j->nnz, j->ts, j->pix, j->w, j->sig,
                       (long)j->periods.size(), j->periods.data(), j->dev);
        if (eng->stepwise_ok() && !stepper_dead_) {
          // the PCG in the stepper's shared rounds
          if (eng->pcg_begin()) {
            Stepping sp;
            sp.eng = eng.get();
            {
              std::lock_guard<std::mutex> lk(smu_);
              incoming_.push_back(&sp);
            }
            scv_in_.notify_all();
            {
              std::unique_lock<std::mutex> lk(smu_);
              scv_done_.wait(lk, [&] { return sp.done; });
            }
            if (sp.failed) throw Error(sp.err);
          }
          eng->pcg_end();
        } else {
          eng->run_solve();
        }
        eng->run_finish();
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
        tm = eng->timings;
        // an engine keeps its buffers for the worker's next job; one sized
        // for a large job gives them back, since the budget counts only the
        // running jobs
        if (j->bytes > budget_ / 8) eng.reset();
      } catch (const std::exception &e) {
        st = 3;
        err = e.what();
        eng.reset();  // a failed job leaves no state behind
        cudaGetLastError();  // an allocation failure is not left pending for the next job
      }
      // the pool keeps the memory of finished jobs for the next ones, but no
      // more than the budget: the rest goes back to the device for other
      // users of the GPU
      {
        int dev = 0;
        cudaMemPool_t pool;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
          cudaMemPoolTrimTo(pool, budget_);
        cudaGetLastError();
      }
      // a job that ran out of device memory (other users of the GPU hold
      // more than the budget assumed) goes back to the head of the queue
      // once, to start when the running jobs leave room
      const bool retry = st == 3 && !j->retried && err.find("out of memory") != std::string::npos;
      if (retry) {
        {
          std::lock_guard<std::mutex> lk(mu_);
          j->retried = true;
          j->state = 0;
          in_flight_ -= j->bytes;
          --running_;
          queue_.push_front(j);
        }
        cv_work_.notify_all();
        continue;
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        j->results = std::move(res);
        j->noiter = noiter;
        j->setup_ms = tm.setup_ms;
        j->iterate_ms = tm.iterate_ms;
        j->finalize_ms = tm.finalize_ms;
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

  // The PCG rounds of the jobs in flight (see the file comment).
  void stepper() {
    constexpr int K = kStepStreams;
    cudaStream_t sm = ssm_, (&sa)[K] = ssa_;
    cudaEvent_t e0 = se0_, (&ek)[K] = sek_;
    if (cudaSetDevice(device_) != cudaSuccess) {
      // the jobs then run their PCG on their own workers; any handed over
      // before this was seen fail
      stepper_dead_ = true;
      for (;;) {
        std::unique_lock<std::mutex> lk(smu_);
        scv_in_.wait(lk, [&] { return sstop_ || !incoming_.empty(); });
        for (Stepping *sp : incoming_) {
          sp->failed = true;
          sp->err = "the PCG stepper could not select the device";
          sp->done = true;
        }
        incoming_.clear();
        scv_done_.notify_all();
        if (sstop_) return;
      }
    }
    g_alloc_stream = sm;
    DevBuf<PcgJob> tab_d;
    DevBuf<double> out_d;
    double *out_h = nullptr;
    size_t cap = 0;
    std::vector<Stepping *> active;
    std::vector<PcgJob> tab;
    auto finish = [&](Stepping *sp, const char *err) {
      std::lock_guard<std::mutex> lk(smu_);
      if (err) {
        sp->failed = true;
        sp->err = err;
      }
      sp->done = true;
    };
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(smu_);
        scv_in_.wait(lk, [&] { return sstop_ || !incoming_.empty() || !active.empty(); });
        for (Stepping *sp : incoming_) active.push_back(sp);
        incoming_.clear();
        if (active.empty() && sstop_) break;
      }
      if (active.empty()) continue;
      const int n = (int)active.size();
      tab.resize(n);
      std::vector<char> stop(n, 0);
      std::vector<std::string> msgs(n);
      std::vector<char> failed(n, 0);
      try {
        if ((size_t)n > cap) {
          if (out_h) cudaFreeHost(out_h);
          out_h = nullptr;
          cap = 0;
          const size_t c = std::max<size_t>(16, 2 * (size_t)n);
          tab_d.alloc(c);
          out_d.alloc(2 * c);
          MADAM_CUDA(cudaMallocHost((void **)&out_h, 2 * c * sizeof(double)));
          cap = c;
        }
        round(active, tab, stop, failed, msgs, sm, sa, e0, ek, tab_d.get(), out_d.get(), out_h);
      } catch (const std::exception &e) {
        // a failure of the shared launches: every job of the round fails
        for (int i = 0; i < n; ++i)
          if (!failed[i]) {
            failed[i] = 1;
            msgs[i] = e.what();
          }
        cudaStreamSynchronize(sm);
        for (int k = 0; k < K; ++k) cudaStreamSynchronize(sa[k]);
      }
      g_alloc_stream = sm;
      {
        std::lock_guard<std::mutex> lk(smu_);
        ++rounds_;
        job_rounds_ += n;
        max_round_ = std::max(max_round_, (long)n);
      }
      std::vector<Stepping *> keep;
      bool any = false;
      for (int i = 0; i < n; ++i) {
        if (failed[i] || stop[i]) {
          active[i]->eng->pcg_use_stream(nullptr);  // back to the job's own stream
          g_alloc_stream = sm;
          finish(active[i], failed[i] ? msgs[i].c_str() : nullptr);
          any = true;
        } else {
          keep.push_back(active[i]);
        }
      }
      active.swap(keep);
      if (any) scv_done_.notify_all();
    }
    if (out_h) cudaFreeHost(out_h);
    tab_d.reset();
    out_d.reset();
    cudaStreamSynchronize(sm);
  }

  // One PCG round of the jobs in `act`: A p of each job on the K job streams,
  // aa, r and ro of all in one launch, z = M r of each, the inner products
  // and CG scalars of all in two launches, one synchronisation, each job's
  // convergence test, then p of those that go on in one launch.  A job whose
  // own step throws is marked in `failed` and left out of the rest.
  template <int K>
  void round(const std::vector<Stepping *> &act, std::vector<PcgJob> &tab,
             std::vector<char> &stop, std::vector<char> &failed, std::vector<std::string> &msgs,
             cudaStream_t sm, cudaStream_t (&sa)[K], cudaEvent_t e0, cudaEvent_t (&ek)[K],
             PcgJob *tab_d, double *out_d, double *out_h) {
    const int n = (int)act.size();
    long long nbmax = 1;
    for (int i = 0; i < n; ++i) {
      act[i]->eng->pcg_use_stream(sa[i % K]);
      tab[i] = act[i]->eng->pcg_job();
      nbmax = std::max(nbmax, tab[i].nb);
    }
    auto fork = [&]() {  // the job streams wait for the main stream
      MADAM_CUDA(cudaEventRecord(e0, sm));
      for (int k = 0; k < K; ++k) MADAM_CUDA(cudaStreamWaitEvent(sa[k], e0, 0));
    };
    auto join = [&]() {  // and the main stream for them
      for (int k = 0; k < K; ++k) {
        MADAM_CUDA(cudaEventRecord(ek[k], sa[k]));
        MADAM_CUDA(cudaStreamWaitEvent(sm, ek[k], 0));
      }
    };
    auto each = [&](auto &&f) {  // a job's own step; a failure drops the job
      for (int i = 0; i < n; ++i) {
        if (failed[i] || stop[i]) continue;
        try {
          f(i);
        } catch (const std::exception &e) {
          msgs[i] = e.what();
          failed[i] = 1;
          tab[i].active = 0;
        }
      }
    };
    auto upload = [&]() {
      MADAM_CUDA(cudaMemcpyAsync(tab_d, tab.data(), n * sizeof(PcgJob), cudaMemcpyHostToDevice,
                                 sm));
    };
    fork();
    each([&](int i) { act[i]->eng->pcg_apply(); });
    join();
    upload();
    pcg_shared(sm, tab_d, n, nbmax, 0, nullptr);
    fork();
    each([&](int i) { act[i]->eng->pcg_precond(); });
    join();
    upload();
    pcg_shared(sm, tab_d, n, nbmax, 1, out_d);
    MADAM_CUDA(cudaMemcpyAsync(out_h, out_d, 2 * n * sizeof(double), cudaMemcpyDeviceToHost, sm));
    MADAM_CUDA(cudaStreamSynchronize(sm));
    each([&](int i) {
      stop[i] = act[i]->eng->pcg_after(out_h[2 * i], out_h[2 * i + 1]) ? 1 : 0;
      if (stop[i]) tab[i].active = 0;
    });
    join();  // the reliable updates a convergence test may run
    upload();
    pcg_shared(sm, tab_d, n, nbmax, 2, nullptr);
    MADAM_CUDA(cudaStreamSynchronize(sm));
  }

  static constexpr int kStepStreams = 4;  // streams the jobs' own kernels spread over
  cudaStream_t ssm_ = nullptr, ssa_[kStepStreams] = {};
  cudaEvent_t se0_ = nullptr, sek_[kStepStreams] = {};
  std::atomic<bool> stepper_dead_{false};
  std::thread stepper_;
  std::mutex smu_;
  std::condition_variable scv_in_, scv_done_;
  std::vector<Stepping *> incoming_;
  bool sstop_ = false;
  long rounds_ = 0, job_rounds_ = 0, max_round_ = 0;

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
    if (nnz != 1 && nnz != 3) madam::fail("only nnz = 1 or nnz = 3 is supported");
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
  if (nout >= 9) {
    out[6] = j->setup_ms;
    out[7] = j->iterate_ms;
    out[8] = j->finalize_ms;
  }
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

int madam_b200_serve_stats(void *srv, double *out, long nout) {
  Server *s = (Server *)srv;
  if (!s || nout < 3) return 1;
  s->stats(out);
  return 0;
}

int madam_b200_serve_close(void *srv) {
  delete (Server *)srv;
  return 0;
}

}  // extern "C"
