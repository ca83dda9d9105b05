"""Benchmark of the B200 destriping solve.

Metric: TOD samples per second per PCG iteration (N_samples / t_iteration)
on the "plain destripe on one B200" workload: nside 512, nside_submap 16,
16 detectors x 4 observations x 2^23 samples at 100 Hz, IQU, 1/f noise
(fknee 0.05 Hz, alpha -1.5), base_first 0.5 s, kfilter, cglimit 1e-12.
Synthetic inputs of that shape are generated on the GPU with a fixed seed.

  value      device-resident PCG iterations (bench_iterations through the
             C-ABI), CUDA events on the library's stream, max over ranks
  e2e        destripe() through the C-ABI with pinned HOST buffers: host->
             device copies, setup, PCG to cglimit and the read-back of the map
             inside the timed region; samples x iterations / wall time, the
             mean of E2E_STEPS calls after one untimed call
  roofline   dominant kernel of the iteration against measured HBM bandwidth
  cpu_baseline  the CPU oracle (C++/OpenMP restatement of the reference;
             the Fortran reference cannot be built here) on a bounded sample

--impl reference times that CPU restatement alone (the reference arm).
Multi-GPU: by default every rank solves its own replica; with --sharded the
ranks run one solve sharded by detector (maps and inner products summed over
NCCL every iteration).  value is the sum over ranks divided by the slowest
rank's time.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
E2E_STEPS = 3

import numpy as np  # noqa: E402


def profiled_traffic(kernel, nsamp):
    """DRAM bytes of one launch of `kernel` at `nsamp` samples, from the committed ncu
    summary (bytes per sample of a smaller capture; traffic grows with the samples)."""
    import re
    for size in ("prof", "mid"):
        try:
            with open(os.path.join(ROOT, "profiles", "%s_%s.md" % (kernel, size))) as f:
                m = re.search(r"dram_bytes_per_sample = ([0-9.]+) B", f.read())
            if m:
                return float(m.group(1)) * nsamp
        except OSError:
            pass
    return None


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + q,
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def config_for(name):
    from libmadam_b200 import synthetic as syn
    if name == "2":
        return syn.config2(), "plain destripe nside512 16det x 4obs x 2^23 @100Hz IQU"
    if name == "1":
        return syn.config1(), "plain destripe nside64 4det x 2^20 @10Hz IQU"
    if name == "3":
        return syn.config3(), ("precision form (float32 TOD, destripe_fp32) nside1024 "
                               "64det x 2^24 @100Hz IQU")
    if name == "mid3":
        cfg = syn.config3()
        cfg.ndet = 16
        cfg.nsamp_obs = 1 << 21
        return cfg, "precision form nside1024 16det x 2^21 @100Hz IQU (profiling size)"
    if name == "prof":
        cfg = syn.config2()
        cfg.nobs = 1
        return cfg, "nside512 16det x 1obs x 2^23 @100Hz IQU (per-segment shapes of config 2)"
    if name == "mid":
        cfg = syn.config2()
        cfg.nobs = 1
        cfg.nsamp_obs = 1 << 21
        return cfg, "nside512 16det x 1obs x 2^21 @100Hz IQU (profiling size)"
    cfg = syn.small_config(ndet=4, nsamp_obs=1 << 18, nobs=2, nside=64, seed=5)
    return cfg, "small ring scan nside64 4det x 2 x 2^18"


def cpu_sample_config(cfg):
    """A bounded sample of the workload for the CPU restatement: the first
    group of 4 detectors (0/45/90/135 deg) over the first observation."""
    from libmadam_b200 import synthetic as syn
    s = syn.ScanConfig(**{k: getattr(cfg, k) for k in cfg.__dataclass_fields__})
    s.ndet = min(4, cfg.ndet)
    s.nobs = 1
    s.extra_pars = dict(cfg.extra_pars)
    return s


def run_cpu(cfg, full=False, parity_fp32=None):
    """Time the CPU restatement: samples/s per PCG iteration, on the bounded
    sample (cpu_sample_config) or, with full=True, on the whole workload.
    With parity_fp32 set (False: destripe, True: destripe_fp32 on the float32
    signal), the GPU library then solves the same inputs and the result
    carries a "parity" block: hits and masks equal, per-pixel errors of the
    destriped map and baselines against the oracle (tests/parity.py), PCG
    iteration counts."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    from libmadam_b200 import synthetic as syn
    s = cfg if full else cpu_sample_config(cfg)
    dev = "cuda" if _has_cuda() else "cpu"
    d = syn.to_numpy(syn.generate(s, device=dev))
    keep = None
    if parity_fp32 is not None:
        if parity_fp32:  # the oracle solves the float32 samples the GPU gets
            d["signal"] = d["signal"].astype(np.float32).astype(np.float64)
        keep = {k: d[k].copy() for k in ("pixels", "signal")}
    O.destripe(d["pars"], d["dets"], d["detweights"], d["timestamps"], d["pixels"],
               d["pixweights"], d["signal"], d["periods"], d["npsd"], d["psdstarts"],
               d["psdfreqs"], d["psdvals"])
    sc = O.scalars()
    n = s.ndet * s.nsamp
    it = max(1, int(sc["noiter"]))
    t_iter = sc["t_iterate"] / it
    what = "the whole workload" if full else "{} detectors x {} samples of the workload".format(
        s.ndet, s.nsamp)
    out = {"value": n / t_iter, "unit": "samples/s per PCG iteration",
           "cores": int(sc["nthreads"]), "kind": "port",
           "sample": "{} ({} PCG iterations, {:.1f} ms/iteration, setup+solve {:.1f} s)".format(
               what, it, 1e3 * t_iter, sc["t_total"]),
           "iterations": it, "ms_per_iteration": 1e3 * t_iter,
           "time_to_cglimit_ms": 1e3 * sc["t_iterate"], "destripe_s": sc["t_total"]}
    if parity_fp32 is not None:
        out["parity"] = gpu_parity(O, d, keep, it, parity_fp32, what)
    return out


def gpu_parity(O, d, keep, oracle_iters, fp32, what):
    """GPU destripe (or destripe_fp32) of the inputs the oracle just solved,
    compared with the oracle's products."""
    import parity
    from libmadam_b200 import libmadam_wrapper as W
    ro = {k: O.result(k) for k in ("map", "hits", "mask", "aa")}
    sig = keep["signal"].astype(np.float32) if fp32 else keep["signal"]
    (W.destripe_fp32 if fp32 else W.destripe)(
        None, d["pars"], d["dets"], d["detweights"], d["timestamps"], keep["pixels"],
        d["pixweights"], sig, d["periods"], d["npsd"], d["psdstarts"], d["psdfreqs"],
        d["psdvals"])
    mp = W.get_result("map").reshape(-1, 3)
    mo = ro["map"].reshape(-1, 3)
    floor = parity.FP32_FLOOR if fp32 else parity.FLOOR
    err = lambda a, b: parity.per_pixel_error(a, b, floor)[0]
    it = int(W.scalars()["noiter"])
    tol = 1e-4 if fp32 else 1e-6
    out = {"sample": what + (", float32 TOD against the float64 oracle" if fp32 else ""),
           "hits_equal": bool(np.array_equal(W.get_result("hits"), ro["hits"])),
           "mask_equal": bool(np.array_equal(W.get_result("mask"), ro["mask"])),
           "pixels_equal": bool(np.array_equal(keep["pixels"], d["pixels"])),
           "map_max_rel_err_iqu": [err(mp[:, c], mo[:, c]) for c in range(3)],
           "baseline_max_rel_err": err(W.get_result("aa"), ro["aa"]),
           "iters": [it, oracle_iters], "iters_equal": it == oracle_iters,
           "tolerance": tol,
           "error_definition": "max |gpu - oracle| / max(|oracle|, {:g} max|oracle|) per "
                               "pixel (per baseline)".format(floor)}
    out["pass"] = bool(out["hits_equal"] and out["mask_equal"] and out["pixels_equal"]
                       and max(out["map_max_rel_err_iqu"]) <= tol
                       and out["baseline_max_rel_err"] <= tol)
    return out


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def reduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reference_arm(args, world, rank):
    """The CPU restatement on the whole workload (all host threads): one
    destripe to cglimit, its PCG iterations are the steps."""
    if rank != 0:
        return 0
    cfg, wname = config_for(args.config)
    res = run_cpu(cfg, full=not args.ref_sample)
    line = {"impl": "reference", "metric": "TOD samples/s per PCG iteration",
            "value": res["value"], "unit": "samples/s per PCG iteration", "n_gpus": args.gpus,
            "steps": res["iterations"], "warmup": 0,
            "ms_per_step": res["ms_per_iteration"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wname, "samples": cfg.ndet * cfg.nsamp, "nside": cfg.nside,
                       "sample": res["sample"],
                       "parallelism": "CPU, {} threads".format(res["cores"])},
            "time_to_cglimit_ms": res["time_to_cglimit_ms"],
            "iterations_to_cglimit": res["iterations"], "destripe_s": res["destripe_s"],
            "cpu_baseline": {"value": res["value"], "unit": res["unit"], "cores": res["cores"],
                             "kind": res["kind"], "sample": res["sample"]},
            "e2e": {"value": res["value"], "unit": res["unit"], "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "reference Fortran/MPI/FFTW build unavailable (no Fortran compiler, MPI, "
                    "FFTW or LAPACK in the image); the C++/OpenMP restatement of its "
                    "destripe path is timed instead"}
    print(json.dumps(line), flush=True)
    return 0


def run_mc(args, world, rank, local):
    """Batched Monte Carlo form (nside 512, 32 detectors x 2^22 samples, nrhs
    noise-only realisations sharing one pointing).  The headline is the
    FP32-TOD multi-right-hand-side solve (float32 realisations, float64
    pixel matrices and reductions); beside it the float64 batched solve of the
    same realisations, the error between the two, and the plain float64
    destripe_with_cache of one realisation at a time."""
    import torch
    from libmadam_b200 import libmadam_wrapper as W
    from libmadam_b200 import synthetic as syn
    cfg = syn.config4()
    if args.config == "mc-prof":  # 4 detectors x 2^20 samples: small enough for ncu captures
        cfg.ndet = 4
        cfg.nsamp_obs = 1 << 20
    cfg.seed += 1000 * rank
    R = args.nrhs
    d = syn.generate(cfg, device="cuda", with_signal=False)
    # realisations rounded to float32 once: the float64 and the float32 solves
    # see the same samples, so their difference is the form's arithmetic
    sigs = syn.noise_realisations(cfg, R + 1, device="cuda").float().double()
    torch.cuda.synchronize()
    n = cfg.ndet * cfg.nsamp
    pars = dict(d["pars"], mcmode=True)
    pix = d["pixels"].reshape(-1)
    wts = d["pixweights"].reshape(-1)
    psd = (d["periods"], d["npsd"], d["psdstarts"], d["psdfreqs"], d["psdvals"])
    W.destripe(None, pars, d["dets"], d["detweights"], d["timestamps"], pix.clone(), wts,
               sigs[R].reshape(-1).clone(), *psd)
    # one realisation at a time (the reference's way), float64
    barrier(world)
    W.destripe_with_cache(None, d["timestamps"], pix.clone(), wts, sigs[0].reshape(-1).clone(), b"")
    t1 = W.timings()
    it1 = int(W.scalars()["noiter"])
    single = n * it1 / (t1["iterate_ms"] * 1e-3)
    # all at once, float64
    W.destripe_with_cache_batch(None, d["timestamps"], pix.clone(), wts, sigs[:R])
    torch.cuda.synchronize()
    t64 = W.timings()
    its64 = W.get_result("noiter_batch")
    aa64 = W.get_result("aa_batch")
    map64 = W.get_result("map_batch")
    value64 = world * n * float(its64.sum()) / (reduce_max(t64["iterate_ms"], world) * 1e-3)
    # all at once, FP32-TOD form (the headline)
    s32 = sigs[:R].float()
    del sigs
    torch.cuda.empty_cache()
    barrier(world)
    clk = Clocks(local)
    W.destripe_with_cache_batch_fp32(None, d["timestamps"], pix.clone(), wts, s32)
    torch.cuda.synchronize()
    clocks = clk.stop()
    tb = W.timings()
    its = W.get_result("noiter_batch")
    t_it = reduce_max(tb["iterate_ms"], world)
    value = world * n * float(its.sum()) / (t_it * 1e-3)
    rel = lambda a, b: float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
    err_aa = rel(W.get_result("aa_batch"), aa64)
    m32 = W.get_result("map_batch").reshape(R, -1, 3)
    m64 = map64.reshape(R, -1, 3)
    err_map = [max(rel(m32[r][:, c], m64[r][:, c]) for r in range(R)) for c in range(3)]
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import parity
    pp = lambda a, b, f=parity.FP32_FLOOR: parity.per_pixel_error(a, b, f)[0]
    a32 = W.get_result("aa_batch").reshape(R, -1)
    a64r = aa64.reshape(R, -1)
    pp_map = [max(pp(m32[r][:, c], m64[r][:, c]) for r in range(R)) for c in range(3)]
    pp_aa = max(pp(a32[r], a64r[r]) for r in range(R))
    pp_map3 = [max(pp(m32[r][:, c], m64[r][:, c], parity.FLOOR) for r in range(R))
               for c in range(3)]
    # the same with the solve's undetermined common offset of baselines and
    # I map removed (the destriping system is singular along it)
    ppo = lambda a, b: parity.per_pixel_error_modulo_offset(a, b, parity.FP32_FLOOR)[0]
    pp_map_off = [max((ppo if c == 0 else pp)(m32[r][:, c], m64[r][:, c]) for r in range(R))
                  for c in range(3)]
    pp_aa_off = max(ppo(a32[r], a64r[r]) for r in range(R))
    n_rel = int(W.scalars()["reliable_updates"])
    line = None
    if rank == 0:
        line = {"metric": "TOD samples/s per PCG iteration (batched Monte Carlo)",
                "value": value, "unit": "samples/s per PCG iteration", "n_gpus": world,
                "steps": int(its.max()), "warmup": 0,
                "ms_per_step": t_it / max(1, int(its.max())), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "batched MC nside512 %ddet x 2^%d @100Hz, %d noise "
                                       "realisations, fknee 0.02-0.2 Hz, float32 TOD"
                                       % (cfg.ndet, cfg.nsamp_obs.bit_length() - 1, R),
                           "samples": n, "nrhs": R, "parallelism": "single GPU"},
                "clocks": clocks,
                "iterations": {"min": int(its.min()), "max": int(its.max()),
                               "single_rhs": it1},
                "batch_iterate_ms": t_it, "batch_setup_ms": tb["setup_ms"],
                "phases_ms_per_iteration": {
                    k: tb[k + "_ms"] / max(1, int(its.max()))
                    for k in ("scatter", "gather", "filter", "precond")},
                "reliable_updates_ms": tb["other_ms"],
                "batch_finalize_ms": tb["finalize_ms"],
                "fp64_batch": {"value": value64, "iterate_ms": t64["iterate_ms"],
                               "iterations_max": int(its64.max()),
                               "speedup_vs_one_at_a_time": value64 / single},
                "fp32_vs_fp64": {"map_rel_err_iqu": err_map, "baseline_rel_err": err_aa,
                                 "map_per_pixel_err_iqu": pp_map,
                                 "baseline_per_baseline_err": pp_aa,
                                 "map_per_pixel_err_iqu_modulo_offset": pp_map_off,
                                 "baseline_per_baseline_err_modulo_offset": pp_aa_off,
                                 "tolerance": 1e-4,
                                 "map_per_pixel_err_iqu_floor_1e-3": pp_map3,
                                 "samples": "the same (float32) samples in both batches",
                                 "error_definition": "max over realisations of max |fp32 - "
                                                     "fp64| / max(|fp64|, 1e-2 max|fp64|)"},
                "reliable_updates": n_rel,
                "single_rhs": {"value": single, "iterate_ms": t1["iterate_ms"],
                               "dtype": "f64"},
                "speedup_vs_one_at_a_time": value / single}
    del s32, d
    W.clear_caches()
    torch.cuda.empty_cache()
    return line


def serve_requests(n, rate, seed):
    """The serving stream's request mix: per request nside in {128, 256, 512,
    1024}, 2-32 detectors, log-uniform 2^18-2^24 samples per detector, fknee
    0.02-0.2 Hz, base_first in {0.25, 0.5, 1, 2} s, float32 TOD for half of
    them, its own seed; and Poisson arrival times at `rate` per second."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n):
        specs.append(dict(
            nside=int(rng.choice([128, 256, 512, 1024])), ndet=int(rng.integers(2, 33)),
            nsamp=int(2 ** rng.uniform(18, 24)), fknee=float(rng.uniform(0.02, 0.2)),
            base_first=float(rng.choice([0.25, 0.5, 1.0, 2.0])), f32=bool(rng.random() < 0.5),
            seed=7000 + i))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    return specs, arrivals


def run_serve(args, world, rank, local):
    """Serving stream with the request mix of the serving workload: requests
    draw nside in {128, 256, 512, 1024}, 2-32 detectors, log-uniform 2^18-2^24
    samples per detector, base_first in {0.25, 0.5, 1, 2} s and their own
    seeded scan, sky and 1/f noise (fknee 0.02-0.2 Hz), cglimit 1e-10, half of
    them float32 TOD (served in the FP32-TOD form); they arrive as a Poisson
    process at args.rate and are served by libmadam_b200.serve.

    A client thread generates the requests' inputs on the device (on its own
    stream) ahead of their arrival, with at most 45% of the free HBM
    outstanding, and a reaper frees them once the job is done, so that a
    stream of any length fits the device.  The clock starts when the client
    has filled that share (or generated every request), so a stream that fits
    it runs with no generation beside the server; a longer one has the
    client generating on the same GPU while it runs (client_generation_s
    counts that time).  Latency is measured from the scheduled arrival to
    the job's end (it includes any wait for the client) and from the
    submission; throughput is samples over the makespan."""
    import threading
    import torch
    from libmadam_b200 import synthetic as syn
    from libmadam_b200.serve import Server
    specs, arrivals = serve_requests(args.requests, args.rate, 5005 + rank)
    free, _ = torch.cuda.mem_get_info()
    gen_cap = 0.45 * free
    cond = threading.Condition()
    ready = [None] * len(specs)
    state = dict(outstanding=0.0, gen_s=0.0, err=None, primed=False, gen_run_s=0.0,
                 pregenerated=0)

    def in_bytes(sp):
        return sp["ndet"] * sp["nsamp"] * (4 + 12 + (4 if sp["f32"] else 8)) + 8 * sp["nsamp"]

    def client():
        try:
            torch.cuda.set_device(local)
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):
                for i, sp in enumerate(specs):
                    b = in_bytes(sp)
                    with cond:
                        if state["outstanding"] > 0 and state["outstanding"] + b > gen_cap:
                            state["primed"] = True
                            cond.notify_all()
                        cond.wait_for(lambda: state["outstanding"] == 0
                                      or state["outstanding"] + b <= gen_cap)
                        state["outstanding"] += b
                    tg = time.perf_counter()
                    cfg = syn.ScanConfig(nside=sp["nside"], nside_submap=16, ndet=sp["ndet"],
                                         nobs=1, nsamp_obs=sp["nsamp"], fsample=100.0,
                                         fknee=sp["fknee"], alpha=-1.0,
                                         base_first=sp["base_first"], seed=sp["seed"],
                                         extra_pars=dict(cglimit=1e-10))
                    d = syn.generate(cfg, device="cuda")
                    d.pop("sky")
                    d["pixels"] = d["pixels"].reshape(-1)
                    d["pixweights"] = d["pixweights"].reshape(-1)
                    d["signal"] = d["signal"].reshape(-1)
                    if sp["f32"]:
                        d["signal"] = d["signal"].float()
                    st.synchronize()
                    with cond:
                        state["gen_s"] += time.perf_counter() - tg
                        if state["primed"]:
                            state["gen_run_s"] += time.perf_counter() - tg
                        else:
                            state["pregenerated"] += 1
                        ready[i] = (d, b)
                        cond.notify_all()
            with cond:
                state["primed"] = True
                cond.notify_all()
        except Exception as e:  # reported by the submitting loop
            with cond:
                state["err"] = e
                state["primed"] = True
                cond.notify_all()

    tickets = [None] * len(specs)
    t_sub = np.zeros(len(specs))
    done = np.zeros(len(specs), dtype=bool)
    infos = [None] * len(specs)
    failures = []

    def reaper():
        left = set()
        nsub = 0
        while not done.all():
            with cond:
                while nsub < len(specs) and tickets[nsub] is not None:
                    left.add(nsub)
                    nsub += 1
            fin = []
            for i in left:
                try:
                    if srv.wait(tickets[i], 0.0) == 2:
                        fin.append(i)
                except RuntimeError as e:  # a failed job
                    failures.append(str(e))
                    fin.append(i)
            for i in fin:
                try:
                    infos[i] = srv.info(tickets[i])
                except RuntimeError:
                    infos[i] = None
                srv.release(tickets[i])
                left.discard(i)
                with cond:
                    state["outstanding"] -= ready[i][1]
                    ready[i] = None
                    tickets[i] = 0
                    done[i] = True
                    cond.notify_all()
            if fin and int(done.sum()) % 8 < len(fin):
                # the client's freed inputs go back to the device (torch keeps
                # them cached otherwise, out of the server's reach)
                torch.cuda.empty_cache()
            if not fin:
                time.sleep(0.001)

    th_c = threading.Thread(target=client, daemon=True)
    th_c.start()
    with cond:
        cond.wait_for(lambda: state["primed"])
        if state["err"] is not None:
            raise state["err"]
    srv = Server(workers=args.workers, mem_fraction=0.8)
    clk = Clocks(local)
    t0 = time.perf_counter()
    th_r = threading.Thread(target=reaper, daemon=True)
    th_r.start()
    for i, ta in enumerate(arrivals):
        dt = ta - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        with cond:
            cond.wait_for(lambda: ready[i] is not None or state["err"] is not None)
            if state["err"] is not None:
                raise state["err"]
            d = ready[i][0]
        t_sub[i] = time.perf_counter() - t0
        tk = srv.submit(d["pars"], d["dets"], d["detweights"], d["timestamps"], d["pixels"],
                        d["pixweights"], d["signal"], d["periods"], d["npsd"], d["psdstarts"],
                        d["psdfreqs"], d["psdvals"])
        with cond:
            tickets[i] = tk
    th_r.join()
    clocks = clk.stop()
    stats = srv.stats()
    srv.close()
    if failures:
        raise RuntimeError("%d serving jobs failed, the first: %s" % (len(failures), failures[0]))
    lat_sub = np.array([inf["t_end"] - inf["t_submit"] for inf in infos])
    lat = lat_sub + (t_sub - arrivals)
    makespan = max(inf["t_end"] for inf in infos) - min(inf["t_submit"] for inf in infos)
    samples = np.array([inf["samples"] for inf in infos])
    iters = np.array([inf["iterations"] for inf in infos])
    line = {"metric": "serving latency p50 / p99 and TOD samples/s",
            "value": float(np.percentile(lat, 50) * 1e3), "unit": "ms (p50 latency)",
            "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "p50_ms_from_submit": float(np.percentile(lat_sub, 50) * 1e3),
            "p99_ms_from_submit": float(np.percentile(lat_sub, 99) * 1e3),
            "n_gpus": 1, "higher_is_better": False, "vs_baseline": None,
            "dtype": "f64 and f32 (mixed TOD)", "data": "synthetic",
            "config": {"workload": "serving stream: %d requests, Poisson %.1f req/s, nside "
                                   "128-1024, 2-32 detectors, 2^18-2^24 samples per detector, "
                                   "base_first 0.25-2 s, cglimit 1e-10, half the requests "
                                   "float32 TOD" % (args.requests, args.rate),
                       "float32_requests": int(sum(sp["f32"] for sp in specs)),
                       "workers": args.workers},
            "clocks": clocks,
            "makespan_s": makespan,
            "arrival_span_s": float(arrivals[-1]),
            "requests_generated_before_the_clock": state["pregenerated"],
            "client_generation_s_while_serving": state["gen_run_s"],
            "samples_per_s": float(samples.sum() / makespan),
            "samples_per_s_per_pcg_iteration": float((samples * iters).sum() / makespan),
            "mean_iterations": float(iters.mean()),
            "total_samples": float(samples.sum()),
            "job_phase_seconds_summed": {
                k: float(sum(inf[k + "_ms"] for inf in infos) / 1e3)
                for k in ("setup", "iterate", "finalize")},
            "queue_seconds_summed": float(sum(inf["t_start"] - inf["t_submit"] for inf in infos)),
            "pcg_rounds": stats["rounds"], "pcg_job_rounds": stats["job_rounds"],
            "most_jobs_in_one_round": stats["max_jobs"],
            "mean_jobs_per_round": stats["job_rounds"] / max(1, stats["rounds"])}
    return line if rank == 0 else None


def extra_serve(args, world, rank, local):
    """The serving stream for the headline line's "serving" key."""
    r = run_serve(args, world, rank, local)
    if r is None:
        return None
    out = {k: v for k, v in r.items() if k not in ("n_gpus", "higher_is_better", "vs_baseline",
                                                   "data", "config")}
    out["workload"] = r["config"]["workload"]
    out["float32_requests"] = r["config"]["float32_requests"]
    out["workers"] = r["config"]["workers"]
    return out


def run_destripe(args, world, rank, local, config, with_e2e=True, with_cpu=True):
    """One destripe() workload: the full solve with inputs resident in HBM
    (time to cglimit), the timed PCG iterations (the step), optionally the
    end-to-end calls from pinned host buffers and the CPU leg, and the
    roofline.  Returns rank 0's JSON line (None on other ranks)."""
    import torch
    from libmadam_b200 import libmadam_wrapper as W
    from libmadam_b200 import synthetic as syn
    cfg, wname = config_for(config)
    cfg.seed += 1000 * rank
    t0 = time.time()
    d = syn.generate(cfg, device="cuda")
    torch.cuda.synchronize()
    t_gen = time.time() - t0
    n = cfg.ndet * cfg.nsamp
    fp32 = config in ("3", "mid3")
    destripe = W.destripe_fp32 if fp32 else W.destripe
    pix = d["pixels"].reshape(-1)
    wts = d["pixweights"].reshape(-1)
    sig = d["signal"].reshape(-1)
    if fp32:
        sig64 = sig
        sig = sig.float()
        d["signal"] = d["signal"].float()
    common = (d["pars"], d["dets"], d["detweights"])
    psd = (d["periods"], d["npsd"], d["psdstarts"], d["psdfreqs"], d["psdvals"])

    # full solve with inputs resident in HBM: time to cglimit
    comm = None
    if args.sharded and world > 1:
        from libmadam_b200.comm import NcclComm
        comm = NcclComm()
    destripe(comm, *common, d["timestamps"], pix, wts, sig, *psd)
    tim = W.timings()
    sca = W.scalars()
    marks = W.setup_marks()
    noiter = int(sca["noiter"])
    if fp32:
        map32, aa32 = W.get_result("map"), W.get_result("aa")

    # timed PCG iterations (the step)
    barrier(world)
    torch.cuda.synchronize()
    clk = Clocks(local)
    l0 = W.kernel_launches()
    b = W.bench_iterations(args.warmup, args.steps)
    launches = W.kernel_launches() - l0
    torch.cuda.synchronize()
    barrier(world)
    clocks = clk.stop()
    ms_iter = reduce_max(b["ms_per_iter"], world)
    value = world * n / (ms_iter * 1e-3)

    # end to end through the C-ABI with pinned host buffers
    e2e = None
    if with_e2e:
        h = {k: d[k].cpu().pin_memory() for k in ("timestamps", "pixels", "pixweights", "signal")}
        hn = {k: v.numpy().reshape(-1) for k, v in h.items()}
        # one untimed call from host buffers (the library's memory pool grows
        # to the host path's buffers), then E2E_STEPS timed calls; each call
        # copies its inputs from pinned host memory and reads the map back
        calls = []
        for rep in range(1 + E2E_STEPS):
            barrier(world)
            t1 = time.perf_counter()
            destripe(comm, *common, hn["timestamps"], hn["pixels"], hn["pixweights"],
                     hn["signal"], *psd)
            m = W.get_result("map")
            t_call = reduce_max(time.perf_counter() - t1, world)
            if rep > 0:
                calls.append(t_call)
        t_e2e = sum(calls) / len(calls)
        it_e2e = int(W.scalars()["noiter"])
        te = W.timings()
        h2d = sum(v.numel() * v.element_size() for v in h.values())
        e2e = {"value": world * n * it_e2e / t_e2e, "unit": "samples/s per PCG iteration",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(m.nbytes),
               "seconds": t_e2e, "seconds_per_call": calls, "warmup_calls": 1,
               "iterations": it_e2e,
               "library_ms": {k: te[k] for k in ("setup_ms", "iterate_ms", "finalize_ms",
                                                  "total_ms")},
               "setup_marks_ms": W.setup_marks()}
        del h, hn

    # the precision form against a float64-TOD solve of the same samples
    fp64_cmp = None
    if fp32:
        # the float64 destripe() of the same samples (the float32 signal
        # widened: the form's arithmetic error) and of the float64 signal the
        # float32 one was rounded from (adds the input's rounding)
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import parity
        sca32 = sca
        del d["signal"], sig
        sig_same = sig64.float().double()
        torch.cuda.empty_cache()
        W.destripe(comm, *common, d["timestamps"], pix, wts, sig_same, *psd)
        ms = W.get_result("map").reshape(-1, 3)
        a_same = W.get_result("aa")
        it64 = int(W.scalars()["noiter"])
        t64 = W.timings()["iterate_ms"]
        b64 = W.bench_iterations(args.warmup, args.steps)
        del sig_same
        torch.cuda.empty_cache()
        W.destripe(comm, *common, d["timestamps"], pix, wts, sig64, *psd)
        m64 = W.get_result("map").reshape(-1, 3)
        a64 = W.get_result("aa")
        m32 = map32.reshape(-1, 3)
        rel = lambda a, b: float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
        pp = lambda a, b, f=parity.FP32_FLOOR: parity.per_pixel_error(a, b, f)[0]
        fp64_cmp = {"same_samples": {
                        "map_per_pixel_err_iqu": [pp(m32[:, c], ms[:, c]) for c in range(3)],
                        "baseline_per_baseline_err": pp(aa32, a_same),
                        "tolerance": 1e-4,
                        "map_per_pixel_err_iqu_floor_1e-3": [pp(m32[:, c], ms[:, c], parity.FLOOR)
                                                             for c in range(3)],
                        "error_definition": "max |fp32 - fp64| / max(|fp64|, 1e-2 max|fp64|)"},
                    "float64_signal": {
                        "map_rel_err_iqu": [rel(m32[:, c], m64[:, c]) for c in range(3)],
                        "baseline_rel_err": rel(aa32, a64),
                        "error_definition": "max |fp32 - fp64| / max|fp64| (includes the "
                                            "float32 rounding of the input)"},
                    "fp64_ms_per_iteration": b64["ms_per_iter"],
                    "fp64_iterations_to_cglimit": it64, "fp64_time_to_cglimit_ms": t64,
                    "speedup_per_iteration": b64["ms_per_iter"] / b["ms_per_iter"],
                    "reliable_updates": sca32["reliable_updates"],
                    "pointing_pairs": sca32["pairs"],
                    "samples_per_pair": n / max(1.0, sca32["pairs"])}
        sca = sca32
        del sig64

    # roofline of the dominant kernel (algorithmic bytes per launch / duration)
    hbm, peak_kind = peaks()
    nb = cfg.ndet * int(sca["noba_short"])
    npix_hit = int(sca["nloc"])
    phases = {"scatter": b["scatter_ms"], "gather": b["gather_ms"], "filter": b["filter_ms"],
              "precond": b["precond_ms"]}
    # pointing entries streamed per iteration: samples, or pairs in the FP32 form
    nent = int(sca["pairs"]) if fp32 and sca["pairs"] > 0 else n
    algo = {"scatter": 16.0 * nent + 8.0 * nent / max(1, cfg.base_first * cfg.fsample),
            "gather": 16.0 * nent + 5 * 8.0 * nb + (16.0 if fp32 else 32.0) * npix_hit,
            "filter": None, "precond": None}
    dom = max(("scatter", "gather"), key=lambda k: phases[k])
    achieved = algo[dom] / (phases[dom] * 1e-3) / 1e9
    kname = {"scatter": "k_scatter_chunks",
             "gather": "k_gather_pairs" if nent != n else "k_gather_chunks"}[dom]
    traffic = profiled_traffic(kname, nent)
    try:
        w_p = float(np.mean(W.get_result("band_widths")))
    except Exception:
        w_p = 0.0
    b_iter = 32.0 * nent + 8.0 * (16 + w_p) * nb + (4 * 3 * 8 + 48) * npix_hit
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": hbm,
                "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                "algorithmic_bytes": algo[dom], "traffic": traffic,
                "iteration": {"algorithmic_bytes": b_iter,
                              "achieved_gbs": b_iter / (ms_iter * 1e-3) / 1e9,
                              "frac": b_iter / (ms_iter * 1e-3) / 1e9 / hbm}}

    cpu = None
    par = None
    if rank == 0 and world == 1 and with_cpu:
        try:
            cpu = run_cpu(cfg, parity_fp32=fp32)
            par = cpu.get("parity")
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as e:  # the CPU leg never blocks the GPU line
            cpu = {"value": None, "unit": "samples/s per PCG iteration", "cores": None,
                   "kind": "port", "sample": "failed: {}".format(e)}

    line = None
    if rank == 0:
        line = {
            "metric": "TOD samples/s per PCG iteration", "value": value,
            "unit": "samples/s per PCG iteration", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_iter, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if fp32 else "f64",
            "data": "synthetic",
            "config": {"workload": wname, "samples": n, "baselines": nb,
                       "hit_pixels": npix_hit, "nside": cfg.nside,
                       "l2": "inputs larger than L2 (pointing {:.1f} GB)".format(16e-9 * n),
                       "parallelism": ("sharded by detector over NCCL" if comm is not None
                                       else "replicas" if world > 1 else "single GPU")},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "e2e": e2e,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "parity": par,
            "time_to_cglimit_ms": tim["iterate_ms"], "iterations_to_cglimit": noiter,
            "destripe_device_ms": tim["total_ms"], "setup_ms": tim["setup_ms"],
            "phases_ms_per_iteration": phases, "generate_s": t_gen,
            "setup_marks_ms": marks,
            "band": {k: sca[k] for k in ("band_rows", "band_transfers", "band_chunks", "nseg", "band_guard")},
        }
        if fp32:
            line["precision"] = ("float32 TOD, pointing pairs and map copy in the projections; "
                                 "float64 pixel matrices, baselines and reductions")
            line["fp64_comparison"] = fp64_cmp
    if comm is not None:
        comm.free()
    d = pix = wts = sig = None
    W.clear_caches()
    torch.cuda.empty_cache()
    return line


def extra_precision(args, world, rank, local):
    """The precision form on its workload (nside 1024, 64 detectors x 2^24
    samples, float32 TOD through destripe_fp32) and the float64 destripe()
    of the same samples, for the line's "precision_form" key."""
    r = run_destripe(args, world, rank, local, "3", with_e2e=False, with_cpu=False)
    if r is None:
        return None
    cmp = r["fp64_comparison"]
    return {"workload": r["config"]["workload"], "value": r["value"], "unit": r["unit"],
            "ms_per_step": r["ms_per_step"], "clocks": r["clocks"], "dtype": r["dtype"],
            "iterations_to_cglimit": r["iterations_to_cglimit"],
            "time_to_cglimit_ms": r["time_to_cglimit_ms"],
            "phases_ms_per_iteration": r["phases_ms_per_iteration"],
            "roofline": r["roofline"],
            "fp64_destripe_ms_per_iteration": cmp["fp64_ms_per_iteration"],
            "fp64_destripe_time_to_cglimit_ms": cmp["fp64_time_to_cglimit_ms"],
            "fp64_destripe_iterations": cmp["fp64_iterations_to_cglimit"],
            "speedup_vs_fp64_destripe_per_iteration": cmp["speedup_per_iteration"],
            "speedup_vs_fp64_destripe_to_cglimit": cmp["fp64_time_to_cglimit_ms"]
            / r["time_to_cglimit_ms"],
            "error_vs_fp64_same_samples": cmp["same_samples"],
            "error_vs_fp64_float64_signal": cmp["float64_signal"],
            "reliable_updates": cmp["reliable_updates"],
            "pointing_pairs": cmp["pointing_pairs"], "samples_per_pair": cmp["samples_per_pair"],
            "target_3x": "not met by this form alone (see batched_mc)"
            if cmp["speedup_per_iteration"] < 3 else "met"}


def extra_mc(args, world, rank, local):
    """The batched Monte Carlo form (nside 512, 32 detectors x 2^22 samples,
    64 noise realisations as one float32-TOD multi-right-hand-side PCG) for
    the line's "batched_mc" key."""
    r = run_mc(args, world, rank, local)
    if r is None:
        return None
    keep = ("metric", "value", "unit", "ms_per_step", "clocks", "dtype", "iterations",
            "batch_iterate_ms", "batch_setup_ms", "phases_ms_per_iteration",
            "reliable_updates_ms", "fp64_batch", "fp32_vs_fp64",
            "reliable_updates", "single_rhs",
            "speedup_vs_one_at_a_time")
    out = {k: r[k] for k in keep}
    out["workload"] = r["config"]["workload"]
    out["target_3x"] = ("met: {:.2f}x the float64 destripe_with_cache one realisation at a "
                        "time".format(r["speedup_vs_one_at_a_time"])
                        if r["speedup_vs_one_at_a_time"] >= 3 else
                        "not met: {:.2f}x".format(r["speedup_vs_one_at_a_time"]))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="2", choices=["2", "1", "3", "prof", "mid", "mid3", "small",
                                                   "mc", "mc-prof", "serve"])
    ap.add_argument("--requests", type=int, default=200,
                    help="serving: requests in the stream (the serving workload names 2000; "
                         "the headline line runs this many)")
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--workers", type=int, default=6)
    ap.add_argument("--nrhs", type=int, default=64)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--only", action="store_true",
                    help="config 2: the headline workload alone, without the precision-form "
                         "and batched Monte Carlo keys")
    ap.add_argument("--ref-sample", action="store_true",
                    help="--impl reference: time the bounded sample instead of the whole "
                         "workload")
    ap.add_argument("--sharded", action="store_true",
                    help="N > 1: one sharded solve over NCCL (each rank its own detectors) "
                         "instead of N independent replicas")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        rc = reference_arm(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return rc

    import torch
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    if args.config in ("mc", "mc-prof"):
        line = run_mc(args, world, rank, local)
    elif args.config == "serve":
        line = run_serve(args, world, rank, local)
    else:
        line = run_destripe(args, world, rank, local, args.config,
                            with_e2e=not args.no_e2e, with_cpu=not args.no_cpu)
        if args.config == "2" and world == 1 and not args.only:
            # the headline line carries the precision form (float32 TOD at
            # nside 1024), the batched Monte Carlo form (64 realisations) and
            # the serving stream, each measured in the same run with its own
            # clocks record; a form that fails is reported in its key and
            # does not take the headline line with it
            for key, fn in (("precision_form", extra_precision), ("batched_mc", extra_mc),
                            ("serving", extra_serve)):
                try:
                    line[key] = fn(args, world, rank, local)
                except Exception as e:  # noqa: BLE001
                    line[key] = {"error": "{}: {}".format(type(e).__name__, e)}
                    torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
