"""Benchmark: Landau gauge fixing of 32^3x64 SU(3) configurations to
theta < 1e-14 (Fourier-accelerated CG), in gauge-fixed configurations per
hour.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--precision mixed|fp64] [--dims 32,32,32,64]

A step is four complete gauge fixes (GLU's FACG to theta < 1e-14).
`value` is measured with the links resident in HBM (the device entry point
gfix_landau_device); `e2e` is the same fixes through the host entry point
gfix_landau from pinned host memory, host->device and device->host copies
inside the timed region.  Both run the mixed FP32->FP64 path by default and
report the plain FP64 path beside it.

Input: beta 6.0 heatbath configurations generated on the GPU before any
timed region (glu_b200.workload.heatbath_config: GLU's heatbath algorithm,
1000 iterations of one heatbath and four over-relaxation sweeps from the unit
start).  A step fixes four of them (seeds 2..5): on thermalised fields the
iteration count of a fix varies twofold between configurations, so the
throughput is that of a set.  At N > 1 every rank fixes the same set on its
own GPU (the same work per GPU): weak scaling, no collective on the data
path.

The reference arm (--impl reference) times GLU itself, compiled from its
sources (oracle/_ref), on the host cores: a bounded sample of FACG
iterations (on the host-built tiled stand-in: the cost of an iteration does
not depend on the configuration), scaled by the iteration counts of GLU's
full fixes of the four configurations (profiles/reference_full_fix.json).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

def metric_name(dims) -> str:
    return "gauge-fixed configs/hour (%dx%dx%dx%d Landau FACG, theta<1e-14)" % tuple(dims)
UNIT = "configs/hour"
ACC = 1e-14
ALPHA = 0.08
MAX_ITERS = 20000
# gauge invariance: the average plaquette of a fixed configuration equals
# the input's to this absolute tolerance
PLAQ_TOL = 1e-13
# the B200's nominal HBM3e bandwidth (GB/s), reported beside the fraction of
# the measured copy peak
HBM_NOMINAL_GBS = 8000.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64", "polish"],
                    help="mixed (default) or fp64; polish only with --profile-only: "
                         "the kernels of a mixed solve's FP64-link phase")
    ap.add_argument("--workload", default="landau",
                    choices=["landau", "coulomb", "ensemble", "gluonprop", "heatbath"],
                    help="landau: 32^3x64 Landau FACG (the headline); coulomb: "
                         "64^3x128 Coulomb FACG, all slices batched; ensemble: "
                         "48 x 16^3x32 + 16 x 24^3x48 Landau FASD in one batch; "
                         "gluonprop: 32^3x64 momentum-space gluon propagators "
                         "(GLU's cuts_struct, GLUON_PROPS); heatbath: 32^3x64 "
                         "heatbath + over-relaxation updates at beta 6.0")
    ap.add_argument("--dims", default=None,
                    help="lattice extents; default 32,32,32,64 (landau) or "
                         "64,64,64,128 (coulomb)")
    ap.add_argument("--beta", type=float, default=6.0,
                    help="landau: coupling of the generated heatbath inputs")
    ap.add_argument("--configs", type=int, default=4,
                    help="landau: configurations fixed per step")
    ap.add_argument("--profile-iters", type=int, default=20)
    ap.add_argument("--cpu-sample-s", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="coulomb: one configuration's time slices split over "
                         "the ranks (strong scaling; ring exchange of the "
                         "boundary gauge field) instead of one per rank")
    ap.add_argument("--profile-only", action="store_true",
                    help="only the per-kernel event timing of --profile-iters "
                         "CG iterations (a short, bounded launch list for ncu)")
    args = ap.parse_args()
    if args.precision == "polish" and not args.profile_only:
        ap.error("--precision polish profiles kernels: it needs --profile-only")
    return args


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows: list[list[str]] = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", "-i", str(self.index),
                     f"--query-gpu={self.Q}", "--format=csv,noheader,nounits"],
                    capture_output=True, text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=6)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[4:8])
                          if v.strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# the input of the Landau workload: beta 6.0 heatbath configurations, 1000
# iterations of one heatbath and four over-relaxation sweeps from the unit
# start, generated on the GPU before any timed region.  One step fixes
# E_CONFIGS of them (seeds 2 .. 1 + E_CONFIGS): the iteration count of a
# fix on a thermalised configuration varies twofold between configurations
# (and between summation orders), so throughput is measured over a set,
# the same set on every rank.
H_INPUT = dict(beta=6.0, iterations=1000, n_or=4)
INPUT_NAME = "heatbath beta 6.0, 1000 x (HB + 4 OR), unit start, seed %d"
E_CONFIGS = 4


def set_input(beta: float, configs: int):
    """--beta / --configs of the Landau workload (defaults 6.0, 4)"""
    global INPUT_NAME, E_CONFIGS
    H_INPUT["beta"] = beta
    INPUT_NAME = "heatbath beta %g, 1000 x (HB + 4 OR), unit start, seed %%d" % beta
    if beta == 6.0:
        INPUT_NAME = "heatbath beta 6.0, 1000 x (HB + 4 OR), unit start, seed %d"
    E_CONFIGS = max(1, int(configs))


def seeds(rank):
    """every rank fixes the same configurations: with iteration counts that
    vary twofold between configurations, distinct sets per rank would make
    the slowest rank's set, not the hardware, set a weak-scaling step"""
    return [2 + i for i in range(E_CONFIGS)]


def workload(dims, rank, i=0):
    from glu_b200.workload import heatbath_config
    return heatbath_config(dims, seed=seeds(rank)[i], **H_INPUT)


def _params(prec: str, cap: int = 0):
    from glu_b200._lib import GfixParams
    p = GfixParams()
    p.gf_alpha = ALPHA
    p.accuracy = ACC
    p.max_iters = MAX_ITERS
    p.algo = 0
    p.sd_fixed_step = 0
    p.precision = 1 if prec == "mixed" else 0
    p.switch_theta = 1e-9
    p.traj_cap = 0
    return p


def peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback 6.65 TB/s"


KERNELS = ["k_deriv", "k_fft_xy_fwd", "k_fft_zt", "k_fft_xy_bwd_pr",
           "k_dir_probe", "k_update", "k_scalar"]


def traffic_from_profiles(name: str, prec: str, dims):
    """dram read+write bytes per launch from the committed ncu summary"""
    f = ROOT / "profiles" / "ncu_traffic.json"
    if not f.exists():
        return None
    d = json.loads(f.read_text())
    e = d.get(f"{name}:{prec}")
    if not e:
        return None
    scale = np.prod(dims) / float(np.prod(e["dims"]))
    return float(e["dram_bytes_per_launch"]) * scale


def gpu_arm(args, dims, rank, world, local):
    import ctypes as C
    import torch
    torch.cuda.set_device(local)
    from glu_b200 import _lib
    from glu_b200._lib import GfixResult, check
    lib = _lib.load()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    Us = [workload(dims, rank, i) for i in range(E_CONFIGS)]
    U = Us[0]
    hosts = [torch.from_numpy(u.view(np.float64).reshape(-1)).pin_memory() for u in Us]
    hworks = [torch.empty_like(h).pin_memory() for h in hosts]
    dpristine = [h.to("cuda") for h in hosts]
    dwork = torch.empty_like(dpristine[0])
    cd = (C.c_size_t * 4)(*dims)
    V = int(np.prod(dims))

    def dev_fix(prec, i):
        # the copy of the pristine input is device work inside the step; the
        # library runs on its own stream, so the copy must be complete
        dwork.copy_(dpristine[i])
        torch.cuda.synchronize()
        r = GfixResult()
        p = _params(prec)
        check(lib.gfix_landau_device(dwork.data_ptr(), cd, C.byref(p), C.byref(r)))
        return r

    def host_fix_all(prec):
        # the step's configurations through one gfix_landau_sequence call:
        # host links in, fixed links back, each configuration's copies
        # overlapping its neighbours' solves
        rs = (GfixResult * E_CONFIGS)()
        p = _params(prec)
        ptrs = (C.c_void_p * E_CONFIGS)(*[h.data_ptr() for h in hworks])
        check(lib.gfix_landau_sequence(ptrs, E_CONFIGS, cd, C.byref(p), rs))
        return rs

    def plaquette(ptr, reunit=False):
        if reunit:
            check(lib.gfix_reunit(ptr, cd))
        o = np.zeros(3)
        check(lib.gfix_observables(ptr, cd, o.ctypes.data_as(C.POINTER(C.c_double))))
        return float(o[2])

    # every fixed configuration must stay on its input's gauge orbit: the
    # average plaquette of the last step's fixed links (host side, after
    # the timed region), reunitarised as GLU's Landau driver does before it
    # reports (output_fixing_info: over a long fix the links drift off
    # SU(3) through GLU's update, which rebuilds one column from the other
    # two), against the input's
    plaq_in = [plaquette(h.data_ptr()) for h in hosts]

    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    out = {}
    with Clocks(local) as clk:
        for prec in ([args.precision, "fp64"] if args.precision == "mixed"
                     else ["fp64"]):
            for _ in range(args.warmup):
                for i in range(E_CONFIGS):
                    dev_fix(prec, i)
            # resident inputs: K steps (each E_CONFIGS fixes) bracketed by
            # barrier + sync
            launches0 = lib.gfix_kernel_launches()
            barrier()
            a, b = ev(), ev()
            a.record()
            per = []
            for _ in range(args.steps):
                per = []
                for i in range(E_CONFIGS):
                    r = dev_fix(prec, i)
                    per.append((int(r.iters), int(r.iters_fp32), float(r.theta)))
            b.record()
            barrier()
            launches = lib.gfix_kernel_launches() - launches0
            ms = max_over_ranks(a.elapsed_time(b))
            # end to end: pinned host buffers, every step's H2D + D2H of its
            # configurations inside the timed call
            e_ms = 0.0
            drift = 0.0
            for k in range(args.steps):
                for i in range(E_CONFIGS):
                    hworks[i].copy_(hosts[i])
                barrier()
                a2, b2 = ev(), ev()
                a2.record()
                rs = host_fix_all(prec)
                b2.record()
                torch.cuda.synchronize()
                e_ms += a2.elapsed_time(b2)
                if [int(r.iters) for r in rs] != [x[0] for x in per]:
                    raise RuntimeError(f"{prec}: the end-to-end fixes took other iteration "
                                       f"counts than the device-resident ones")
                if k == args.steps - 1:
                    for i in range(E_CONFIGS):
                        drift = max(drift, abs(plaquette(hworks[i].data_ptr(), True)
                                               - plaq_in[i]))
            e_ms = max_over_ranks(e_ms)
            if not drift < PLAQ_TOL:
                raise RuntimeError(f"{prec}: a fixed configuration left its gauge orbit "
                                   f"(plaquette changed by {drift:.3e})")
            out[prec] = dict(ms=ms, e2e_ms=e_ms, per=per, launches=launches,
                             plaq_drift=drift)
    clocks = clk.summary()
    res = dict(out=out, clocks=clocks, V=V)
    # per-kernel device times for the roofline (events on the launch stream)
    # fp64: the FP64 solve; fp32 and polish: the two phases of a mixed one
    # (FP32 throughout; FP64 links with FP32 fields)
    prof = {}
    for tag, code in (("fp64", 0), ("fp32", 1), ("polish", 2)):
        ms = np.zeros(7)
        by = np.zeros(7)
        p = _params("fp64")
        p.precision = code
        check(lib.gfix_profile_landau(
            dpristine[0].data_ptr(), cd, C.byref(p), args.profile_iters,
            ms.ctypes.data_as(C.POINTER(C.c_double)),
            by.ctypes.data_as(C.POINTER(C.c_double))))
        prof[tag] = (ms, by)
    res["prof"] = prof
    if dist is not None:
        dist.destroy_process_group()
    return res, U


def reference_iters(dims):
    """Iteration counts of the reference's own full fixes of the step's
    configurations (rank 0 seeds), from the committed measurements; None if
    any is missing."""
    f = ROOT / "profiles" / "reference_full_fix.json"
    if not f.exists():
        return None
    rec = {e.get("input"): int(e["iters"]) for e in json.loads(f.read_text())
           if tuple(e["dims"]) == tuple(dims)}
    its = [rec.get(INPUT_NAME % sd) for sd in seeds(0)]
    return None if any(i is None for i in its) else its


def cpu_sample(U, dims, sample_s: float, nthreads: int, algo: str = "FACG"):
    """Seconds per FACG (FASD) iteration of the reference (oracle/_ref) with
    nthreads OpenMP threads, from two runs of k1 < k2 iterations (acc 1e-30:
    exactly k iterations, no continuation), and the fixed cost of a call."""
    from oracle.oracle import REF_SO, Oracle, Reference
    if REF_SO.exists():
        R = Reference()
        R.setup(dims, nthreads, ALPHA)
        kind = "reference"

        def run(k):
            R.put_links(U)
            R.lib.ref_reset_fft_seconds()
            t = time.perf_counter()
            R.landau_fa(1e-30, k, algo)
            return time.perf_counter() - t, R.fft_seconds()
    else:  # the oracle port, single threaded
        O = Oracle()
        kind, nthreads = "port", 1

        def run(k):
            t = time.perf_counter()
            O.landau(U, dims, ALPHA, 1e-30, k, algo)
            return time.perf_counter() - t, 0.0
    t1, f1 = run(1)
    k2 = max(2, int(sample_s / max(t1, 1e-3)))
    t2, f2 = run(k2)
    s_iter = (t2 - t1) / (k2 - 1)
    fixed = max(t1 - s_iter, 0.0)
    return dict(kind=kind, cores=nthreads, s_iter=s_iter, fixed_s=fixed,
                fft_thread_s_iter=(f2 - f1) / (k2 - 1), sample_iters=k2,
                sample_s=t1 + t2)


def physical_cores() -> int | None:
    """Physical cores of this host (distinct core, socket pairs of lscpu),
    or None when lscpu is unavailable."""
    try:
        out = subprocess.run(["lscpu", "-p=CORE,SOCKET"], capture_output=True,
                             text=True, timeout=10).stdout
        pairs = {ln.strip() for ln in out.splitlines() if ln and not ln.startswith("#")}
        return len(pairs) or None
    except Exception:
        return None


def recorded_seconds(dims):
    """Wall seconds of the reference's own full fixes of the step's
    configurations (profiles/reference_full_fix.json), or None."""
    f = ROOT / "profiles" / "reference_full_fix.json"
    if not f.exists():
        return None
    rec = {e.get("input"): e for e in json.loads(f.read_text())
           if tuple(e["dims"]) == tuple(dims) and "seconds" in e}
    es = [rec.get(INPUT_NAME % sd) for sd in seeds(0)]
    if any(e is None for e in es):
        return None
    return sum(float(e["seconds"]) for e in es), int(es[0].get("threads", 0))


def reference_model(s, n_ref, dims):
    """The reference's time for one step (the step's full fixes) from a
    sample `s` of cpu_sample: fixed cost per call + seconds per iteration x
    the full fixes' iteration counts.  Beside it the same with the FFT phase
    taken out: the reference's Fourier acceleration runs its four fields'
    transforms one per thread (an omp for over the fields), so the phase
    lasts the FFT stand-in's thread-seconds / min(4, threads) of wall time
    per iteration.  And the recorded wall time of the reference's own full
    fixes, when present, with the model's deviation from it."""
    t_set = E_CONFIGS * s["fixed_s"] + s["s_iter"] * sum(n_ref)
    fft_wall = s["fft_thread_s_iter"] / max(1, min(4, s["cores"]))
    t_nofft = E_CONFIGS * s["fixed_s"] + max(s["s_iter"] - fft_wall, 0.0) * sum(n_ref)
    out = {"value": E_CONFIGS * 3600.0 / t_set, "t_set": t_set,
           "value_excluding_fft": E_CONFIGS * 3600.0 / t_nofft,
           "fft_wall_s_per_iteration": fft_wall,
           "s_per_iteration_excluding_fft": max(s["s_iter"] - fft_wall, 0.0),
           "threads": s["cores"], "physical_cores": physical_cores()}
    rec = recorded_seconds(dims)
    if rec is not None:
        out["recorded_full_fix_seconds"] = rec[0]
        out["recorded_threads"] = rec[1]
        out["model_deviation"] = t_set / rec[0] - 1.0
    return out


def emit(d):
    print(json.dumps(d), flush=True)


def reference_arm(args, dims, rank, world):
    if rank != 0:
        return
    # GLU's per-iteration cost does not depend on the configuration: it is
    # sampled on the tiled stand-in (built on the host, so this arm loads
    # nothing of ours), the iteration counts are those of GLU's own full
    # fixes of the heatbath configurations
    from glu_b200.workload import tiled_config
    U = tiled_config(dims, seed=2)
    n_ref = reference_iters(dims)
    cores = os.cpu_count() or 1
    for _ in range(max(args.warmup, 0) and 1):
        cpu_sample(U, dims, min(args.cpu_sample_s, 5.0), cores)
    samples = [cpu_sample(U, dims, args.cpu_sample_s, cores)
               for _ in range(max(args.steps, 1))]
    s_iter = statistics.median(s["s_iter"] for s in samples)
    fixed = statistics.median(s["fixed_s"] for s in samples)
    if n_ref is None:
        emit({"impl": "reference", "unavailable":
              "no recorded full-fix iteration counts for dims %s" % (dims,)})
        return
    # one step: the E_CONFIGS fixes, each GLU's recorded iteration count
    s0 = samples[0]
    model = reference_model(dict(s0, s_iter=s_iter, fixed_s=fixed,
                                 fft_thread_s_iter=statistics.median(
                                     x["fft_thread_s_iter"] for x in samples)),
                            n_ref, dims)
    t_set = model["t_set"]
    value = model["value"]
    emit({"metric": metric_name(dims), "value": value, "unit": UNIT, "n_gpus": world,
          "steps": args.steps, "warmup": args.warmup,
          "ms_per_step": t_set * 1e3, "higher_is_better": True,
          "scaling": "weak", "vs_baseline": None, "dtype": "f64",
          "data": "synthetic: %d configurations, %s (generated on the GPU)"
                  % (E_CONFIGS, (INPUT_NAME % 2).replace(
                      "seed 2", "seeds 2..%d" % (1 + E_CONFIGS))),
          "config": {"workload": "Landau FACG theta<1e-14, %s, %d configurations per step"
                                 % ("x".join(map(str, dims)), E_CONFIGS),
                     "dims": list(dims), "gf_alpha": ALPHA, "accuracy": ACC,
                     "full_fix_iters": n_ref, "parallelism": "host OpenMP"},
          "impl": "reference",
          "cpu_baseline": {"value": value, "unit": UNIT, "cores": s0["cores"],
                           "physical_cores": model["physical_cores"],
                           "kind": s0["kind"],
                           "value_excluding_fft": model["value_excluding_fft"],
                           "model": {k: v for k, v in model.items() if k != "t_set"},
                           "sample": "%d x %d FACG iterations per step, "
                                     "%.3f s/iteration (%.3f without the FFT phase) "
                                     "x %s iterations" %
                                     (len(samples), s0["sample_iters"], s_iter,
                                      model["s_per_iteration_excluding_fft"], n_ref)},
          "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                  "d2h_bytes_per_step": 0}})


def gpu_line(args, dims, world, res, cpu):
    prec = args.precision
    o = res["out"][prec]
    o64 = res["out"]["fp64"]
    steps = args.steps
    ms_step = o["ms"] / steps
    nfix = world * steps * E_CONFIGS
    value = nfix * 3600e3 / o["ms"]
    e2e = nfix * 3600e3 / o["e2e_ms"]
    V = res["V"]
    # dominant kernel over the step's fixes: per-launch time x launches
    peak, peak_src = peaks()
    it32 = sum(x[1] for x in o["per"]) if prec == "mixed" else 0
    it64 = sum(x[0] for x in o["per"]) - it32
    share = []
    for tag, n in (("fp32", it32), ("polish" if prec == "mixed" else "fp64", it64)):
        ms, by = res["prof"][tag]
        for k in range(6):
            share.append((ms[k] * n, tag, k, ms[k], by[k]))
    tot = sum(s[0] for s in share)
    top = max(share)
    _, tag, k, k_ms, k_by = top
    achieved = k_by / (k_ms * 1e-3) / 1e9
    traffic = traffic_from_profiles(KERNELS[k], tag, dims)
    per_kernel = {f"{KERNELS[j]}:{t}": {"ms": round(m, 5), "GB/s": round(b / (m * 1e-3) / 1e9, 1)}
                  for t in ("fp32", "polish", "fp64") if (t == "fp64" or prec == "mixed")
                  for j, (m, b) in enumerate(zip(*res["prof"][t])) if j < 6}
    line = {
        "metric": metric_name(dims), "value": value, "unit": UNIT, "n_gpus": world,
        "steps": steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if prec == "mixed" else "f64",
        "data": "synthetic: %d configurations per step, %s (generated on the GPU "
                "before timing)" % (E_CONFIGS, (INPUT_NAME % 2).replace(
                    "seed 2", "seeds 2..%d on every rank" % (1 + E_CONFIGS))),
        "config": {"workload": "Landau FACG theta<1e-14, %s, %d configurations per step"
                               % ("x".join(map(str, dims)), E_CONFIGS),
                   "dims": list(dims), "gf_alpha": ALPHA, "accuracy": ACC,
                   "precision": prec, "switch_theta": 1e-9 if prec == "mixed" else None,
                   "iters_per_config": [x[0] for x in o["per"]],
                   "iters_fp32_per_config": [x[1] for x in o["per"]],
                   "final_theta_max": max(x[2] for x in o["per"]),
                   "plaquette_change_max": max(o["plaq_drift"], o64["plaq_drift"]),
                   "ms_per_config": ms_step / E_CONFIGS,
                   "fp64_only": {"value": nfix * 3600e3 / o64["ms"],
                                 "ms_per_step": o64["ms"] / steps,
                                 "iters_per_config": [x[0] for x in o64["per"]],
                                 "e2e": nfix * 3600e3 / o64["e2e_ms"]},
                   "l2": "inputs (%.2f GB of links each) larger than the 126 MB L2" % (V * 576 / 1e9),
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": E_CONFIGS * V * 576,
                "d2h_bytes_per_step": E_CONFIGS * V * 576},
        "roofline": {"bound": "hbm", "kernel": f"{KERNELS[k]} ({tag})",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src,
                     "frac_of_nominal": achieved / HBM_NOMINAL_GBS,
                     "traffic": traffic, "algorithmic_bytes": k_by,
                     "share_of_fix": top[0] / tot if tot else None,
                     "per_kernel": per_kernel},
        "gpu_launches": o["launches"],
        "clocks": res["clocks"],
    }
    if cpu:
        line["cpu_baseline"] = cpu
    return line


def profile_only(args, dims):
    import ctypes as C
    import torch
    from glu_b200 import _lib
    from glu_b200._lib import check
    lib = _lib.load()
    # the per-iteration kernel costs do not depend on the configuration: the
    # tiled stand-in keeps this launch list short (no heatbath generation)
    from glu_b200.workload import tiled_config
    U = tiled_config(dims, seed=2)
    d = torch.from_numpy(U.view(np.float64).reshape(-1)).to("cuda")
    cd = (C.c_size_t * 4)(*dims)
    ms = np.zeros(7)
    by = np.zeros(7)
    pp = _params(args.precision)
    if args.precision == "polish":
        pp.precision = 2
    check(lib.gfix_profile_landau(d.data_ptr(), cd, C.byref(pp),
                                  args.profile_iters,
                                  ms.ctypes.data_as(C.POINTER(C.c_double)),
                                  by.ctypes.data_as(C.POINTER(C.c_double))))
    tag = {"mixed": "fp32", "fp64": "fp64", "polish": "polish"}[args.precision]
    emit({"profile": tag, "dims": list(dims), "iters": args.profile_iters,
          "kernels": {f"{KERNELS[k]}:{tag}": {"ms": ms[k], "bytes": by[k],
                                              "GB/s": by[k] / (ms[k] * 1e-3) / 1e9 if ms[k] else None}
                      for k in range(7)}})


# ---------------------------------------------------------------------------
# Coulomb workload: every time slice of a 64^3x128 configuration fixed to
# theta < 1e-14 (GLU's Coulomb_FA, FACG), all slices in one batched launch
# sequence.  FP64.

def c_metric_name(dims) -> str:
    return ("Coulomb-gauge-fixed configs/hour (%dx%dx%dx%d FACG, theta<1e-14 per slice)"
            % tuple(dims))
C_ALPHA = 0.08
C_KERNELS = ["k_cderiv", "k_fft_xy_fwd_c", "k_fft_z_c", "k_fft_xy_bwd_sums_c",
             "k_cprobe", "k_cupdate", "k_cscalar"]


# the input of the Coulomb workload: a beta 6.0 heatbath configuration
# generated on the GPU (seed 4, rank r: 4 + r), C_HB_ITERS iterations of one
# heatbath and four over-relaxation sweeps from the unit start -- 1000 at
# 64^3x128 would take ~3.5 minutes of GPU time per run, and its plaquette is
# settled well before 200
C_HB_ITERS = 200
C_INPUT = "heatbath beta 6.0, %d x (HB + 4 OR), unit start, seed %%d" % C_HB_ITERS


def coulomb_input(dims, seed):
    """the Coulomb workload's input, on the device (no host copy)"""
    from glu_b200.workload import heatbath_config_device
    return heatbath_config_device(dims, seed=seed, iterations=C_HB_ITERS, beta=6.0, n_or=4)


def _cparams(prec: str = "fp64"):
    p = _params(prec)
    p.gf_alpha = C_ALPHA
    return p


def coulomb_steps_record(dims):
    """Slice steps (iterations + one SD start per slice) of a full Coulomb
    fix of this workload, recorded from a GPU run (the per-slice iteration
    counts of the GPU path follow the reference's within a few)."""
    f = ROOT / "profiles" / "coulomb_full_fix.json"
    if f.exists():
        for e in json.loads(f.read_text()):
            if tuple(e["dims"]) == tuple(dims) and e.get("input") == C_INPUT % 4:
                return int(e["slice_steps"]), e
    return None, None


def coulomb_cpu_sample(U2, dims, nthreads, k=3):
    """Seconds per slice step of GLU's Coulomb_FA (oracle/_ref) on the
    host cores: a 2-slice lattice of the same spatial extent, k iterations
    per run at an unreachable accuracy, so each slice runs 1 + 8 restarts of
    (1 SD start + k CG steps)."""
    from oracle.oracle import REF_SO, Reference
    if not REF_SO.exists():
        raise RuntimeError("oracle/_ref (the reference build) is not present")
    d2 = (dims[0], dims[1], dims[2], 2)
    R = Reference()
    R.setup(d2, nthreads, C_ALPHA)
    R.put_links(U2)
    t = time.perf_counter()
    it = R.coulomb_fa(1e-30, k, "FACG")["iters"]
    el = time.perf_counter() - t
    steps = it + 2 * 9  # + one SD start per run
    return dict(kind="reference", cores=nthreads, s_step=el / steps,
                steps=steps, seconds=el)


def coulomb_gpu(args, dims, rank, world, local):
    import ctypes as C
    import torch
    torch.cuda.set_device(local)
    from glu_b200 import _lib
    from glu_b200._lib import GfixResult, check
    lib = _lib.load()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    U = coulomb_input(dims, 4 + rank)
    dpristine = torch.view_as_real(U).reshape(-1).contiguous()
    del U
    dwork = torch.empty_like(dpristine)
    hwork = torch.empty(dpristine.shape, dtype=torch.float64, pin_memory=True)
    cd = (C.c_size_t * 4)(*dims)
    V = int(np.prod(dims))
    T = dims[3]
    sth = np.zeros(T)
    sit = np.zeros(T, dtype=np.uintp)

    def fix(ptr, device, prec):
        r = GfixResult()
        p = _cparams(prec)
        fn = lib.gfix_coulomb_device if device else lib.gfix_coulomb
        check(fn(ptr, cd, C.byref(p), C.byref(r),
                 sth.ctypes.data_as(C.POINTER(C.c_double)),
                 sit.ctypes.data_as(C.POINTER(C.c_size_t))))
        return r

    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    out = {}
    with Clocks(local) as clk:
        for prec in ([args.precision, "fp64"] if args.precision == "mixed"
                     else ["fp64"]):
            for _ in range(args.warmup):
                dwork.copy_(dpristine)
                fix(dwork.data_ptr(), True, prec)
            ms = 0.0
            launches0 = lib.gfix_kernel_launches()
            iters = []
            for _ in range(args.steps):
                # the pristine copy is refreshed outside the timed region
                dwork.copy_(dpristine)
                barrier()
                a, b = ev(), ev()
                a.record()
                r = fix(dwork.data_ptr(), True, prec)
                b.record()
                barrier()
                ms += a.elapsed_time(b)
                iters.append(int(r.iters))
            launches = lib.gfix_kernel_launches() - launches0
            ms = max_over_ranks(ms)
            theta = float(np.max(sth))
            slice_iters = sit.astype(np.int64).copy()
            e_ms = 0.0
            for _ in range(args.steps):
                hwork.copy_(dpristine)
                barrier()
                a, b = ev(), ev()
                a.record()
                fix(hwork.data_ptr(), False, prec)
                b.record()
                torch.cuda.synchronize()
                e_ms += a.elapsed_time(b)
            e_ms = max_over_ranks(e_ms)
            out[prec] = dict(ms=ms, e2e_ms=e_ms, iters=iters, theta=theta,
                             iters_fp32=int(r.iters_fp32),
                             slice_iters=slice_iters, launches=launches)
    prof = {}
    for prec in ("fp64", "mixed") if args.precision == "mixed" else ("fp64",):
        pm = np.zeros(7)
        pb = np.zeros(7)
        check(lib.gfix_profile_coulomb(dpristine.data_ptr(), cd,
                                       C.byref(_cparams(prec)), args.profile_iters,
                                       pm.ctypes.data_as(C.POINTER(C.c_double)),
                                       pb.ctypes.data_as(C.POINTER(C.c_double))))
        prof["fp32" if prec == "mixed" else "fp64"] = (pm, pb)
    U2 = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the first two slices of the input, for the host sample
        U2 = torch.view_as_complex(
            dpristine[: 2 * V // T * 72].reshape(-1, 2)).reshape(-1, 4, 3, 3).cpu().numpy()
    if dist is not None:
        dist.destroy_process_group()
    res = dict(out[args.precision])
    res.update(clocks=clk.summary(), prof=prof, V=V, out=out)
    return res, U2


def coulomb_line(args, dims, world, res, cpu):
    steps = args.steps
    peak, peak_src = peaks()
    # dominant kernel over a fix: per-step time x slice steps in its precision
    n32 = res["iters_fp32"] if args.precision == "mixed" else 0
    n64 = res["iters"][-1] - n32
    cand = [(res["prof"][tag][0][j] * n, tag, j)
            for tag, n in (("fp32", n32), ("fp64", n64)) if tag in res["prof"]
            for j in range(6)]
    _, tag, k = max(cand)
    pm, pb = res["prof"][tag]
    achieved = pb[k] / (pm[k] * 1e-3) / 1e9
    traffic = traffic_from_profiles(C_KERNELS[k], tag, dims)
    V = res["V"]
    return {
        "metric": c_metric_name(dims), "value": world * steps * 3600e3 / res["ms"],
        "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": res["ms"] / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if args.precision == "mixed" else "f64",
        "data": "synthetic: %s (generated on the GPU before timing; rank r: seed 4 + r)"
                % (C_INPUT % 4),
        "config": {"workload": "Coulomb FACG theta<1e-14 per slice, %s" % "x".join(map(str, dims)),
                   "dims": list(dims), "gf_alpha": C_ALPHA, "accuracy": ACC,
                   "precision": args.precision, "iters": res["iters"][-1],
                   "iters_fp32": res["iters_fp32"],
                   "switch_theta": 1e-9 if args.precision == "mixed" else None,
                   "fp64_only": {"value": world * steps * 3600e3 / res["out"]["fp64"]["ms"],
                                 "ms_per_step": res["out"]["fp64"]["ms"] / steps,
                                 "iters": res["out"]["fp64"]["iters"][-1],
                                 "e2e": world * steps * 3600e3 / res["out"]["fp64"]["e2e_ms"]},
                   "slice_iters_min_max": [int(res["slice_iters"].min()),
                                           int(res["slice_iters"].max())],
                   "slice_steps": int(res["slice_iters"].sum() + dims[3]),
                   "final_theta_max": res["theta"],
                   "l2": "inputs (%.2f GB of links) larger than the 126 MB L2" % (V * 576 / 1e9),
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "e2e": {"value": world * steps * 3600e3 / res["e2e_ms"], "unit": UNIT,
                "h2d_bytes_per_step": V * 576, "d2h_bytes_per_step": V * 576},
        "roofline": {"bound": "hbm", "kernel": "%s (%s)" % (C_KERNELS[k], tag),
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src,
                     "frac_of_nominal": achieved / HBM_NOMINAL_GBS,
                     "traffic": traffic, "algorithmic_bytes": pb[k],
                     "per_kernel": {"%s:%s" % (C_KERNELS[j], t):
                                    {"ms": round(res["prof"][t][0][j], 5),
                                     "GB/s": round(res["prof"][t][1][j] / (res["prof"][t][0][j] * 1e-3) / 1e9, 1)
                                     if res["prof"][t][1][j] else None}
                                    for t in res["prof"] for j in range(7)}},
        "gpu_launches": res["launches"],
        "clocks": res["clocks"],
        **({"cpu_baseline": cpu} if cpu else {}),
    }


def coulomb_profile_only(args, dims):
    import ctypes as C
    import torch
    from glu_b200 import _lib
    from glu_b200._lib import check
    from glu_b200.workload import tiled_config_device
    lib = _lib.load()
    d = torch.view_as_real(tiled_config_device(dims, seed=4)).reshape(-1).contiguous()
    cd = (C.c_size_t * 4)(*dims)
    ms = np.zeros(7)
    by = np.zeros(7)
    check(lib.gfix_profile_coulomb(d.data_ptr(), cd, C.byref(_cparams(args.precision)),
                                   args.profile_iters,
                                   ms.ctypes.data_as(C.POINTER(C.c_double)),
                                   by.ctypes.data_as(C.POINTER(C.c_double))))
    emit({"profile": "coulomb " + ("fp32" if args.precision == "mixed" else "fp64"),
          "dims": list(dims), "iters": args.profile_iters,
          "kernels": {C_KERNELS[k]: {"ms": ms[k], "bytes": by[k],
                                     "GB/s": by[k] / (ms[k] * 1e-3) / 1e9 if ms[k] else None}
                      for k in range(7)}})


def coulomb_shard(args, dims, rank, world, local):
    """One configuration, its time slices split over the ranks
    (glu_b200.shard): every step fixes the whole configuration."""
    import datetime
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    from glu_b200.shard import coulomb_sharded, slice_blocks
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    t0, t1 = slice_blocks(dims[3], world)[rank]
    lcu = dims[0] * dims[1] * dims[2]
    U = coulomb_input(dims, 4)
    block = torch.view_as_real(U[t0 * lcu:t1 * lcu]).reshape(-1).contiguous()
    del U
    bdims = (dims[0], dims[1], dims[2], t1 - t0)
    work = torch.empty_like(block)
    hwork = torch.empty(block.shape, dtype=torch.float64, pin_memory=True)
    p = _cparams(args.precision)
    from glu_b200 import _lib
    lib = _lib.load()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    with Clocks(local) as clk:
        ms, e_ms, iters = 0.0, 0.0, 0
        l0 = 0
        for k in range(args.warmup + args.steps):
            if k == args.warmup:
                l0 = lib.gfix_kernel_launches()
            work.copy_(block)
            barrier()
            a, b = ev(), ev()
            a.record()
            r = coulomb_sharded(work, bdims, params=p)
            b.record()
            barrier()
            if k >= args.warmup:
                ms += a.elapsed_time(b)
                iters = r.iters
        launches = lib.gfix_kernel_launches() - l0
        for _ in range(args.steps):
            hwork.copy_(block)
            barrier()
            a, b = ev(), ev()
            a.record()
            work.copy_(hwork, non_blocking=True)
            coulomb_sharded(work, bdims, params=p)
            hwork.copy_(work)
            b.record()
            barrier()
            e_ms += a.elapsed_time(b)
    ms, e_ms = max_over_ranks(ms), max_over_ranks(e_ms)
    if rank == 0:
        steps = args.steps
        emit({"metric": c_metric_name(dims), "value": steps * 3600e3 / ms, "unit": UNIT,
              "n_gpus": world, "steps": steps, "warmup": args.warmup,
              "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "strong",
              "vs_baseline": None, "dtype": "f32+f64" if args.precision == "mixed" else "f64",
              "data": "synthetic: %s (generated on the GPU before timing)" % (C_INPUT % 4),
              "config": {"workload": "Coulomb FACG theta<1e-14 per slice, %s, slices split over ranks"
                                     % "x".join(map(str, dims)),
                         "dims": list(dims), "precision": args.precision, "iters": iters,
                         "slices_per_rank": t1 - t0,
                         "l2": "inputs larger than the 126 MB L2",
                         "parallelism": "time slices sharded over %d GPUs, ring exchange of "
                                        "one slice's gauge field" % world},
              "e2e": {"value": steps * 3600e3 / e_ms, "unit": UNIT,
                      "h2d_bytes_per_step": block.numel() * 8 * world,
                      "d2h_bytes_per_step": block.numel() * 8 * world},
              "gpu_launches": launches, "clocks": clk.summary()})
    if world > 1:
        dist.destroy_process_group()


def coulomb_main(args, dims, rank, world, local):
    if args.profile_only:
        coulomb_profile_only(args, dims)
        return
    if args.impl == "reference":
        if rank != 0:
            return
        n_steps, _ = coulomb_steps_record(dims)
        if n_steps is None:
            emit({"impl": "reference", "unavailable":
                  "no recorded slice-step count of a full Coulomb fix for dims %s" % (dims,)})
            return
        from glu_b200.workload import tiled_config_device
        U = tiled_config_device((dims[0], dims[1], dims[2], 8), seed=4, device="cpu")
        U2 = U[: 2 * dims[0] * dims[1] * dims[2]].numpy()
        cores = os.cpu_count() or 1
        samples = [coulomb_cpu_sample(U2, dims, cores) for _ in range(max(args.steps, 1))]
        s_step = statistics.median(x["s_step"] for x in samples)
        t_fix = s_step * n_steps
        value = 3600.0 / t_fix
        emit({"metric": c_metric_name(dims), "value": value, "unit": UNIT, "n_gpus": world,
              "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_fix * 1e3,
              "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
              "dtype": "f64", "data": "synthetic (8^4 GLU heatbath tiled + random gauge)",
              "config": {"workload": "Coulomb FACG theta<1e-14 per slice, %s" % "x".join(map(str, dims)),
                         "dims": list(dims), "slice_steps": n_steps,
                         "parallelism": "host OpenMP"},
              "impl": "reference",
              "cpu_baseline": {"value": value, "unit": UNIT, "cores": samples[0]["cores"],
                               "kind": "reference",
                               "sample": "%d x %d slice steps of a 2-slice %dx%dx%d lattice; "
                                         "%.3f s/slice step x %d slice steps"
                                         % (len(samples), samples[0]["steps"], dims[0], dims[1],
                                            dims[2], s_step, n_steps)},
              "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                      "d2h_bytes_per_step": 0}})
        return
    if args.shard:
        coulomb_shard(args, dims, rank, world, local)
        return
    res, U2 = coulomb_gpu(args, dims, rank, world, local)
    cpu = None
    if U2 is not None:
        try:
            s = coulomb_cpu_sample(U2, dims, os.cpu_count() or 1)
            n_steps = int(res["out"]["fp64"]["slice_iters"].sum() + dims[3])
            t_fix = s["s_step"] * n_steps
            cpu = {"value": 3600.0 / t_fix, "unit": UNIT, "cores": s["cores"],
                   "kind": s["kind"],
                   "sample": "%d slice steps of a 2-slice %dx%dx%d lattice (%.1f s); "
                             "%.3f s/slice step x %d slice steps of the full fix"
                             % (s["steps"], dims[0], dims[1], dims[2], s["seconds"],
                                s["s_step"], n_steps)}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "kind": "unavailable", "sample": str(e)}
    if rank == 0:
        emit(coulomb_line(args, dims, world, res, cpu))


# ---------------------------------------------------------------------------
# Ensemble workload: 48 configurations of 16^3x32 and 16 of 24^3x48 fixed in
# one batch (gfix_batch_*), Landau FASD to theta < 1e-12, mixed precision.
# A step is the fix of the whole ensemble; value counts configurations.

E_GROUPS = ((48, (16, 16, 16, 32)), (16, (24, 24, 24, 48)))
E_ACC = 1e-12


def e_metric_name() -> str:
    return ("gauge-fixed configs/hour (ensemble 48x16^3x32 + 16x24^3x48, "
            "Landau FASD, theta<1e-12)")


E_HB_ITERS = 500  # heatbath steps (1 HB + 4 OR) generating each configuration


def ensemble_configs(rank: int = 0, tiled: bool = False):
    """(dims, links) per configuration: heatbath configurations generated on
    the GPU, beta spread evenly over 5.9 .. 6.1 across the 64, seeds
    100..163 (offset by 64 per rank), E_HB_ITERS steps of one heatbath and
    four over-relaxation sweeps from the unit start.  tiled: the host-built
    stand-in of the same shapes (the 8^4 heatbath configuration tiled, with
    a seeded gauge transformation), for timing the reference's iterations,
    whose cost does not depend on the configuration."""
    from glu_b200.workload import heatbath_config, tiled_config
    ntot = sum(n for n, _ in E_GROUPS)
    out, k = [], 0
    for n, dims in E_GROUPS:
        for _ in range(n):
            seed = 100 + 64 * rank + k
            beta = 5.9 + 0.2 * k / (ntot - 1)
            U = (tiled_config(dims, seed=seed) if tiled else
                 heatbath_config(dims, seed=seed, iterations=E_HB_ITERS, beta=beta))
            out.append((dims, U))
            k += 1
    return out


def _eparams(prec: str):
    p = _params(prec)
    p.algo = 1          # FASD (line search)
    p.accuracy = E_ACC
    return p


def ensemble_main(args, rank, world, local):
    import ctypes as C
    import torch
    if args.impl == "reference":
        if rank != 0:
            return
        cfgs = ensemble_configs(0, tiled=True)
        rec = ensemble_iters_record()
        if rec is None:
            emit({"impl": "reference", "unavailable":
                  "no recorded FASD iteration counts of the ensemble"})
            return
        cores = os.cpu_count() or 1
        t_fix = 0.0
        samples = []
        for n, dims in E_GROUPS:
            U = next(u for d, u in cfgs if d == dims)
            s = cpu_sample(U, dims, args.cpu_sample_s / 2, cores, "FASD")
            samples.append(s)
            t_fix += n * s["fixed_s"] + s["s_iter"] * rec[str(dims[0])]
        value = len(cfgs) * 3600.0 / t_fix
        emit({"metric": e_metric_name(), "value": value, "unit": UNIT,
              "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
              "ms_per_step": t_fix * 1e3, "higher_is_better": True,
              "scaling": "weak", "vs_baseline": None, "dtype": "f64",
              "data": "synthetic: GLU's FASD cost per iteration sampled on the 8^4 GLU heatbath "
                      "tiled + random gauge stand-in; iteration counts are the FP64 FASD counts "
                      "recorded on the heatbath ensemble (beta 5.9-6.1, seeds 100-163)",
              "config": {"workload": "ensemble 48x16^3x32 + 16x24^3x48 Landau FASD theta<1e-12",
                         "configs": len(cfgs), "full_fix_iters_by_group": rec,
                         "parallelism": "host OpenMP, one configuration at a time"},
              "impl": "reference",
              "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores,
                               "kind": samples[0]["kind"],
                               "sample": "; ".join("%s: %d FASD iterations, %.3f s/iteration"
                                                   % ("x".join(map(str, d)), s["sample_iters"], s["s_iter"])
                                                   for (n, d), s in zip(E_GROUPS, samples))},
              "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                      "d2h_bytes_per_step": 0}})
        return
    torch.cuda.set_device(local)
    from glu_b200 import _lib
    from glu_b200._lib import GfixResult, check
    lib = _lib.load()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    cfgs = ensemble_configs(rank)
    pristine = [torch.from_numpy(u.view(np.float64).reshape(-1)).to("cuda") for _, u in cfgs]
    work = [torch.empty_like(t) for t in pristine]
    hwork = [torch.empty(t.shape, dtype=torch.float64, pin_memory=True) for t in pristine]
    cds = [(C.c_size_t * 4)(*d) for d, _ in cfgs]
    nbytes = sum(t.numel() * 8 for t in pristine)
    sites = sum(int(np.prod(d)) for d, _ in cfgs)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    out = {}
    with Clocks(local) as clk:
        for prec in ([args.precision, "fp64"] if args.precision == "mixed" else ["fp64"]):
            p = _eparams(prec)
            res = {}
            for mode in ("device", "host"):
                b = lib.gfix_batch_create(C.byref(p))
                if not b:
                    check(-1)
                try:
                    for i in range(len(cfgs)):
                        ptr = work[i].data_ptr() if mode == "device" else hwork[i].data_ptr()
                        add = lib.gfix_batch_add_device if mode == "device" else lib.gfix_batch_add
                        if add(b, ptr, cds[i]) < 0:
                            check(-1)
                    ms = 0.0
                    l0 = 0
                    for k in range(args.warmup + args.steps):
                        if k == args.warmup:
                            l0 = lib.gfix_kernel_launches()
                        for i in range(len(cfgs)):
                            (work[i] if mode == "device" else hwork[i]).copy_(pristine[i])
                        barrier()
                        a, e = ev(), ev()
                        a.record()
                        check(lib.gfix_batch_run(b))
                        e.record()
                        barrier()
                        if k >= args.warmup:
                            ms += a.elapsed_time(e)
                    launches = lib.gfix_kernel_launches() - l0
                    its = []
                    for i in range(len(cfgs)):
                        r = GfixResult()
                        check(lib.gfix_batch_result(b, i, C.byref(r)))
                        its.append((int(r.iters), int(r.iters_fp32), float(r.theta)))
                    res[mode] = dict(ms=max_over_ranks(ms), iters=its, launches=launches)
                finally:
                    lib.gfix_batch_destroy(b)
            out[prec] = res
    prec = args.precision
    steps = args.steps
    n = len(cfgs)
    o = out[prec]["device"]
    line = {
        "metric": e_metric_name(), "value": world * n * steps * 3600e3 / o["ms"],
        "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": o["ms"] / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if prec == "mixed" else "f64",
        "data": "synthetic: heatbath configurations generated on the GPU before timing, "
                "beta 5.9-6.1, seeds 100-163, %d x (HB + 4 OR) from the unit start" % E_HB_ITERS,
        "config": {"workload": "ensemble 48x16^3x32 + 16x24^3x48 Landau FASD theta<1e-12",
                   "configs": n, "sites": sites, "precision": prec,
                   "switch_theta": 1e-9 if prec == "mixed" else None,
                   "iters_min_max": [min(x[0] for x in o["iters"]), max(x[0] for x in o["iters"])],
                   "iters_total": sum(x[0] for x in o["iters"]),
                   "final_theta_max": max(x[2] for x in o["iters"]),
                   "fp64_only": {"value": world * n * steps * 3600e3 / out["fp64"]["device"]["ms"],
                                 "ms_per_step": out["fp64"]["device"]["ms"] / steps,
                                 "iters_total": sum(x[0] for x in out["fp64"]["device"]["iters"]),
                                 "iters_by_group": {
                                     str(d[0]): sum(x[0] for x, (dd, _) in
                                                    zip(out["fp64"]["device"]["iters"], cfgs)
                                                    if dd == d)
                                     for _, d in E_GROUPS},
                                 "e2e": world * n * steps * 3600e3 / out["fp64"]["host"]["ms"]},
                   "l2": "inputs (%.2f GB of links) larger than the 126 MB L2" % (nbytes / 1e9),
                   "parallelism": "one batch per GPU" if world > 1 else "single GPU, one batch"},
        "e2e": {"value": world * n * steps * 3600e3 / out[prec]["host"]["ms"], "unit": UNIT,
                "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
        "gpu_launches": o["launches"],
        "clocks": clk.summary(),
    }
    # roofline: the kernel with the largest share of the batch's device time,
    # from per-kernel event times of each shape and phase (gfix_profile_landau:
    # CG iterations of the same kernels, on one configuration of the shape)
    # weighted by the iterations the batch spent in that shape and phase
    peak, peak_src = peaks()
    share = []
    i0 = 0
    for cnt, dims in E_GROUPS:
        its = o["iters"][i0:i0 + cnt]
        it32 = sum(x[1] for x in its) if prec == "mixed" else 0
        it64 = sum(x[0] for x in its) - it32
        phases = ((("fp32", 1, it32), ("polish", 2, it64)) if prec == "mixed"
                  else (("fp64", 0, it64),))
        for tag, code, n_it in phases:
            if n_it <= 0:
                continue
            pms, pby = np.zeros(7), np.zeros(7)
            pp = _eparams("fp64")
            pp.precision = code
            check(lib.gfix_profile_landau(pristine[i0].data_ptr(), cds[i0], C.byref(pp),
                                          args.profile_iters,
                                          pms.ctypes.data_as(C.POINTER(C.c_double)),
                                          pby.ctypes.data_as(C.POINTER(C.c_double))))
            for k in range(6):
                share.append((pms[k] * n_it, tag, dims, k, pms[k], pby[k]))
        i0 += cnt
    if share:
        tot = sum(x[0] for x in share)
        top = max(share, key=lambda x: x[0])
        _, tag, dims, k, k_ms, k_by = top
        achieved = k_by / (k_ms * 1e-3) / 1e9
        line["roofline"] = {"bound": "hbm",
                            "kernel": "%s (%s, %s)" % (KERNELS[k], tag, "x".join(map(str, dims))),
                            "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "peak_source": peak_src,
                            "frac_of_nominal": achieved / HBM_NOMINAL_GBS,
                            # no ncu capture of these shapes: their fields fit
                            # in L2, so scaling the 32^3x64 one would mislead
                            "traffic": None,
                            "algorithmic_bytes": k_by,
                            "share_of_fix": top[0] / tot if tot else None}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            f64 = out["fp64"]["device"]["iters"]
            t_fix = 0.0
            desc = []
            cores = os.cpu_count() or 1
            i0 = 0
            for cnt, dims in E_GROUPS:
                s = cpu_sample(cfgs[i0][1], dims, args.cpu_sample_s / 2, cores, "FASD")
                its = sum(x[0] for x in f64[i0:i0 + cnt])
                t_fix += cnt * s["fixed_s"] + s["s_iter"] * its
                desc.append("%s: %d FASD iterations sampled, %.3f s/iteration x %d iterations"
                            % ("x".join(map(str, dims)), s["sample_iters"], s["s_iter"], its))
                i0 += cnt
            line["cpu_baseline"] = {"value": n * 3600.0 / t_fix, "unit": UNIT,
                                    "cores": cores, "kind": s["kind"], "sample": "; ".join(desc)}
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "kind": "unavailable", "sample": str(e)}
    if rank == 0:
        emit(line)


def ensemble_iters_record():
    f = ROOT / "profiles" / "ensemble_fix.json"
    if f.exists():
        return json.loads(f.read_text()).get("fasd_fp64_iters_by_group")
    return None


# ---------------------------------------------------------------------
# gluon propagators: GLU's cuts_struct (CUTTYPE = GLUON_PROPS) with the cut
# of GLU's shipped input file (CONF/input_file: CYLINDER_CUT, MAXMOM 4,
# CYL_WIDTH 2.0, ANGLE 60, FIELD_DEFINITION LINEAR)

G_CUT = dict(cuttype="GLUON_PROPS", mom_cut="CYLINDER_CUT", field_definition="LINEAR",
             maxmom=4, angle=60, cyl_width=2.0)
G_UNIT = "measurements/hour"


def g_metric_name(dims) -> str:
    return ("gluon propagator measurements/hour (%dx%dx%dx%d Landau-fixed, "
            "GLUON_PROPS CYLINDER_CUT MAXMOM 4)" % tuple(dims))


def g_workload(dims) -> dict:
    return {"workload": "gluon propagators %s (cuts_struct GLUON_PROPS)" % "x".join(map(str, dims)),
            "cut": "CYLINDER_CUT MAXMOM 4 CYL_WIDTH 2.0 ANGLE 60, LINEAR fields"}


def g_reference_time(U, dims, nthreads):
    """seconds of one GLU cuts_struct on the host cores (oracle/_ref)."""
    import tempfile
    from oracle import oracle as O
    R = O.Reference()
    R.setup(dims, nthreads)
    R.put_links(U)
    with tempfile.TemporaryDirectory() as td:
        t0 = time.perf_counter()
        R.cuts(td, 6, 2, 4, 0, 60, 2.0, flow=1)
        return time.perf_counter() - t0


def g_input(dims, rank):
    """the synthetic stand-in, Landau-fixed to theta < 1e-14 on the GPU
    (outside any timed region)."""
    from glu_b200 import gfix
    from glu_b200.workload import tiled_config
    U = tiled_config(dims, seed=2 + rank)
    return gfix.landau_fix(U, dims, accuracy=ACC, precision="MIXED").links


def gluonprop_main(args, dims, rank, world, local):
    import ctypes as C
    import torch
    if args.impl == "reference":
        if rank != 0:
            return
        from glu_b200.workload import tiled_config
        U = tiled_config(dims, seed=2)  # the measurement's cost is gauge-independent
        cores = os.cpu_count() or 1
        secs = [g_reference_time(U, dims, cores) for _ in range(max(1, min(args.steps, 2)))]
        t = statistics.median(secs)
        value = 3600.0 / t
        emit({"metric": g_metric_name(dims), "value": value, "unit": G_UNIT,
              "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
              "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
              "dtype": "f64", "data": "synthetic (8^4 GLU heatbath tiled + random gauge)",
              "config": dict(g_workload(dims), parallelism="host OpenMP"),
              "impl": "reference",
              "cpu_baseline": {"value": value, "unit": G_UNIT, "cores": cores,
                               "kind": "reference",
                               "sample": "%d full GLU cuts_struct runs (FFT: the oracle's FFTW stand-in)" % len(secs)},
              "e2e": {"value": value, "unit": G_UNIT, "h2d_bytes_per_step": 0,
                      "d2h_bytes_per_step": 0}})
        return
    torch.cuda.set_device(local)
    from glu_b200 import _lib, cuts
    from glu_b200._lib import check
    lib = _lib.load()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if args.profile_only:
        # a short, bounded launch list for ncu: two measurements, no fix
        from glu_b200.workload import tiled_config
        U = tiled_config(dims, seed=2)
        d = torch.from_numpy(U.view(np.float64).reshape(-1).copy()).cuda()
        info = cuts.CutInfo(**G_CUT)
        for _ in range(2):
            r = cuts.measure_device(d, dims, info)
        torch.cuda.synchronize()
        print(json.dumps({"workload": "gluonprop profile-only", "momenta": len(r["mom"]),
                          "pspace_err": r["pspace_err"]}))
        return
    U = g_input(dims, rank)
    d_links = torch.from_numpy(U.view(np.float64).reshape(-1).copy()).cuda()
    h_links = torch.from_numpy(U.view(np.float64).reshape(-1).copy()).pin_memory()
    info = cuts.CutInfo(**G_CUT)
    ci = info.c()
    nmom = len(cuts.veclist(dims, info))
    cd = (C.c_size_t * 4)(*dims)
    o0, o1, perr = np.zeros(nmom), np.zeros(nmom), C.c_double(0.0)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    V = int(np.prod(dims))
    # L2 flush between timed steps: the transforms' inputs (1.2 GB of links
    # at 32^3x64) exceed the 126 MB L2 anyway; a 256 MB write makes it so
    # for every shape
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def run(mode):
        ms = 0.0
        l0 = 0
        for k in range(args.warmup + args.steps):
            if k == args.warmup:
                l0 = lib.gfix_kernel_launches()
            flush.zero_()
            barrier()
            a, e = ev(), ev()
            a.record()
            if mode == "device":
                rc = lib.gfix_cuts_measure_device(d_links.data_ptr(), cd, C.byref(ci), nmom,
                                                  o0.ctypes.data_as(_lib._dp),
                                                  o1.ctypes.data_as(_lib._dp), C.byref(perr))
            else:
                rc = lib.gfix_cuts_measure(h_links.data_ptr(), cd, C.byref(ci), nmom,
                                           o0.ctypes.data_as(_lib._dp),
                                           o1.ctypes.data_as(_lib._dp), C.byref(perr))
            e.record()
            if rc != 0:
                raise RuntimeError(lib.gfix_cuts_error().decode())
            barrier()
            if k >= args.warmup:
                ms += a.elapsed_time(e)
        return max_over_ranks(ms), lib.gfix_kernel_launches() - l0

    with Clocks(local) as clk:
        ms_dev, launches = run("device")
        ms_host, _ = run("host")
        kms = (C.c_float * 3)()
        if lib.gfix_profile_cuts(d_links.data_ptr(), cd, C.byref(ci), 10, kms) != 0:
            raise RuntimeError(lib.gfix_cuts_error().decode())
        # the same with FIELD_DEFINITION = LOGARITHMIC (eigenvalues and the
        # exact logarithm of every link inside the xy pass)
        lms = (C.c_float * 3)()
        ci_log = cuts.CutInfo(**dict(G_CUT, field_definition="LOGARITHMIC")).c()
        if lib.gfix_profile_cuts(d_links.data_ptr(), cd, C.byref(ci_log), 10, lms) != 0:
            raise RuntimeError(lib.gfix_cuts_error().decode())
    steps = args.steps
    hbm, peak_src = peaks()
    # algorithmic bytes per launch: xy pass reads the links (4 x 9 complex
    # FP64 per site) and writes 16 complex fields; zt pass reads and writes
    # the 16 fields
    xy_bytes = V * (4 * 9 * 16 + 16 * 16)
    zt_bytes = V * (2 * 16 * 16)
    xy_ms, zt_ms, rest_ms = (float(x) for x in kms)
    dom = ("k_cut_xy", xy_bytes, xy_ms) if xy_ms >= zt_ms else ("k_cut_zt", zt_bytes, zt_ms)
    achieved = dom[1] / (dom[2] * 1e-3) / 1e9
    traffic = traffic_from_profiles(dom[0], "fp64", dims)
    line = {
        "metric": g_metric_name(dims), "value": world * steps * 3600e3 / ms_dev,
        "unit": G_UNIT, "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": ms_dev / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (8^4 GLU heatbath beta 6.0 tiled + seeded random gauge, "
                "Landau-fixed to theta<1e-14 before timing)",
        "config": dict(g_workload(dims), momenta=nmom,
                       l2="256 MB flush between steps; %.2f GB of links" % (V * 576 / 1e9),
                       kernel_ms={"xy (Lie fields + x,y transforms)": xy_ms,
                                  "zt (z,t transforms)": zt_ms,
                                  "gather + contraction": rest_ms},
                       log_kernel_ms={"xy (logarithms + x,y transforms)": float(lms[0]),
                                      "zt": float(lms[1]), "gather + contraction": float(lms[2])},
                       parallelism="one configuration per GPU" if world > 1 else "single GPU"),
        "roofline": {"bound": "hbm", "kernel": dom[0], "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                     "frac_of_nominal": achieved / HBM_NOMINAL_GBS,
                     "peak_source": peak_src,
                     "other": {"k_cut_zt" if dom[0] == "k_cut_xy" else "k_cut_xy":
                               ((zt_bytes / zt_ms if dom[0] == "k_cut_xy" else xy_bytes / xy_ms)
                                / 1e6 / hbm)}},
        "e2e": {"value": world * steps * 3600e3 / ms_host, "unit": G_UNIT,
                "h2d_bytes_per_step": V * 576, "d2h_bytes_per_step": 2 * nmom * 8},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            t = g_reference_time(U, dims, os.cpu_count() or 1)
            line["cpu_baseline"] = {"value": 3600.0 / t, "unit": G_UNIT,
                                    "cores": os.cpu_count() or 1, "kind": "reference",
                                    "sample": "one full GLU cuts_struct (%.1f s; FFT: the oracle's FFTW stand-in)" % t}
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": G_UNIT, "kind": "unavailable",
                                    "sample": str(e)}
    if rank == 0:
        emit(line)


# ---------------------------------------------------------------------
# configuration generation: GLU's heatbath + over-relaxation update
# (hb_update's update_lattice: one heatbath sweep and four over-relaxation
# sweeps per step), beta 6.0

H_BETA, H_NOR = 6.0, 4
H_UNIT = "update steps/hour"


def h_metric_name(dims) -> str:
    return ("heatbath + 4 over-relaxation update steps/hour (%dx%dx%dx%d, beta 6.0)"
            % tuple(dims))


def h_reference_seconds(dims, nthreads, steps=2):
    """seconds per update step of GLU's own heatbath (oracle/_ref) on the
    host cores, from a thermalised-like start: a bounded sample of steps"""
    from oracle import oracle as O
    from glu_b200.workload import tiled_config
    R = O.Reference()
    R.setup(dims, nthreads, 0.08, 11)
    R.put_links(tiled_config(dims, seed=2))
    t0 = time.perf_counter()
    R.heatbath(H_BETA, steps, H_NOR)
    return (time.perf_counter() - t0) / steps, steps


def heatbath_main(args, dims, rank, world, local):
    import torch
    cfg = {"workload": "heatbath %s beta %.1f, 1 HB + %d OR sweeps per step"
                       % ("x".join(map(str, dims)), H_BETA, H_NOR),
           "generator": "Philox4x32-10, seed 1 + rank"}
    if args.impl == "reference":
        if rank != 0:
            return
        cores = os.cpu_count() or 1
        t, n = h_reference_seconds(dims, cores, max(1, min(args.steps, 2)))
        value = 3600.0 / t
        emit({"metric": h_metric_name(dims), "value": value, "unit": H_UNIT,
              "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
              "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
              "dtype": "f64", "data": "synthetic (8^4 GLU heatbath tiled + random gauge)",
              "config": dict(cfg, parallelism="host OpenMP"), "impl": "reference",
              "cpu_baseline": {"value": value, "unit": H_UNIT, "cores": cores,
                               "kind": "reference",
                               "sample": "%d GLU update steps (hb_lattice + 4 OR_lattice)" % n},
              "e2e": {"value": value, "unit": H_UNIT, "h2d_bytes_per_step": 0,
                      "d2h_bytes_per_step": 0}})
        return
    torch.cuda.set_device(local)
    import ctypes as C
    from glu_b200 import _lib
    from glu_b200.workload import tiled_config
    lib = _lib.load()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    U = tiled_config(dims, seed=2 + rank)
    V = int(np.prod(dims))
    d = torch.from_numpy(U.view(np.float64).reshape(-1).copy()).cuda()
    h = torch.from_numpy(U.view(np.float64).reshape(-1).copy()).pin_memory()
    cd = (C.c_size_t * 4)(*dims)
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    seed = 1 + rank

    def run(mode, it0):
        ms, l0 = 0.0, 0
        for k in range(args.warmup + args.steps):
            if k == args.warmup:
                l0 = lib.gfix_kernel_launches()
            barrier()
            a, e = ev(), ev()
            a.record()
            if mode == "device":
                rc = lib.gfix_heatbath_device(d.data_ptr(), cd, H_BETA, 1, H_NOR, seed,
                                              it0 + k, None)
            else:
                rc = lib.gfix_heatbath(h.data_ptr(), cd, H_BETA, 1, H_NOR, seed, it0 + k, None)
            e.record()
            if rc != 0:
                raise RuntimeError(lib.gfix_update_error().decode())
            barrier()
            if k >= args.warmup:
                ms += a.elapsed_time(e)
        return max_over_ranks(ms), lib.gfix_kernel_launches() - l0

    with Clocks(local) as clk:
        ms_dev, launches = run("device", 0)
        ms_host, _ = run("host", 1000)
        # one step's kernels alone: the layout conversion is part of the
        # device call; time 10 steps in one call to see the sweeps
        a, e = ev(), ev()
        barrier()
        a.record()
        if lib.gfix_heatbath_device(d.data_ptr(), cd, H_BETA, 10, H_NOR, seed, 5000, None):
            raise RuntimeError(lib.gfix_update_error().decode())
        e.record()
        barrier()
        ms10 = a.elapsed_time(e) / 10
    steps = args.steps
    hbm, peak_src = peaks()
    # algorithmic bytes of one (direction, colour) launch: the updated links
    # read and written (2 x 144 B x V/2), the other colour's links of that
    # direction and all links of the other three directions read for the
    # staples (144 B x (V/2 + 3 V)): 648 B per site; 8 launches per sweep
    sweep_bytes = 8 * 648 * V
    sweeps = 1 + H_NOR
    achieved = sweep_bytes * sweeps / (ms10 * 1e-3) / 1e9
    line = {
        "metric": h_metric_name(dims), "value": world * steps * 3600e3 / ms_dev,
        "unit": H_UNIT, "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": ms_dev / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (8^4 GLU heatbath beta 6.0 tiled + seeded random gauge)",
        "config": dict(cfg, ms_per_step_in_10_step_call=ms10,
                       l2="%.2f GB of links, larger than the 126 MB L2" % (V * 576 / 1e9),
                       parallelism="one lattice per GPU" if world > 1 else "single GPU"),
        "roofline": {"bound": "hbm", "kernel": "k_update", "achieved": achieved,
                     "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "frac_of_nominal": achieved / HBM_NOMINAL_GBS,
                     "traffic": traffic_from_profiles("k_update_hb", "fp64", dims),
                     "peak_source": peak_src},
        "e2e": {"value": world * steps * 3600e3 / ms_host, "unit": H_UNIT,
                "h2d_bytes_per_step": V * 576, "d2h_bytes_per_step": V * 576},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            t, n = h_reference_seconds(dims, os.cpu_count() or 1)
            line["cpu_baseline"] = {"value": 3600.0 / t, "unit": H_UNIT,
                                    "cores": os.cpu_count() or 1, "kind": "reference",
                                    "sample": "%d GLU update steps, %.2f s each" % (n, t)}
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": H_UNIT, "kind": "unavailable",
                                    "sample": str(e)}
    if rank == 0:
        emit(line)


# The other configurations of the benchmark table, each run as its own
# bench.py process after the headline's measurement (rank 0 of a one-GPU
# default run), so that the default run's line records them too: the
# ensemble (FASD, mixed), Landau 48^3x96 (one beta 6.2 configuration) and
# Coulomb 64^3x128.  Bounded by OTHERS_BUDGET_S seconds in all
# (GLU_GFIX_BENCH_OTHERS_S overrides; 0 turns this off); a workload that
# would not fit, fails or prints no line is listed as skipped, with why.
OTHERS_BUDGET_S = 780.0
OTHER_WORKLOADS = [
    ("ensemble", ["--workload", "ensemble"], 300.0),
    ("landau 48x48x48x96", ["--dims", "48,48,48,96", "--beta", "6.2", "--configs", "1"], 300.0),
    ("coulomb 64x64x64x128", ["--workload", "coulomb"], 360.0),
]


def compact_line(line: dict) -> dict:
    """The figures of another workload's bench line kept in the default
    line: metric, value, end-to-end value, step time, iteration counts,
    the FP64 comparison, the roofline fraction and the clocks."""
    c = line.get("config", {})
    keep = {k: line.get(k) for k in ("metric", "value", "unit", "steps", "warmup",
                                     "ms_per_step", "dtype", "data")}
    keep["e2e"] = (line.get("e2e") or {}).get("value")
    keep["workload"] = c.get("workload")
    for k in ("iters_per_config", "iters_total", "iters_min_max", "slice_iters_max",
              "iters", "final_theta_max", "plaquette_change_max"):
        if k in c:
            keep[k] = c[k]
    f64 = c.get("fp64_only")
    if isinstance(f64, dict):
        keep["fp64_only"] = {k: f64.get(k) for k in ("value", "e2e")}
    r = line.get("roofline") or {}
    keep["roofline"] = {k: r.get(k) for k in ("kernel", "frac", "unit", "achieved")}
    keep["clocks"] = line.get("clocks")
    return keep


def other_workloads() -> list:
    budget = float(os.environ.get("GLU_GFIX_BENCH_OTHERS_S", OTHERS_BUDGET_S))
    if budget <= 0:
        return []
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "LOCAL_WORLD_SIZE")}
    t0 = time.monotonic()
    out = []
    for name, extra, limit in OTHER_WORKLOADS:
        left = budget - (time.monotonic() - t0)
        if left < 60.0:
            out.append({"workload": name, "skipped": "the default run's time budget "
                        "(%.0f s) is spent" % budget})
            continue
        cmd = [sys.executable, str(ROOT / "bench.py"), *extra, "--steps", "1",
               "--warmup", "3", "--no-cpu-baseline"]
        t1 = time.monotonic()
        try:
            p = subprocess.run(cmd, capture_output=True, text=True, cwd=str(ROOT),
                               env=env, timeout=min(limit, left))
            lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
            if p.returncode != 0 or not lines:
                tail = (p.stderr or p.stdout).strip().splitlines()[-1:] or [""]
                out.append({"workload": name, "skipped": "exit %d: %s" % (p.returncode,
                                                                           tail[0][:200])})
                continue
            rec = compact_line(json.loads(lines[-1]))
            rec["command"] = "python bench.py " + " ".join(cmd[2:])
            rec["wall_s"] = round(time.monotonic() - t1, 1)
            out.append(rec)
        except subprocess.TimeoutExpired:
            out.append({"workload": name, "skipped": "did not finish within %.0f s"
                        % min(limit, left)})
        except Exception as e:  # reported, never fatal to the headline line
            out.append({"workload": name, "skipped": str(e)[:200]})
    return out


def main():
    args = parse()
    if args.dims is None:
        args.dims = ("32,32,32,64" if args.workload in ("landau", "gluonprop", "heatbath")
                     else "64,64,64,128")
    dims = tuple(int(x) for x in args.dims.split(","))
    rank, world, local = dist_env()
    if args.workload == "coulomb":
        coulomb_main(args, dims, rank, world, local)
        return
    if args.workload == "ensemble":
        ensemble_main(args, rank, world, local)
        return
    if args.workload == "gluonprop":
        gluonprop_main(args, dims, rank, world, local)
        return
    if args.workload == "heatbath":
        heatbath_main(args, dims, rank, world, local)
        return
    set_input(args.beta, args.configs)
    if args.profile_only:
        profile_only(args, dims)
        return
    if args.impl == "reference":
        reference_arm(args, dims, rank, world)
        return
    res, U = gpu_arm(args, dims, rank, world, local)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            n_ref = reference_iters(dims)
            s = cpu_sample(U, dims, args.cpu_sample_s, os.cpu_count() or 1)
            src = "GLU's recorded full fixes"
            if n_ref is None:  # our FP64 counts stand in for GLU's
                n_ref = [x[0] for x in res["out"]["fp64"]["per"]]
                src = "our FP64 fixes' counts"
            model = reference_model(s, n_ref, dims)
            cpu = {"value": model["value"], "unit": UNIT, "cores": s["cores"],
                   "physical_cores": model["physical_cores"], "kind": s["kind"],
                   "value_excluding_fft": model["value_excluding_fft"],
                   "model": {k: v for k, v in model.items() if k != "t_set"},
                   "sample": "%d FACG iterations (%.1f s); %.3f s/iteration x %s "
                             "iterations (%s); FFT stand-in %.3f thread-s/iteration "
                             "(%.3f s of wall time)"
                             % (s["sample_iters"], s["sample_s"], s["s_iter"], n_ref, src,
                                s["fft_thread_s_iter"], model["fft_wall_s_per_iteration"])}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "kind": "unavailable", "sample": str(e)}
    if rank == 0:
        line = gpu_line(args, dims, world, res, cpu)
        if world == 1 and args.dims == "32,32,32,64":
            # the headline's workspaces and tensors go before the others run
            import torch
            from glu_b200 import _lib
            del res, U
            _lib.load().gfix_release()
            torch.cuda.empty_cache()
            line["other_workloads"] = other_workloads()
        emit(line)


if __name__ == "__main__":
    main()
