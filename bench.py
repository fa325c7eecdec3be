"""Benchmark of the LDDMM registration hot path on B200.

Workload (default): one 3D sphere -> cube registration -- icosphere radius 1,
4 subdivisions (2562 vertices / 5120 triangles) onto the surface of [-1,1]^3 with a
32 x 32 quad grid per face (12288 triangles), Matern nu=3/2 deformation kernel width
0.4, varifold Gaussian(0.15) x Binet, 20 time steps, L-BFGS memory 5, at most 500
iterations (tolerance 1e-6, Wolfe 1e-4 / 0.9), zero initial momenta.  One "step" is
one whole registration.  Synthetic data, generated deterministically.

Metric: registrations/s (whole job, all ranks); the JSON line also reports pair
interactions/s, the objective's relative error against the FP64 oracle at the
returned point, the FP32 roofline of the dominant sweep, the reference's C++ path
timed on the host cores, and (key "population") the uneven 256-pair batch registered
in one context to 1e-5 relative objective change next to the reference's FP64 GPU
path on a seeded stratified sample of its pairs, measured in the same run.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun: every rank runs its own registration (independent
replicas, no data-path collective); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "registrations/s at 1e-5 rel. objective; Gpair-interactions/s vs FP32 peak"
UNIT = "registrations/s"
WORKLOAD = "sphere2cube: icosphere 2562 v / 5120 t -> cube 12288 t, Matern nu=3/2 w=0.4, " \
           "varifold G(0.15) x Binet, T=20, L-BFGS m=5, <=500 iterations"
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2
BATCH_PAIRS = 8  # registrations in the batched-form measurement
# the config object both arms print (identical, so that the two lines compare)
CONFIG = {"workload": WORKLOAD,
          "l2": "GPU arm: 256 MiB device memset before every timed registration; "
                "CPU arm: not applicable"}
POP_PAIRS = 256  # the uneven population: pairs registered together in one context
POP_SAMPLE = 32  # population pairs also registered by the reference's FP64 GPU path
POP_WORKLOAD = ("population: 256 star-shaped pairs (seed 0), 500-20000 landmarks and "
                "1000-40000 target triangles log-uniform, Gaussian 0.3, varifold G(0.1) x "
                "Binet, T=10, to 1e-5 relative objective change")

# The FP64 registration of this workload (CPU oracle, 500 iterations; generator
# tests/golden/make_c2_reference.py): its objective is what a registration has to
# reach (within 1e-5 relative), and its evaluation count turns the reference's
# per-evaluation CPU time into registrations/s (a whole reference registration does
# not fit the bench's time budget).
with open(os.path.join(ROOT, "tests", "golden", "sphere2cube_fp64_500.json")) as _f:
    FP64_REGISTRATION = json.load(_f)
EVALS_PER_REGISTRATION = int(FP64_REGISTRATION["evals"])


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--itr", type=int, default=500)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-population", action="store_true",
                    help="skip the 256-pair population leg and its FP64 GPU baseline")
    ap.add_argument("--mode", choices=["registration", "objgrd", "large_pair", "ws_gemm"],
                    default="registration",
                    help="objgrd: only time device-resident objective+gradient evaluations "
                         "(the command the ncu captures in profiles/ use); large_pair: the "
                         "163,842-landmark star-surface pair, --itr L-BFGS iterations "
                         "timed (default 100); ws_gemm: the warm-start network's tcgen05 "
                         "BF16 GEMM on its layer shapes, against the bf16 peak and torch")
    ap.add_argument("--evals", type=int, default=20)
    ap.add_argument("--subdiv", type=int, default=4,
                    help="objgrd mode: icosphere subdivisions of the source (4: 2562 points)")
    ap.add_argument("--persistent", type=int, default=0,
                    help="objgrd mode: 1 persistent time-loop sweeps, -1 per-step launches, "
                         "0 automatic")
    return ap.parse_args()


def workload():
    from lddmm_b200 import problem

    return problem.sphere_to_cube()


# ------------------------------------------------------------------ clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        try:
            with open(self.f.name) as fh:
                for line in fh:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        finally:
            os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4)
                          if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ------------------------------------------------------- reference (CPU) arm

def _ref_eval_worker(args):
    """One objgrd evaluation of the workload by the reference's C++ path (compiled
    from its own sources into oracle/_ref), or by the oracle port when that build is
    absent.  Returns (seconds, kind)."""
    import numpy as np

    sys.path.insert(0, ROOT)
    from oracle.oracle import Oracle, Reference

    P = workload()
    alp = np.random.default_rng(0).normal(size=P.var_num) * 0.01
    if Reference.available(3):
        R, kind = Reference(3), "reference"
    else:
        R, kind = Oracle(threads=1), "port"
    t0 = time.perf_counter()
    R.objgrd(P, alp)
    return time.perf_counter() - t0, kind


def mem_available_gb() -> float:
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) / 1e6
    except OSError:
        pass
    return 16.0


def reference_workers() -> int:
    # the reference stores an N x N x T kernel stack: ~1.05 GB per process here
    return max(1, min(os.cpu_count() or 1, int(mem_available_gb() / 1.6), 64))


def run_reference(args):
    import multiprocessing as mp

    from lddmm_b200 import replicas

    if not replicas.rank_env().reports:
        return  # the reference arm runs on rank 0 alone; the other ranks exit
    n = reference_workers()
    ctx = mp.get_context("spawn")
    with ctx.Pool(n) as pool:
        for _ in range(args.warmup):
            pool.map(_ref_eval_worker, range(n))
        t0 = time.perf_counter()
        times, kinds = [], set()
        for _ in range(args.steps):
            out = pool.map(_ref_eval_worker, range(n))
            times += [t for t, _ in out]
            kinds |= {k for _, k in out}
        wall = time.perf_counter() - t0
    per_eval = statistics.mean(times)
    value = n / (per_eval * EVALS_PER_REGISTRATION)
    kind = "reference" if kinds == {"reference"} else "port"
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": CONFIG,
        "cpu_baseline": {
            "value": value, "unit": UNIT, "cores": n, "kind": kind,
            "sample": f"{n} processes x one objective+gradient evaluation per step "
                      f"(mean {per_eval:.2f} s), scaled by {EVALS_PER_REGISTRATION} "
                      f"evaluations per registration"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------- population (uneven batch)

def population_leg(stream, local, flush):
    """The uneven 256-pair population registered in one context (one launch per sweep
    for all pairs, the L-BFGS loop as one device-side graph), to 1e-5 relative
    objective change, device-resident, CUDA events on the context stream; next to it
    the reference's plain FP64 GPU path (CUDA/src compiled unmodified, oracle/_ref) on
    a seeded stratified sample of the same pairs, each run for the iterations that
    pair took here, and this build's batch of exactly that sample."""
    import ctypes as C

    import numpy as np
    import torch

    from lddmm_b200 import _lib, api, problem
    from oracle.oracle import ReferenceCuda

    t0 = time.perf_counter()
    probs = problem.population(POP_PAIRS, seed=0, workers=max(1, min(os.cpu_count() or 1, 32)))
    t_gen = time.perf_counter() - t0

    def batch(ps, reps):
        with api.Context(ps, stream=stream.cuda_stream, device=local) as ctx:
            d = torch.zeros(ctx.var_total, dtype=torch.float64, device="cuda")
            res = (_lib.Result * len(ps))()

            def run(itr):
                o = _lib.Opt(itr, 1e-12, 1e-4, 0.9, 5, 0, 1e-5)
                d.zero_()
                rc = _lib.lib.lddmm_lbfgs_device(ctx.handle, C.byref(o),
                                                 C.c_void_p(d.data_ptr()), res)
                if rc < 0 and rc != -3:
                    _lib.check(rc)

            run(2)  # the context's first L-BFGS call (host-driven cycles)
            # a whole untimed run first: inside this bench the first full run of the
            # 256-pair batch measured 0.5-1.0 s slower than the next ones (standalone the
            # difference is 0.13 s; the clock sampler starts beside it)
            run(2000)
            ms = []
            for _ in range(reps):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                run(2000)
                e1.record(stream)
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
            out = [dict(iters=r.iters, evals=r.evals, status=r.status, f=r.fcn) for r in res]
            cnt = ctx.counters()
            # after the timed runs: one evaluation's sweeps and the tuned launch shape
            info = {"sweep_ms": {k: round(float(v), 4) for k, v in
                                 ctx.time_sweeps(reps=1).items()},
                    "launch_shape": ctx.launch_shape()}
            info["reps_ms"] = [round(x, 2) for x in ms]
            return statistics.median(ms), out, cnt, info

    with ClockSampler(local) as clk:
        ms_all, res_all, cnt, info = batch(probs, 3)
    clocks = clk.summary()
    pairs_eval = [2 * P.T * P.nde_num ** 2 + P.dfm_elm_num * (P.dfm_elm_num + P.tgt_elm_num)
                  for P in probs]
    inter = sum(r["evals"] * w + P.tgt_elm_num ** 2
                for r, w, P in zip(res_all, pairs_eval, probs))

    # stratified sample: pairs sorted by their work here, POP_SAMPLE strata of equal
    # count, one pair drawn per stratum (seeded); the FP64 time of the whole population
    # is estimated as the sum over strata of (stratum size x the drawn pair's time)
    work = np.array([r["evals"] * w for r, w in zip(res_all, pairs_eval)], dtype=np.float64)
    order = np.argsort(work, kind="stable")
    strata = np.array_split(order, POP_SAMPLE)
    rng = np.random.default_rng(1)
    pick = [int(st[rng.integers(0, len(st))]) for st in strata]
    R = ReferenceCuda(3)
    p0 = probs[pick[0]]
    R.lbfgs(p0, np.zeros(p0.var_num), itr_max=1, tol=1e-12)  # library start-up
    ref = []
    for k in pick:
        P = probs[k]
        r = R.lbfgs(P, np.zeros(P.var_num), itr_max=max(1, res_all[k]["iters"]), tol=1e-12)
        ref.append(dict(pair=k, landmarks=P.nde_num, iters=res_all[k]["iters"],
                        evals=r["evals"], ms_lbfgs=r["ms_lbfgs"], ms_total=r["ms_total"]))
    ref_lbfgs_s = sum(r["ms_lbfgs"] for r in ref) * 1e-3
    ref_total_s = sum(r["ms_total"] for r in ref) * 1e-3
    est_lbfgs_s = sum(len(st) * r["ms_lbfgs"] for st, r in zip(strata, ref)) * 1e-3
    ms_sample, _, _, _ = batch([probs[k] for k in pick], 3)
    secs = ms_all * 1e-3
    return {
        "workload": POP_WORKLOAD, "pairs": POP_PAIRS,
        "registrations_per_s": POP_PAIRS / secs, "seconds": secs,
        "gpair_interactions_per_s": inter / secs / 1e9,
        "iters_median": float(np.median([r["iters"] for r in res_all])),
        "iters_max": int(max(r["iters"] for r in res_all)),
        "status": sorted({int(r["status"]) for r in res_all}),
        "kernel_launches": cnt["launches"], "generation_s": t_gen, "clocks": clocks,
        "cycle": info,
        "fp64_gpu_reference": {
            "path": "reference CUDA/src (FP64, cuBLAS), compiled unmodified for sm_100a",
            "sample": f"{POP_SAMPLE} pairs, one per stratum of the pairs sorted by work "
                      f"(seed 1); each run for the iterations it took here",
            "sample_seconds_lbfgs": ref_lbfgs_s, "sample_seconds_total": ref_total_s,
            "population_seconds_estimated": est_lbfgs_s,
            "pairs": ref},
        "ours_sample_seconds": ms_sample * 1e-3,
        "speedup_vs_fp64_gpu_same_sample": ref_lbfgs_s / (ms_sample * 1e-3),
        "speedup_vs_fp64_gpu_population_estimated": est_lbfgs_s / secs,
    }


# ----------------------------------------------------------------- our arm

def run_ours(args):
    import ctypes as C

    import numpy as np
    import torch

    from lddmm_b200 import _lib, api, replicas

    env = replicas.rank_env()
    world, rank, local = env.world, env.rank, env.local
    torch.cuda.set_device(local)
    dist = replicas.init(env, "nccl")

    P = workload()
    # one explicit stream shared by torch and the context, so that the CUDA events
    # below bracket the context's kernels
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = api.Context(P, stream=stream.cuda_stream, device=local)
    nvar = ctx.var_total
    d_alp = torch.zeros(nvar, dtype=torch.float64, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    opt = _lib.Opt(args.itr, 1e-6, 1e-4, 0.9, 5, 0, 0.0)
    res = (_lib.Result * 1)()

    def registration():
        d_alp.zero_()
        rc = _lib.lib.lddmm_lbfgs_device(ctx.handle, C.byref(opt), C.c_void_p(d_alp.data_ptr()),
                                         res)
        if rc < 0:
            _lib.check(rc)
        return ctx.counters()

    for _ in range(max(args.warmup, 0)):
        flush.zero_()
        registration()
    torch.cuda.synchronize()
    replicas.barrier(dist)
    torch.cuda.synchronize()
    launches = 0
    evals = 0
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t_start.record(stream)
        for _ in range(args.steps):
            flush.zero_()
            c = registration()
            launches += c["launches"]
            evals += c["evals"]
        t_end.record(stream)
        torch.cuda.synchronize()
    ms = t_start.elapsed_time(t_end)
    replicas.barrier(dist)
    ms = replicas.max_over_ranks(dist, ms, "cuda")  # the job lasts as long as its slowest rank
    clocks = clk.summary()
    r = res[0]
    x = d_alp.cpu().numpy()
    iters, status, f_final = r.iters, r.status, r.fcn

    # e2e: the reference-facing single call (MEX LDDMM3D equivalent) on HOST buffers,
    # context creation, host<->device copies and the whole registration inside.
    ini = np.ascontiguousarray(P.ini_nde)
    alp0 = np.zeros(nvar)
    out = np.zeros(nvar)
    ifo = P.elm_ifo  # rows x N, one contiguous column per vertex (getElmIfo layout)
    L = _lib.lib

    def e2e_call():
        return L.lddmm_LDDMM(3, P.nde_num, P.dfm_elm_num, P.elm_ifo.shape[1], P.tgt_elm_num,
                             _lib.dptr(ini), _lib.dptr(alp0), _lib.iptr(P.elm_vtx),
                             _lib.iptr(ifo), _lib.dptr(P.tgt_cen), _lib.dptr(P.tgt_vol),
                             _lib.dptr(P.tgt_dir), b"G", P.cen_width, b"B", P.dir_width,
                             P.dis_wgt, P.knl_order, P.knl_width, P.time_stp, P.time_num,
                             args.itr, 1e-6, 1e-4, 0.9, 5, 0, _lib.dptr(out))

    e2e_call()
    torch.cuda.synchronize()
    replicas.barrier(dist)
    e_steps = max(1, min(args.steps, 3))
    # lddmm_LDDMM is synchronous (it returns with optAlpVec in host memory): host wall
    # time around the calls is the end-to-end time
    t0 = time.perf_counter()
    for _ in range(e_steps):
        _lib.check(min(e2e_call(), 0))
    e_ms = replicas.max_over_ranks(dist, (time.perf_counter() - t0) * 1e3, "cuda")
    h2d = (ini.nbytes + alp0.nbytes + P.elm_vtx.nbytes + ifo.nbytes + P.tgt_cen.nbytes
           + P.tgt_dir.nbytes + P.tgt_vol.nbytes)
    d2h = out.nbytes

    # batched form: BATCH_PAIRS copies of the workload registered together in one
    # context (one launch per sweep for all pairs), device-resident, same options
    batched = None
    if rank == 0:
        with api.Context([P] * BATCH_PAIRS, stream=stream.cuda_stream, device=local) as cb:
            d_b = torch.zeros(cb.var_total, dtype=torch.float64, device="cuda")
            res_b = (_lib.Result * BATCH_PAIRS)()

            def batch_registration():
                d_b.zero_()
                _lib.check(min(_lib.lib.lddmm_lbfgs_device(cb.handle, C.byref(opt),
                                                           C.c_void_p(d_b.data_ptr()), res_b), 0))

            for _ in range(2):
                batch_registration()
            torch.cuda.synchronize()
            b0 = torch.cuda.Event(enable_timing=True)
            b1 = torch.cuda.Event(enable_timing=True)
            flush.zero_()
            b0.record(stream)
            batch_registration()
            b1.record(stream)
            torch.cuda.synchronize()
            b_ms = b0.elapsed_time(b1)
            batched = {"pairs": BATCH_PAIRS, "registrations_per_s": BATCH_PAIRS / (b_ms * 1e-3),
                       "ms_per_batch": b_ms,
                       "iters": [r.iters for r in res_b], "status": [r.status for r in res_b]}

    population = None
    if rank == 0 and world == 1 and not args.no_population:
        population = population_leg(stream, local, flush)

    # roofline of the dominant sweep: live per-launch timing (CUDA events on the
    # context stream) of one evaluation at the returned point
    sweeps = ctx.time_sweeps(reps=5)
    peak = C.c_double()
    _lib.check(L.lddmm_fp32_peak(local, C.byref(peak)))
    T, N, Ed, Et = P.T, P.nde_num, P.dfm_elm_num, P.tgt_elm_num
    fl = {k: L.lddmm_flops_per_pair(i, 3, P.knl_order, b"G", b"B")
          for i, k in enumerate(("shoot", "adjoint", "varifold"))}
    pairs_launch = {"shoot": N * N, "adjoint": N * N, "varifold": Ed * (Ed + Et)}
    per_eval_ms = {"shoot": T * sweeps["shoot"], "adjoint": T * sweeps["adjoint"],
                   "varifold": sweeps["varifold"]}
    dom = max(per_eval_ms, key=per_eval_ms.get)
    achieved = pairs_launch[dom] * fl[dom] / (sweeps[dom] * 1e-3) / 1e12
    pipes = _pipe_peaks(local)
    mufu = _mufu_frac(dom, P, pairs_launch[dom], sweeps[dom], pipes)
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as fh:
            traffic = json.load(fh).get(dom)
    except (OSError, ValueError):
        pass

    pairs_per_eval = 2 * T * N * N + Ed * (Ed + Et)
    evals_per_reg = evals / max(args.steps, 1)
    value = replicas.job_rate(args.steps, world, ms * 1e-3)
    gpairs = (evals * pairs_per_eval + args.steps * Et * Et) * world / (ms * 1e-3) / 1e9

    # accuracy at the returned point against the FP64 oracle (rank 0)
    rel_f = None
    cpu = None
    if rank == 0:
        from oracle.oracle import Oracle, Reference

        orc = Oracle(threads=min(os.cpu_count() or 1, 32))
        with api.Context(P) as c2:
            fg, _ = c2.objgrd(x)
        fo, _ = orc.objgrd(P, x)
        rel_f = abs(fg[0] - fo) / abs(fo)
        if world == 1 and not args.no_cpu_baseline:
            alp = np.random.default_rng(0).normal(size=P.var_num) * 0.01
            if Reference.available(3):
                R, kind = Reference(3), "reference"
            else:
                R, kind = Oracle(threads=1), "port"
            t0 = time.perf_counter()
            R.objgrd(P, alp)
            te = time.perf_counter() - t0
            cpu = {"value": 1.0 / (te * EVALS_PER_REGISTRATION), "unit": UNIT, "cores": 1,
                   "kind": kind,
                   "sample": f"one objective+gradient evaluation ({te:.2f} s, single "
                             f"thread) scaled by {EVALS_PER_REGISTRATION} evaluations "
                             f"per registration"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 kernels + f64 optimiser", "data": "synthetic",
            "config": CONFIG,
            "details": {"parallelism": f"replicas x{world}",
                       "iters": iters, "status": status, "evals_per_registration": evals_per_reg,
                       "f_final": f_final, "rel_err_f_vs_fp64_oracle": rel_f,
                       "f_fp64_registration": FP64_REGISTRATION["f"],
                       "rel_diff_vs_fp64_registration":
                           abs(f_final - FP64_REGISTRATION["f"]) / abs(FP64_REGISTRATION["f"]),
                       "gpair_interactions_per_s": gpairs,
                       "cluster": list(ctx.launch_config()),
                       "sweep_ms": {k: round(v, 5) for k, v in sweeps.items()}},
            "roofline": {"bound": "fp32", "kernel": f"{dom} sweep", "achieved": achieved,
                         "peak": peak.value, "unit": "TFLOP/s", "frac": achieved / peak.value,
                         "peak_source": "measured FP32 FMA probe (lddmm_fp32_peak), same GPU",
                         "flops_per_pair": fl[dom], "pairs_per_launch": pairs_launch[dom],
                         "traffic": traffic, "fp32x2_peak_tflops": pipes["fp32x2_tflops"],
                         "mufu": mufu},
            "cpu_baseline": cpu,
            "e2e": {"value": replicas.job_rate(e_steps, world, e_ms * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "call": "lddmm_LDDMM (host buffers; context set-up inside)"},
            "gpu_launches": launches,
            "clocks": clocks,
            "batched": batched,
            "population": population,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    replicas.barrier(dist)
    replicas.finish(dist)


def run_objgrd(args):
    """Device-resident objective + gradient evaluations of the workload at a fixed
    momentum field; prints ms per evaluation."""
    import ctypes as C

    import numpy as np
    import torch

    from lddmm_b200 import _lib, api, problem

    P = problem.sphere_to_cube(subdiv=args.subdiv)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = api.Context(P, stream=stream.cuda_stream, persistent=args.persistent)
    alp = torch.from_numpy(np.random.default_rng(0).normal(size=P.var_num) * 0.01).cuda()
    f = torch.zeros(1, dtype=torch.float64, device="cuda")
    g = torch.zeros_like(alp)

    def ev():
        _lib.check(_lib.lib.lddmm_objgrd_device(ctx.handle, C.c_void_p(alp.data_ptr()),
                                                C.c_void_p(f.data_ptr()),
                                                C.c_void_p(g.data_ptr()), 1))

    for _ in range(max(args.warmup, 1)):
        ev()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.evals):
        ev()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.evals
    print(json.dumps({"mode": "objgrd", "points": P.nde_num, "ms_per_eval": ms,
                      "f": float(f.item()), "cluster": list(ctx.launch_config())}), flush=True)
    ctx.close()


def _pipe_peaks(device):
    """Probe-measured throughput of the pipes the sweeps use (lddmm_pipe_peaks)."""
    import ctypes as C

    from lddmm_b200 import _lib

    out = (C.c_double * 3)()
    _lib.check(_lib.lib.lddmm_pipe_peaks(device, out))
    return {"fp32_tflops": out[0], "fp32x2_tflops": out[1], "ex2_gops": out[2]}


def _mufu_per_pair(sweep, P):
    """MUFU operations per pair as the sweeps execute them: a Gaussian deformation
    kernel one ex2, a 3D Matern kernel a square root and an ex2; the varifold's
    Gaussian centre kernel one ex2 (Cauchy: one reciprocal), plus one ex2 for the
    'O' / 'U' direction kernels ('B' and 'L' none)."""
    if sweep in ("shoot", "adjoint"):
        return 1 if P.knl_order == -1 else 2
    return 1 + (1 if P.dir_type in ("O", "U") else 0)


def _mufu_frac(sweep, P, pairs, ms, pipes):
    """The sweep's MUFU rate against the probe's ex2 rate: the second ceiling of an
    all-pairs sweep next to the FP32 FMA one."""
    m = _mufu_per_pair(sweep, P)
    g = pairs * m / (ms * 1e-3) / 1e9
    return {"ops_per_pair": m, "achieved_gops": g, "peak_gops": pipes["ex2_gops"],
            "frac": g / pipes["ex2_gops"]}


def run_large_pair(args):
    """One large pair: a star-shaped surface on the 7-times subdivided icosphere
    (163,842 landmarks, 327,680 triangles) onto a star-shaped target on the 6-times
    subdivided icosphere (81,920 triangles), Gaussian 0.3, varifold Gaussian 0.1 x
    Binet, T = 10.  Times ``--itr`` L-BFGS iterations from zero momenta (CUDA events
    on the context stream; tolerance 0 so every iteration runs) and the sweeps of one
    evaluation; prints one JSON line."""
    import ctypes as C

    import numpy as np
    import torch

    from lddmm_b200 import _lib, api, culling, problem

    itr = args.itr if args.itr != 500 else 100
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    P = problem.star_pair()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = api.Context(P, stream=stream.cuda_stream)
    sweeps = ctx.time_sweeps(reps=2)
    peak = C.c_double()
    _lib.check(_lib.lib.lddmm_fp32_peak(local, C.byref(peak)))
    T, N, Ed, Et = P.T, P.nde_num, P.dfm_elm_num, P.tgt_elm_num
    pairs_launch = {"shoot": N * N, "adjoint": N * N, "varifold": Ed * (Ed + Et)}
    frac = {}
    for i, k in enumerate(("shoot", "adjoint", "varifold")):
        fl = _lib.lib.lddmm_flops_per_pair(i, 3, P.knl_order, b"G", b"B")
        tf = pairs_launch[k] * fl / (sweeps[k] * 1e-3) / 1e12
        frac[k] = {"ms": sweeps[k], "flops_per_pair": fl, "tflops": tf,
                   "frac_of_measured_fp32": tf / peak.value}
    # the varifold sweep skips sub-tiles beyond its centre kernel's cut-off: its
    # roofline counts the pairs it evaluates, its effective rate all of them
    kept = culling.varifold_kept_fraction(P)  # zero momenta: the source geometry
    if kept is not None:
        v = frac["varifold"]
        v["pairs_computed_fraction"] = kept
        v["tflops_effective"] = v["tflops"]
        v["tflops"] *= kept
        v["frac_of_measured_fp32"] *= kept
    pipes = _pipe_peaks(local)
    for k in frac:
        evaluated = pairs_launch[k] * (frac[k].get("pairs_computed_fraction") or 1.0)
        frac[k]["mufu"] = _mufu_frac(k, P, evaluated, sweeps[k], pipes)
    x0 = np.zeros(ctx.var_total)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        _, res = ctx.lbfgs(x0, itr_max=itr, tol=0.0)
        e1.record(stream)
        torch.cuda.synchronize()
    s = e0.elapsed_time(e1) * 1e-3
    r = res[0]
    pairs_eval = 2 * T * N * N + Ed * (Ed + Et)
    print(json.dumps({
        "mode": "large_pair", "landmarks": N, "triangles": Ed, "target_triangles": Et,
        "time_steps": T, "iterations": r["iters"], "evaluations": r["evals"],
        "status": r["status"], "f": r["f"], "seconds": s,
        "ms_per_evaluation": s * 1e3 / max(r["evals"], 1),
        "gpair_interactions_per_s": (r["evals"] * pairs_eval + Et * Et) / s / 1e9,
        "sweeps": frac, "fp32_peak_tflops": peak.value, "pipe_peaks": pipes,
        "clocks": clk.summary()}),
        flush=True)
    ctx.close()


def _bf16_peak():
    """Dense bf16 TFLOP/s: the pool's measured figure when the file is present, else
    the earlier measurement on this pool (burst)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["bf16_tflops"]), "measured (MEASURED_PEAKS.json, burst)"
    except (OSError, ValueError, KeyError, TypeError):
        return 1590.0, "fallback 1.59 PFLOP/s (earlier measurement on this pool)"


def run_ws_gemm(args):
    """C[m x n] = A[m x k] B[n x k]^T in BF16 with FP32 output through
    lddmm_ws_gemm_bf16 (tcgen05.mma, TMEM accumulator), on the warm-start network's
    layer shapes at a 64-pair batch (2562 points or 5120 triangles per pair), CUDA
    events around each launch with a 256 MiB L2 flush before it; torch's bf16 matmul
    (cuBLAS) on the same shapes for context, with FP32 output (torch.mm out_dtype, the
    same bytes written as ours) and with its default BF16 output (half the output
    bytes).  Prints one JSON line."""
    import ctypes as C

    import torch

    from lddmm_b200 import _lib

    torch.cuda.set_device(0)
    peak, peak_src = _bf16_peak()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    shapes = [(64 * 2562, 256, 256), (64 * 2562, 256, 80), (64 * 2562, 32, 256),
              (64 * 5120, 64, 64), (64 * 2562, 256, 2048)]
    out = []
    for m, n, k in shapes:
        a = torch.randn(m, k, device="cuda").to(torch.bfloat16)
        b = torch.randn(n, k, device="cuda").to(torch.bfloat16)
        c = torch.empty(m, n, device="cuda", dtype=torch.float32)

        def ours():
            _lib.check(_lib.lib.lddmm_ws_gemm_bf16(
                C.c_void_p(a.data_ptr()), k, C.c_void_p(b.data_ptr()), k, m, n, k,
                C.c_void_p(c.data_ptr()), n, C.c_void_p(stream.cuda_stream)))

        def ref():
            torch.matmul(a, b.t())

        def ref32():
            torch.mm(a, b.t(), out_dtype=torch.float32)

        fns = [("ours", ours), ("torch", ref)]
        try:
            ref32()
            fns.append(("torch32", ref32))
        except (RuntimeError, TypeError):
            pass  # no FP32-output bf16 GEMM in this torch build
        res = {}
        for name, fn in fns:
            for _ in range(max(args.warmup, 3)):
                fn()
            ts = []
            for _ in range(max(args.steps, 5)):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            ms = statistics.median(ts)
            res[name] = {"ms": ms, "tflops": 2.0 * m * n * k / (ms * 1e-3) / 1e12}
        err = float((c - torch.matmul(a.float(), b.float().t())).abs().max()
                    / torch.matmul(a.float(), b.float().t()).abs().max())
        out.append({"m": m, "n": n, "k": k, "ours": res["ours"], "torch_bf16": res["torch"],
                    "torch_bf16_fp32_out": res.get("torch32"),
                    "hbm_gbs": (m * k * 2 + n * k * 2 + m * n * 4) / (res["ours"]["ms"] * 1e-3)
                    / 1e9,
                    "frac_of_peak": res["ours"]["tflops"] / peak, "rel_err_vs_fp32": err})
    print(json.dumps({"mode": "ws_gemm", "peak_tflops": peak, "peak_source": peak_src,
                      "shapes": out}), flush=True)


def main():
    args = parse()
    if args.mode == "ws_gemm":
        run_ws_gemm(args)
        return
    if args.mode == "objgrd":
        run_objgrd(args)
        return
    if args.mode == "large_pair":
        run_large_pair(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
