"""Benchmark of the CTMRG hot path on B200.

Workload (default): spin-1/2 Heisenberg (sublattice-rotated), single-site
iPEPS A of shape (5,5,5,5,2), i.i.d. N(0,1) seeded, max|A| = 1, chi = 100
(enlarged-corner matrices 2500 x 2500).  One step = one energy+gradient
evaluation (fg! of optim_gs): init_ctm1, 30 CTMRG iterations (4 directional
moves each) with the energy every iteration (the reference's conv_fun), then
the pullback of ad_max_iter = 4 further iterations + the energy.

By default both forms run on the same input: the mixed form (3xTF32
contractions on the tensor cores, FP64 projector / normalisation / final
energy) gives ``value``; the plain FP64 form is timed beside it
(``fp64``), with the ratio and the mixed form's energy and gradient errors
against the FP64 form and the 30-iteration energy against the oracle's
(tests/golden/d5_chi100_30.json).  CTMRG moves/s is measured on the forward
part alone and reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision both|fp64|mixed]
                    [--workload d5chi100|d4chi64]
    python bench.py --impl reference ...   # CPU arm (see below)
    python bench.py --forward-only 6       # profiling aid: 6 forward iterations, no timing
    python bench.py --gemm-shapes          # FP64 DMMA GEMM vs cuBLAS on the engine's shapes
    python bench.py --tf32-shapes          # 3xTF32 tcgen05 GEMM on the engine's shapes

Timing: K steps timed with CUDA events recorded on the engine's own stream,
L2 flushed (512 MB write) between steps, max over ranks; value = E+grad
evaluations/s of the whole job.  e2e = the same metric through the public API
(fg) with host buffers: A and H copied in, energy and gradient copied out,
inside the timed region.  Under torchrun each rank runs an independent
replica: a CTMRG run of one iPEPS is a sequential chain of dependent moves
with no data-parallel split, so N GPUs run N independent evaluations.

Reference arm: the reference is Julia, which is not installed, so
``--impl reference`` times the CPU FP64 oracle (a restatement of the
reference's algorithm) on the host cores.  Each of its steps is one forward
CTMRG iteration (with the energy) of the same workload, timed as it runs;
one pullback iteration is timed after them, and the evaluations/s value is
derived from those two times (30 forward + 4 pullback iterations per
evaluation), as the line's ``value_derivation`` states.  It is the CPU
baseline, not a target.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "ipeps.jl_b200")


def load_pkg():
    if "ipeps_b200" in sys.modules:
        return sys.modules["ipeps_b200"]
    spec = importlib.util.spec_from_file_location("ipeps_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ipeps_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


# ---------------------------------------------------------------- inputs
def random_A(D, d, seed):
    """N(0,1) from numpy default_rng, column-major (Julia) order, max|A| = 1."""
    rng = np.random.default_rng(seed)
    A = rng.standard_normal(D ** 4 * d).reshape((D, D, D, D, d), order="F")
    return np.asfortranarray(A / np.abs(A).max())


def tout(a, b):
    """basis.jl:16-21: reshape(tcon([a,b], [[-1,-3],[-2,-4]]), d1*d2, d3*d4) (column-major)."""
    c = np.einsum("ac,bd->abcd", a, b)
    s = c.shape
    return c.reshape((s[0] * s[1], s[2] * s[3]), order="F")


def heisenberg(Jz=1.0):
    """basis.jl:31-35"""
    Sx = np.array([[0, 1], [1, 0]]) / 2
    Sy = np.array([[0, -1j], [1j, 0]]) / 2
    Sz = np.array([[1, 0], [0, -1]]) / 2
    H = Jz * tout(Sz, Sz) - tout(Sx, Sx) - tout(Sy, Sy)
    H = np.asfortranarray(H.astype(np.complex128))
    return [H, H]


WORKLOADS = {
    # the headline configuration: Heisenberg D=5 chi=100 (enlarged corners 2500 x 2500), 30 CTMRG iterations
    "d5chi100": dict(model="heisenberg", D=5, d=2, chi=100, iters=30, ad_iters=4,
                     golden="d5_chi100_30.json"),
    # the smaller configuration (enlarged corners 1024 x 1024)
    "d4chi64": dict(model="heisenberg", D=4, d=2, chi=64, iters=30, ad_iters=4, golden="config2.json"),
}
WORKLOAD = WORKLOADS["d5chi100"]


def workload_name(w):
    return ("heisenberg D=%d d=%d chi=%d: E+grad evaluation = init_ctm1 + %d CTMRG iterations with the energy "
            "per iteration + pullback of %d iterations and the energy" % (w["D"], w["d"], w["chi"], w["iters"],
                                                                          w["ad_iters"]))


WORKLOAD_NAME = workload_name(WORKLOAD)


def workload_cfg(pkg, chi, iters, ad_iters):
    cfg = pkg.default_config()
    cfg.update(chi=chi, min_iter=iters, max_iter=iters, rg_tol=0.0, ad_max_iter=ad_iters)
    return cfg


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + ",".join(self.FIELDS),
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == len(self.FIELDS):
                self.samples.append(parts)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        if not self.samples:
            return None
        mhz = []
        maxmhz = 0.0
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                mhz.append(float(s[1]))
                maxmhz = max(maxmhz, float(s[2]))
            except ValueError:
                continue
            for n, v in zip(names, s[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": maxmhz or None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------- helpers
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def measure_fp64_peak(torch):
    """cuBLAS DGEMM (torch.matmul float64, 8192^3) on this GPU: the FP64 roofline denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def _oracle(threads):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch
    import ipeps_oracle as O
    if threads:
        torch.set_num_threads(threads)
    return torch, O


def _oracle_workload(O, torch, seed):
    D, d, chi = WORKLOAD["D"], WORKLOAD["d"], WORKLOAD["chi"]
    A = torch.tensor(random_A(D, d, seed))
    H = O.heisenberg(1.0)
    cfg = O.default_config()
    cfg.update(chi=chi, min_iter=1, max_iter=1, rg_tol=0.0, ad_max_iter=1)
    return A, H, cfg


def _oracle_pullback_iter(O, torch, ts, A, H):
    """One pullback iteration of run_gs (ad_max_iter = 1) + the energy, timed."""
    ts1 = O._detach_ts(ts)
    xv = A.clone().requires_grad_(True)
    t0 = time.perf_counter()
    y = O.run_gs(ts1, H, xv)
    torch.autograd.grad(y.real, xv)
    return time.perf_counter() - t0


def cpu_oracle_eg_sample(seed, budget_s=12.0, threads=None):
    """CPU oracle on a bounded sample of the workload.  Times (a) forward CTMRG
    iterations with the energy (~budget_s) and (b) the pullback of one CTMRG
    iteration + the energy (torch autograd with the reference's svd_back), and
    scales to one E+grad evaluation = iters forward + ad_iters pullback
    iterations.  Returns (evals/s, moves/s, sample description, threads)."""
    torch, O = _oracle(threads)
    A, H, cfg = _oracle_workload(O, torch, seed)
    ts = O.make_ctm_tensors(A, cfg)
    chi = WORKLOAD["chi"]
    with torch.no_grad():
        for _ in range(2):  # first iterations have small chi
            ts, _ = O.rg_step(ts, chi)
        t0 = time.perf_counter()
        it = 0
        while True:
            ts, _ = O.rg_step(ts, chi)
            O.get_gs_energy(ts, H)
            it += 1
            if time.perf_counter() - t0 > budget_s:
                break
    t_iter = (time.perf_counter() - t0) / it
    t_ad = _oracle_pullback_iter(O, torch, ts, A, H)
    t_eval = WORKLOAD["iters"] * t_iter + WORKLOAD["ad_iters"] * t_ad
    sample = (f"CPU oracle (torch float64, {torch.get_num_threads()} threads): {it} forward iterations "
              f"({t_iter:.2f} s each) and one pullback iteration ({t_ad:.1f} s) timed; one E+grad evaluation = "
              f"{WORKLOAD['iters']} x forward + {WORKLOAD['ad_iters']} x pullback = {t_eval:.1f} s")
    return 1.0 / t_eval, 4.0 / t_iter, sample, torch.get_num_threads(), t_eval


# ---------------------------------------------------------------- arms
def run_reference(args):
    """CPU arm: the oracle restatement of the reference on the host cores.

    Warm-up steps are forward iterations from init_ctm1 (the environment grows
    to chi); each timed step is one forward CTMRG iteration + energy of the
    same workload, and ms_per_step is their measured mean.  One pullback
    iteration is timed after the steps.  The evaluations/s value is derived
    from the two measured times (value_derivation)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    D, d, chi = WORKLOAD["D"], WORKLOAD["d"], WORKLOAD["chi"]
    threads = os.cpu_count() or 1
    t_start = time.perf_counter()
    torch, O = _oracle(threads)
    A, H, cfg = _oracle_workload(O, torch, seed=1000)
    ts = O.make_ctm_tensors(A, cfg)
    step_s = []
    with torch.no_grad():
        for i in range(max(args.warmup, 2) + args.steps):
            t0 = time.perf_counter()
            ts, _ = O.rg_step(ts, chi)
            O.get_gs_energy(ts, H)
            if i >= max(args.warmup, 2):
                step_s.append(time.perf_counter() - t0)
    t_iter = statistics.mean(step_s)
    t_ad = _oracle_pullback_iter(O, torch, ts, A, H)
    t_eval = WORKLOAD["iters"] * t_iter + WORKLOAD["ad_iters"] * t_ad
    value = 1.0 / t_eval
    sample = (f"CPU oracle (torch float64, {torch.get_num_threads()} threads): {len(step_s)} forward iterations "
              f"timed as the steps ({t_iter:.2f} s each) and one pullback iteration ({t_ad:.1f} s)")
    line = {"impl": "reference", "metric": metric_name(), "value": value,
            "unit": "evals/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_iter, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME, "D": D, "chi": chi,
                       "step": "one forward CTMRG iteration + energy of the workload (bounded CPU sample)"},
            "value_derivation": {"formula": "1 / (%d x forward iteration + %d x pullback iteration)"
                                 % (WORKLOAD["iters"], WORKLOAD["ad_iters"]),
                                 "forward_iteration_s": t_iter, "pullback_iteration_s": t_ad,
                                 "one_evaluation_s": t_eval, "extrapolated": True},
            "moves_per_s": 4.0 / t_iter,
            "cpu_baseline": {"value": value, "unit": "evals/s", "cores": torch.get_num_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": time.perf_counter() - t_start,
            "reference_note": "iPEPS.jl is Julia; no Julia toolchain on this machine, so the CPU arm is the "
                              "oracle restatement of its algorithm"}
    print(json.dumps(line))
    return 0


def metric_name():
    return ("E+grad evals/s, mixed form (3xTF32 contractions) with the plain FP64 form beside it "
            "(Heisenberg D=%d chi=%d); CTMRG moves/s in moves_per_s" % (WORKLOAD["D"], WORKLOAD["chi"]))


def golden_energies():
    p = os.path.join(ROOT, "tests", "golden", WORKLOAD["golden"])
    if not os.path.exists(p):
        return None
    with open(p) as f:
        g = json.load(f)
    return g.get("energies")


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    pkg = load_pkg()
    forms = ["mixed", "fp64"] if args.precision == "both" else [args.precision]
    D, d, chi, iters, ad_iters = (WORKLOAD[k] for k in ("D", "d", "chi", "iters", "ad_iters"))
    cfg = workload_cfg(pkg, chi, iters, ad_iters)
    H = heisenberg(1.0)
    A = random_A(D, d, seed=1000 + rank)
    moves_per_fwd = 4 * iters
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    class Form:
        """one precision form: its engine (own CUDA stream) and environment"""

        def __init__(self, name):
            self.name = name
            self.eng = pkg.Engine(local, precision=name)
            self.ext = torch.cuda.ExternalStream(self.eng.stream_ptr())
            self.ts = pkg.CTMTensors(A, cfg, engine=self.eng)
            self.last = None

        def forward(self):
            # inputs resident: A already on the device; re-initialise and iterate
            self.eng.check(self.eng.lib.ipeps_env_init(self.ts.h))
            _, info = pkg.run_ctm(self.ts, conv_fun="energy", H=H)
            return info

        def step(self):
            info = self.forward()
            E, g = pkg.energy_grad(self.ts, H, ad_iters)
            self.last = (info["log"][-1]["obj"].real, E, g)

        def e2e(self):
            pkg.fg(A, H, cfg, engine=self.eng)

        def timed(self, fn, k):
            times = []
            for _ in range(k):
                flush.zero_()
                torch.cuda.synchronize()
                s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s.record(self.ext)
                fn()
                e.record(self.ext)
                e.synchronize()
                times.append(s.elapsed_time(e) / 1e3)
            return times

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(t):
        if world > 1:
            tt = torch.tensor([t], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            return float(tt.item())
        return t

    if args.forward_only > 0:
        cfg.update(min_iter=args.forward_only, max_iter=args.forward_only)
        f = Form(forms[0])
        info = f.forward()
        if rank == 0:
            print(json.dumps({"forward_only": args.forward_only, "workload": WORKLOAD_NAME, "precision": forms[0],
                              "energy": info["log"][-1]["obj"].real}))
        f.ts.close()
        return 0

    fm = {n: Form(n) for n in forms}
    main = fm[forms[0]]

    # ---- timed region of the headline form: K E+grad evaluations, events on the engine stream,
    # L2 flushed between steps, clocks sampled meanwhile
    for _ in range(args.warmup):
        main.step()
    barrier()
    main.eng.reset_stats()
    sampler = ClockSampler(local)
    sampler.start()
    times = main.timed(main.step, args.steps)
    barrier()
    clocks = sampler.stop()
    st = main.eng.stats()
    launches = sum(f["launches"] for f in st["families"].values())
    t_max = max_over_ranks(sum(times))
    value = args.steps * world / t_max

    # ---- side measurements on min(K, 5) steps: the other form, forward-only moves/s, e2e
    ks = max(1, min(args.steps, 5))
    side = {}
    for n in forms[1:]:
        f = fm[n]
        for _ in range(min(args.warmup, 3)):
            f.step()
        barrier()
        side[n] = ks * world / max_over_ranks(sum(f.timed(f.step, ks)))
    moves = {}
    for n in forms:
        f = fm[n]
        moves[n] = moves_per_fwd * ks * world / max_over_ranks(sum(f.timed(f.forward, ks)))

    # e2e: public API with host buffers (A, H in; energy, gradient out) each step
    te = max_over_ranks(sum(main.timed(main.e2e, ks)))
    e2e_value = ks * world / te
    h2d = A.nbytes + 2 * H[0].nbytes * 2   # A, and H for the run and for the gradient call
    d2h = A.nbytes + 8 + 32 * iters        # gradient, energy, per-iteration log
    barrier()

    # ---- live per-kernel-family profile of one E+grad step of each form (events around each launch)
    prof = {}
    for n in forms:
        f = fm[n]
        f.eng.prof_enable(True)
        f.step()
        prof[n] = f.eng.prof_query()
        f.eng.prof_enable(False)

    if rank == 0:
        peaks, peak_kind = measured_peaks()
        fp64_peak = measure_fp64_peak(torch)

        def gemm_roofline(pr, gname, total_ms):
            g = pr[gname]
            achieved = g["flops"] / (g["ms"] / 1e3) / 1e12 if g["ms"] > 0 else 0.0
            if gname == "gemm_f64":
                peak, note = fp64_peak, ("cuBLAS DGEMM 8192^3 measured in this run "
                                         "(FP64 has no entry in MEASURED_PEAKS.json)")
                kern = "gemm_f64 (DMMA m8n8k4 FP64 tensor cores)"
            else:
                key = "bf16_tflops_sustained" if "bf16_tflops_sustained" in peaks else "bf16_tflops"
                peak = peaks[key] / 2 / 3
                note = f"{peak_kind} {key} / 2 (TF32) / 3 (three split products per credited flop)"
                kern = "gemm_tf32x3 (tcgen05.mma kind::tf32, TMEM accumulators)"
            return {"bound": "tensor", "kernel": kern, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak if peak else None, "traffic": None, "peak_source": note,
                    "kernel_share_of_device_time": g["ms"] / total_ms if total_ms else None,
                    "launches_in_profiled_step": g["launches"]}

        def roofline(n):
            """the dominant GEMM family of the profiled step (by event-timed device
            time), with the 3xTF32 kernel beside it in the mixed form"""
            pr = prof[n]
            total_ms = sum(v["ms"] for v in pr.values())
            gemms = [k for k in ("gemm_f64", "gemm_tf32x3") if pr[k]["ms"] > 0]
            gname = max(gemms, key=lambda k: pr[k]["ms"])
            out = gemm_roofline(pr, gname, total_ms)
            dom = max(pr.items(), key=lambda kv: kv[1]["ms"])
            out["dominant_family"] = dom[0]
            out["families_ms"] = {k: round(v["ms"], 3) for k, v in pr.items()}
            if n == "mixed" and gname != "gemm_tf32x3" and pr["gemm_tf32x3"]["ms"] > 0:
                out["tf32x3"] = gemm_roofline(pr, "gemm_tf32x3", total_ms)
            pm = pr["permute"]
            if pm["ms"] > 0:
                # the HBM-bound family: the tcon planner's permutes (one read and one
                # write of every element) and the 3xTF32 operand splits (FP64 in,
                # hi/lo TF32 planes out), over their event-timed device time (the
                # events bracket each launch, so short launches read a little low)
                gbs = pm["bytes"] / (pm["ms"] / 1e3) / 1e9
                out["permute"] = {"bound": "hbm", "kernel": "permute_rows / permute_tiled / split_kc / split_tr",
                                  "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                                  "frac": gbs / peaks["hbm_gbs"], "traffic": None,
                                  "peak_source": f"{peak_kind} hbm_gbs",
                                  "bytes_per_launch": pm["bytes"] / max(1, pm["launches"]),
                                  "kernel_share_of_device_time": pm["ms"] / total_ms if total_ms else None,
                                  "launches_in_profiled_step": pm["launches"]}
            return out

        acc = {}
        gold = golden_energies()
        for n in forms:
            e30, E, g = fm[n].last
            acc[n] = {"E": E, "E_iter%d" % iters: e30,
                      "dE_vs_oracle_iter%d" % iters: (abs(e30 - gold[iters - 1]) if gold else None)}
        if "fp64" in fm and "mixed" in fm:
            _, E64, g64 = fm["fp64"].last
            _, Em, gm = fm["mixed"].last
            acc["mixed_vs_fp64"] = {"dE": abs(Em - E64),
                                    "grad_rel": float(np.linalg.norm(gm - g64) / np.linalg.norm(g64))}
        cpu = None
        if not args.no_cpu_baseline:
            v, mv, sample, nth, _ = cpu_oracle_eg_sample(seed=1000, budget_s=args.cpu_budget,
                                                         threads=os.cpu_count())
            cpu = {"value": v, "unit": "evals/s", "cores": nth, "kind": "port", "sample": sample, "moves_per_s": mv}
        out = {
            "metric": metric_name(),
            "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if forms[0] == "fp64" else "f64 (3xTF32 contractions)",
            "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME, "precision": forms[0],
                       "l2": "flushed between steps (512 MB write)", "replicas": world},
            "moves_per_s": moves[forms[0]],
            "e2e": {"value": e2e_value, "unit": "evals/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches),
            "roofline": roofline(forms[0]),
            "projector": {"calls": st["projector_calls"], "jacobi_sweeps_per_call":
                          st["jacobi_sweeps"] / max(1, st["projector_calls"]),
                          "extra_passes": st["extra_passes"], "series_cap_hits": st["series_cap_hits"],
                          "adjoint_series_terms": st["series_terms"], "adjoint_series_retries": st["series_retries"]},
            "accuracy": acc,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        for n in forms[1:]:
            out[n] = {"evals_per_s": side[n], "moves_per_s": moves[n], "steps": ks, "roofline": roofline(n)}
        if "fp64" in side:
            out["mixed_over_fp64"] = value / side["fp64"] if forms[0] == "mixed" else None
        print(json.dumps(out))
    for f in fm.values():
        f.ts.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_gemm_shapes():
    """ipeps_gemm_f64 (10 products from one input upload; device time of the
    GEMM family by the engine's CUDA-event profile, split-K sums included)
    against torch.matmul (cuBLAS DGEMM, CUDA events)."""
    import numpy as np
    import torch
    pkg = load_pkg()
    eng = pkg.Engine(0)
    shapes = [("N", "N", 2500, 160, 2500), ("T", "N", 2500, 160, 2500), ("T", "N", 160, 160, 2500),
              ("N", "N", 2500, 200, 2500), ("T", "N", 2500, 200, 2500),
              ("N", "N", 2500, 2500, 100), ("N", "N", 250000, 50, 25), ("N", "T", 4096, 4096, 4096),
              ("N", "N", 4096, 4096, 4096)]
    rng = np.random.default_rng(0)
    for oa, ob, m, n, k in shapes:
        A = rng.standard_normal((m, k) if oa == "N" else (k, m))
        B = rng.standard_normal((k, n) if ob == "N" else (n, k))
        pkg.host.gemm_f64(oa, ob, A, B, engine=eng, reps=2)  # warm-up
        eng.prof_enable(True)
        pkg.host.gemm_f64(oa, ob, A, B, engine=eng, reps=10)
        pr = eng.prof_query()
        eng.prof_enable(False)
        dt = (pr["gemm_f64"]["ms"] + pr["reduce"]["ms"]) / 10 / 1e3
        a, b = torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda")
        fa = (lambda x: x) if oa == "N" else (lambda x: x.T)
        fb = (lambda x: x) if ob == "N" else (lambda x: x.T)
        for _ in range(3):
            fa(a) @ fb(b)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(10):
            fa(a) @ fb(b)
        e1.record()
        torch.cuda.synchronize()
        dc = e0.elapsed_time(e1) / 10 / 1e3
        fl = 2.0 * m * n * k
        print(json.dumps({"op": oa + ob, "m": m, "n": n, "k": k, "dmma_us": round(dt * 1e6, 1),
                          "dmma_tflops": round(fl / dt / 1e12, 2), "cublas_us": round(dc * 1e6, 1),
                          "cublas_tflops": round(fl / dc / 1e12, 2)}), flush=True)
    return 0


def run_pullback_profile(args):
    """The E+grad pullback alone (energy_grad: ad_iters checkpointed iterations
    from a converged environment, the energy on a tape, the backward with the
    projector adjoints) of the workload, in one precision form.  Each pullback
    follows the forward iterations on the same environment, as in an E+grad
    step; one warm-up, then one pullback bracketed by cudaProfilerStart /
    cudaProfilerStop (ncu --profile-from-start off captures only it), timed by
    CUDA events, with the per-family device profile of a third one and the
    projector/adjoint counters.  Also times the checkpoint iterations alone
    (ad_iters CTMRG steps at the pullback's residual tolerance, from a copy of
    the converged environment without sketch seeds)."""
    import torch
    pkg = load_pkg()
    form = "fp64" if args.precision == "both" else args.precision
    D, d, chi, iters, ad_iters = (WORKLOAD[k] for k in ("D", "d", "chi", "iters", "ad_iters"))
    cfg = workload_cfg(pkg, chi, iters, ad_iters)
    H = heisenberg(1.0)
    A = random_A(D, d, seed=1000)
    eng = pkg.Engine(0, precision=form)
    ext = torch.cuda.ExternalStream(eng.stream_ptr())
    ts = pkg.CTMTensors(A, cfg, engine=eng)
    pkg.run_ctm(ts, conv_fun="energy", H=H)
    C = [ts.get_CT(k) for k in range(1, 5)]
    ts.close()

    def fresh():
        t = pkg.CTMTensors(A, cfg, engine=eng, init=False)
        for k in range(4):
            t.set_CT(k + 1, *C[k])
        return t

    def timed(fn):
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(ext)
        fn()
        e.record(ext)
        e.synchronize()
        return s.elapsed_time(e)

    # as in an E+grad step, the pullback follows the forward iterations on the
    # same environment (its projectors' sketches are seeded from them)
    t = pkg.CTMTensors(A, cfg, engine=eng)
    pkg.run_ctm(t, conv_fun="energy", H=H)
    pkg.energy_grad(t, H, ad_iters)
    eng.check(eng.lib.ipeps_env_init(t.h))
    pkg.run_ctm(t, conv_fun="energy", H=H)
    eng.reset_stats()
    torch.cuda.profiler.start()
    ms = timed(lambda: pkg.energy_grad(t, H, ad_iters))
    torch.cuda.profiler.stop()
    st = eng.stats()
    eng.check(eng.lib.ipeps_env_init(t.h))
    pkg.run_ctm(t, conv_fun="energy", H=H)
    eng.prof_enable(True)
    eng.prof_phases()
    pkg.energy_grad(t, H, ad_iters)
    prof = eng.prof_query()
    phases = eng.prof_phases()
    eng.prof_enable(False)
    t.close()
    t = fresh()
    t.Params["svd_resid_tol"] = 1e-12
    t._push_params()
    ms_ck = timed(lambda: [pkg.rg_step(t) for _ in range(ad_iters)])
    t.close()
    print(json.dumps({"pullback": WORKLOAD_NAME, "precision": form, "pullback_ms": round(ms, 2),
                      "checkpoint_iterations_ms": round(ms_ck, 2),
                      "launches": int(sum(f["launches"] for f in st["families"].values())),
                      "projector": {k: st[k] for k in ("projector_calls", "extra_passes", "resid_misses",
                                                       "series_terms", "series_retries", "series_cap_hits")},
                      "families_ms_serialised": {k: round(v["ms"], 3) for k, v in prof.items() if v["ms"] > 0},
                      "phases_ms_profiled": {k: round(v, 2) for k, v in phases.items()}}),
          flush=True)
    eng.close()
    return 0


def run_optim_gs(args):
    """The full optim_gs of the D=5 chi=100 workload (L-BFGS over A on the unit
    sphere, optim_gs.jl:14-118) for args.optim_gs steps in each form, from the
    same seeded A: every step's fg! runs CTMRG from init_ctm1 with the energy
    criterion (rg_tol 1e-8, at most 30 iterations) and the pullback of 4
    iterations.  Reports E+grad evals/s per form, the energies after each step
    and the difference of the final energies."""
    import torch
    pkg = load_pkg()
    D, d, chi = (WORKLOAD[k] for k in ("D", "d", "chi"))
    H = heisenberg(1.0)
    A0 = random_A(D, d, seed=1000)
    cfg = pkg.default_config()
    cfg.update(chi=chi, min_iter=4, max_iter=30, rg_tol=1e-8, ad_max_iter=4)
    out = {"optim_gs": WORKLOAD_NAME.split(":")[0], "lbfgs_steps": args.optim_gs,
           "fg": "CTMRG from init_ctm1, energy criterion rg_tol 1e-8, min 4 / max 30 iterations, pullback of 4"}
    for form in ("fp64", "mixed"):
        eng = pkg.Engine(0, precision=form)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = pkg.drivers.optim_gs(H, A0, dict(cfg), iterations=args.optim_gs, engine=eng)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        out[form] = {"seconds": round(dt, 2), "evals": r["evals"], "evals_per_s": r["evals"] / dt,
                     "steps_done": len(r["energies"]), "E_final": r["energies"][-1],
                     "energies": [float(e) for e in r["energies"]]}
        eng.close()
    out["dE_final_mixed_vs_fp64"] = abs(out["mixed"]["E_final"] - out["fp64"]["E_final"])
    out["mixed_over_fp64_evals_per_s"] = out["mixed"]["evals_per_s"] / out["fp64"]["evals_per_s"]
    print(json.dumps(out), flush=True)
    return 0


def run_es_momentum(args):
    """One momentum of the excited-state workload (Heisenberg D=3 d=2 chi=48):
    a ground state from args.es_gs_steps L-BFGS steps of optim_gs from a seeded
    A, prepare_basis (reconverged environment, normalised state, E0/2
    subtracted, the 161 tangent vectors), then optim_es at (px, py) = (pi, 0)
    over the whole basis and evaluate_es.  Reports the seconds per momentum
    (momenta/s) and the lowest four band energies."""
    import torch
    pkg = load_pkg()
    eng = pkg.Engine(0)
    H = heisenberg(1.0)
    A0 = random_A(3, 2, seed=21)
    cfg = pkg.default_config()
    cfg.update(chi=48, min_iter=4, max_iter=40, rg_tol=1e-8, ad_max_iter=4)
    r = pkg.drivers.optim_gs(H, A0, dict(cfg), iterations=args.es_gs_steps, engine=eng)
    ts, H2, basis = pkg.drivers.prepare_basis(H, r["A"], dict(cfg), engine=eng)
    workers = [pkg.Engine(0) for _ in range(max(args.es_workers, 1) - 1)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    effH, effN = pkg.drivers.optim_es(1.0, 0.0, ts, H2, basis, engines=([eng] + workers) if workers else None)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    for w in workers:
        w.close()
    es = pkg.drivers.band_energies(effH, effN, 1e-3)
    print(json.dumps({"es_momentum": "heisenberg D=3 d=2 chi=48, (px, py) = (pi, 0)", "basis_vectors": int(basis.shape[1]),
                      "gs_lbfgs_steps": args.es_gs_steps, "E_gs": r["energies"][-1],
                      "contexts": max(args.es_workers, 1),
                      "seconds_per_momentum": round(dt, 2), "momenta_per_s": 1.0 / dt,
                      "get_es_grad_per_s": basis.shape[1] / dt,
                      "lowest_bands": [float(x) for x in es[:4]]}), flush=True)
    ts.close()
    eng.close()
    return 0


def run_tf32_shapes():
    """ipeps_gemm_tf32x3 (3xTF32 on tcgen05: operand splits + GEMM, device time
    by CUDA events, mean over 10 repetitions) on the engine's shapes; credited
    flops are 2MNK of the FP64-equivalent product, against the TF32 tensor
    peak / 3 (three split products per credited flop)."""
    pkg = load_pkg()
    eng = pkg.Engine(0)
    peaks, kind = measured_peaks()
    key = "bf16_tflops"
    peak = peaks[key] / 2 / 3
    shapes = [("N", "N", 2500, 160, 2500), ("T", "N", 2500, 160, 2500), ("T", "N", 160, 160, 2500),
              ("N", "N", 2500, 2500, 100), ("N", "N", 250000, 50, 25), ("N", "T", 4096, 4096, 4096),
              ("N", "N", 8192, 8192, 8192)]
    rng = np.random.default_rng(0)
    for oa, ob, m, n, k in shapes:
        A = rng.standard_normal((m, k) if oa == "N" else (k, m))
        B = rng.standard_normal((k, n) if ob == "N" else (n, k))
        _, ms = pkg.host.gemm_tf32x3(oa, ob, A, B, engine=eng, reps=11, timing=True)
        fl = 2.0 * m * n * k
        print(json.dumps({"op": oa + ob, "m": m, "n": n, "k": k, "us": round(ms * 1e3, 1),
                          "tflops": round(fl / (ms / 1e3) / 1e12, 2),
                          "frac_of_peak": round(fl / (ms / 1e3) / 1e12 / peak, 3),
                          "peak": round(peak, 1), "peak_source": f"{kind} {key} / 2 / 3"}), flush=True)
    return 0


def run_projector_shapes():
    """The truncated-SVD projector alone (ipeps_projector, host buffers; device
    time from the engine's per-family profile) on synthetic enlarged corners of
    the workload's size: R1, R2 of N x N, N = chi D^2, with a decaying spectrum;
    the kernel-level aid behind the projector's ncu captures."""
    pkg = load_pkg()
    D, chi = WORKLOAD["D"], WORKLOAD["chi"]
    N = chi * D * D
    rng = np.random.default_rng(0)
    s = np.exp(-0.02 * np.arange(N))
    U, _ = np.linalg.qr(rng.standard_normal((N, N)))
    R1 = (U * np.sqrt(s)) @ rng.standard_normal((N, N)) / np.sqrt(N)
    R2 = np.linalg.solve(rng.standard_normal((N, N)) / np.sqrt(N), (np.sqrt(s)[:, None] * U.T))
    for prec in ("fp64", "mixed"):
        eng = pkg.Engine(0, precision=prec)
        pkg.get_projector(R1, R2, chi, engine=eng)  # warm-up (kernel loads, pool)
        eng.prof_enable(True)
        reps = 3
        t0 = time.perf_counter()
        for _ in range(reps):
            P1, P2, S = pkg.get_projector(R1, R2, chi, engine=eng)
        wall = (time.perf_counter() - t0) / reps
        prof = eng.prof_query()
        eng.prof_enable(False)
        st = eng.stats()
        print(json.dumps({"projector": f"N={N} chi={chi}", "precision": prec, "wall_ms_per_call": round(1e3 * wall, 2),
                          "device_ms_per_call": {k: round(v["ms"] / reps, 3) for k, v in prof.items() if v["ms"] > 0},
                          "launches_per_call": {k: v["launches"] // reps for k, v in prof.items() if v["launches"]},
                          "jacobi_sweeps": st["jacobi_sweeps"], "extra_passes": st["extra_passes"],
                          "s_head": [float(x) for x in S[:3]]}), flush=True)
        eng.close()
    return 0


def run_orth_shapes():
    """The projector's CholeskyQR alone (ipeps_orth, three passes, host buffers)
    on Gaussian 2500 x k sketches, k = 160, 128, 101: device time per pass of
    the Cholesky and the triangular solve (the engine's small_linalg family;
    the Gram product is the gemm_f64 family), the aid behind the Cholesky's
    ncu summary."""
    pkg = load_pkg()
    eng = pkg.Engine(0, precision="fp64")
    rng = np.random.default_rng(1)
    for k in (160, 128, 101):
        Y = rng.standard_normal((2500, k))
        pkg.orth(Y, 3, engine=eng)  # warm-up (kernel loads, pool)
        eng.prof_enable(True)
        reps = 20
        for _ in range(reps):
            Q, _ = pkg.orth(Y, 3, engine=eng)
        prof = eng.prof_query()
        eng.prof_enable(False)
        print(json.dumps({"orth": f"N=2500 k={k}", "passes": 3,
                          "small_linalg_us_per_pass": round(1e3 * prof["small_linalg"]["ms"] / (3 * reps), 2),
                          "gram_us_per_pass": round(1e3 * prof["gemm_f64"]["ms"] / (3 * reps), 2),
                          "orthogonality": float(np.abs(Q.T @ Q - np.eye(k)).max())}), flush=True)
    eng.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"])
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="d5chi100", choices=sorted(WORKLOADS))
    ap.add_argument("--forward-only", type=int, default=0, metavar="ITERS",
                    help="profiling aid: run ITERS forward CTMRG iterations of the workload once, no timing")
    ap.add_argument("--gemm-shapes", action="store_true",
                    help="kernel aid: FP64 GEMM throughput of the engine's DMMA kernel and of cuBLAS on the "
                         "projector's and the contractions' shapes, one JSON line per shape")
    ap.add_argument("--tf32-shapes", action="store_true",
                    help="kernel aid: 3xTF32 tcgen05 GEMM throughput (splits included) on the engine's shapes")
    ap.add_argument("--projector-shapes", action="store_true",
                    help="kernel aid: the projector alone on synthetic enlarged corners of the workload's size")
    ap.add_argument("--orth-shapes", action="store_true",
                    help="kernel aid: the projector's CholeskyQR alone on 2500 x k sketches (k = 160, 128, 101)")
    ap.add_argument("--optim-gs", type=int, default=0, metavar="STEPS",
                    help="workload aid: optim_gs (L-BFGS) for STEPS steps in each form, evals/s and final energies")
    ap.add_argument("--es-momentum", action="store_true",
                    help="workload aid: one excited-state momentum over the whole tangent basis (D=3 chi=48)")
    ap.add_argument("--es-gs-steps", type=int, default=10, help="L-BFGS steps of the ground state for --es-momentum")
    ap.add_argument("--es-workers", type=int, default=4,
                    help="contexts (streams, host threads) running --es-momentum's basis vectors concurrently")
    ap.add_argument("--pullback-profile", action="store_true",
                    help="profiling aid: one E+grad pullback of the workload alone, between cudaProfilerStart/Stop")
    args = ap.parse_args()
    global WORKLOAD, WORKLOAD_NAME
    if args.projector_shapes:
        WORKLOAD = WORKLOADS[args.workload]
        return run_projector_shapes()
    if args.orth_shapes:
        return run_orth_shapes()
    if args.optim_gs > 0:
        WORKLOAD = WORKLOADS[args.workload]
        WORKLOAD_NAME = workload_name(WORKLOAD)
        return run_optim_gs(args)
    if args.es_momentum:
        return run_es_momentum(args)
    if args.pullback_profile:
        WORKLOAD = WORKLOADS[args.workload]
        WORKLOAD_NAME = workload_name(WORKLOAD)
        return run_pullback_profile(args)
    if args.gemm_shapes:
        return run_gemm_shapes()
    if args.tf32_shapes:
        return run_tf32_shapes()
    WORKLOAD = WORKLOADS[args.workload]
    WORKLOAD_NAME = workload_name(WORKLOAD)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
