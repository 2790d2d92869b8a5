#!/usr/bin/env python
"""Benchmark of the Gibbs-sweep hot path: sweeps/s of BPMF at K = 32 on the synthetic
138,000 x 27,000 matrix with 20M power-law observations (alpha = 2), mixed-precision batched
sampler vs the FP64 sampler, both on one B200, with the CPU oracle timed beside them.

A step is one Gibbs sweep (sample both modes, update both Normal-Wishart priors; test-set
evaluation excluded from the timed region and reported separately).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is the mixed-precision sweep rate with the data already resident in HBM, timed with CUDA
events on the library's stream; `e2e` is the same metric through the C ABI with host buffers
(data upload and CSR build, per-sweep RMSE read-back and the final prediction read-back inside
the timed region).  `--impl reference` times the CPU oracle (FP64 restatement of the reference,
OpenMP on all host cores).  Under torchrun (N > 1) the ranks run one chain whose half-sweeps
are split by rows (an all-gather of the new rows after each), or with `--sharding replicas`
one independent chain each.
Both GPU arms pick their row samplers' work split and CTA shape with the library's autotuner at
initialisation (outside the timed region; `--no-autotune` keeps the default shapes).
"""
import argparse
import json
import math
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

METRIC = "Gibbs sweeps/s at K=32: mixed-prec batched vs FP64 plain, equal test RMSE"
UNIT = "sweeps/s"
K_LATENT = 32
ALPHA = 2.0
PROFILE_SUMMARY = ROOT / "profiles" / "k_gram_tc_fused_bpmf_powerlaw_k32.md"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=float, default=1.0, help="workload scale (1.0 = full size)")
    ap.add_argument("--cpu-seconds", type=float, default=20.0,
                    help="budget of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="default work split and CTA shape (no autotuner) in the headline arms")
    ap.add_argument("--e2e-steps", type=int, default=0, help="sweeps of the e2e run (0: = steps)")
    ap.add_argument("--no-side", action="store_true",
                    help="skip the side-information legs (Macau block-CG and univariate priors)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the 512-problem batched leg")
    ap.add_argument("--no-precision", action="store_true",
                    help="skip the Gram precision sweep on the 2,000 x 1,500 matrix")
    ap.add_argument("--sharding", choices=["rows", "replicas"], default=None,
                    help="one chain with each half-sweep's rows split over the ranks (rows, the "
                         "default for N > 1; given explicitly it also runs at N = 1) or one "
                         "independent chain per rank (replicas)")
    ap.add_argument("--no-uniform", action="store_true",
                    help="skip the K = 10 legs on the 2,000 x 1,500 matrix (GPU and CPU rates)")
    ap.add_argument("--only", choices=["all", "mixed", "fp64", "macau", "univariate", "precision",
                                       "batched"],
                    default="all",
                    help="profiling runs: time one sampler and print its phase times only")
    return ap.parse_args()


def workload(scale, seed):
    from macau_b200 import workloads
    return workloads.bpmf_powerlaw(seed=seed, scale=scale)


def config_dict(w, args, n):
    return {"workload": w["name"], "K": K_LATENT, "alpha": ALPHA,
            "holdout": "10% random", "rows": w["shape"][0], "cols": w["shape"][1],
            "ntrain": int(len(w["vals"])), "ntest": int(len(w["tvals"])),
            "parallelism": f"independent chains x{n}" if n > 1 else "single GPU",
            "l2": "inputs larger than L2 (per sweep the two packed CSR streams are %.0f MB)"
                  % (2 * len(w["vals"]) * 8 / 1e6),
            "eval": "excluded from the timed sweeps"}


# ------------------------------------------------------------------------ clocks
class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while the timed region runs."""

    FIELDS = ("index,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id=None):
        self.bus_id = (bus_id or "").lower()
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 10:
                self.rows.append(parts)

    def __exit__(self, *a):
        time.sleep(0.2)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = self.rows
        if self.bus_id:
            mine = [r for r in rows if self.bus_id.endswith(r[1].lower()[-12:]) or
                    r[1].lower().endswith(self.bus_id[-12:])]
            rows = mine or rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[6 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[4]) for r in rows
                                                         if r[4].replace(".", "").isdigit())
                if any(r[4].replace(".", "").isdigit() for r in rows) else None}


# ------------------------------------------------------------------------ helpers
def make_sampler(w, compute, seed, device, burnin=10 ** 6, nsamples=1, autotune=0):
    """autotune: 0 default work split and CTA shape, 1 the autotuner with its choice cache,
    2 the autotuner timing every candidate (mg_set_option "autotune", run by mg_init)."""
    from macau_b200 import _lib
    s = _lib.Sampler(K_LATENT, ALPHA, seed=seed, compute=compute, device=device)
    s.set_relation_data(w["rows"], w["cols"], w["vals"], w["shape"])
    s.set_relation_data_test(w["trows"], w["tcols"], w["tvals"], w["shape"])
    s.set_samples(burnin, nsamples)
    if autotune:
        s.set_option("autotune", autotune)
    s.init()
    return s


def sampler_bytes(st, w, compute, mode):
    """Algorithmic bytes of one latent-sampler launch (mode 0 = rows, 1 = columns): the CSR
    stream, the task list, one compulsory read of the other factor and the latent writes."""
    KP = 32
    N = w["shape"][mode]
    No = w["shape"][1 - mode]
    nnz = st["nnz"][mode]
    tasks = st["ntasks"][mode] * 32
    if compute == "mixed":
        return nnz * 8 + tasks + No * KP * 2 + N * KP * (4 + 2)
    return nnz * (4 + 8) + tasks + No * KP * 8 + N * KP * 8


def read_traffic():
    """DRAM bytes per half-sweep of the sampler (the fused k_gram_tc, mean of the two modes, full
    size) from the committed ncu summary, if any."""
    try:
        for line in PROFILE_SUMMARY.read_text().splitlines():
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":")[1].split()[0])
    except OSError:
        pass
    return None


def side_info_legs(device, sweeps=20, cpu_sweeps=2):
    """Sweep rates with side information on the 20,000 x 500 matrix with a binary 20,000 x
    32,768 Zipf feature matrix (K = 32): the Macau prior (block-CG link solve) and the univariate
    prior, FP64 and mixed, each beside the CPU oracle's FP64 sweep of the same model."""
    from macau_b200 import _lib, workloads
    from oracle import oracle as orc
    from tests.gpu_helpers import oracle_model
    import scipy.sparse as sp
    w = workloads.macau_side()
    fr, fc, _, shp = w["side"]
    cores = orc.set_threads(os.cpu_count() or 1)
    out = {"workload": w["name"], "K": K_LATENT, "alpha": ALPHA, "cg_tol": 1e-6,
           "lambda_beta": 5.0}
    for prior in ("macau", "univariate"):
        leg = {}
        for comp, name in ((_lib.MG_COMPUTE_FP64, "fp64"), (_lib.MG_COMPUTE_MIXED, "mixed")):
            s = _lib.Sampler(K_LATENT, ALPHA, seed=5, compute=comp, device=device)
            s.set_relation_data(w["rows"], w["cols"], w["vals"], w["shape"])
            if prior == "macau":
                s.set_side(0, fr, fc, None, shp, 5.0, 1e-6)
            else:
                s.set_side_univariate(0, fr, fc, None, shp, 5.0)
            s.set_samples(10 ** 6, 1)
            s.init()
            s.time_sweeps(0, 3, eval=False)
            t, _ = s.time_sweeps(3, sweeps, eval=False)
            st = s.stats()
            leg[name] = {"sweeps_per_s": sweeps / t, "ms_per_sweep": t / sweeps * 1e3}
            if prior == "macau":
                leg[name]["cg_iters_last"] = st["cg_iters"][0]
            s.close()
        m = oracle_model(w, K_LATENT, ALPHA, 5)
        if prior == "univariate":
            F = sp.coo_matrix((np.ones(len(fr)), (fr, fc)), shape=shp)
            m.set_side_one(0, orc.Csr.from_scipy(F, True), orc.Csr.from_scipy(F.T, True), 5.0)
        n_cpu = cpu_sweeps if prior == "macau" else 5 * cpu_sweeps
        m.sweep(0, 10 ** 6)
        t0 = time.perf_counter()
        for it in range(1, 1 + n_cpu):
            m.sweep(it, 10 ** 6)
        tc = time.perf_counter() - t0
        leg["cpu_oracle"] = {"sweeps_per_s": n_cpu / tc, "sample": f"{n_cpu} FP64 sweeps",
                             "cores": cores}
        leg["mixed_over_cpu"] = leg["mixed"]["sweeps_per_s"] / leg["cpu_oracle"]["sweeps_per_s"]
        out[prior] = leg
    return out


def uniform_legs(device, burnin=200, nsamples=200):
    """The CPU-scale BPMF case: the 2,000 x 1,500 uniform matrix (60,000 entries, 10% holdout,
    K = 10, alpha = 4, seed 0), burnin + nsamples sweeps.  Sweep rates (CUDA events) of the GPU
    FP64 and mixed samplers, the CPU oracle's FP64 rate on all host cores, and each chain's
    posterior-mean test RMSE."""
    from macau_b200 import _lib, workloads
    from oracle import oracle as orc
    from tests.gpu_helpers import oracle_model
    w = workloads.bpmf_uniform(seed=0)
    K, alpha, n = 10, 4.0, burnin + nsamples
    out = {"workload": w["name"], "K": K, "alpha": alpha, "burnin": burnin, "nsamples": nsamples}
    for comp, name in ((_lib.MG_COMPUTE_FP64, "gpu_fp64"), (_lib.MG_COMPUTE_MIXED, "gpu_mixed")):
        s = _lib.Sampler(K, alpha, seed=0, compute=comp, device=device)
        s.set_relation_data(w["rows"], w["cols"], w["vals"], w["shape"])
        s.set_relation_data_test(w["trows"], w["tcols"], w["tvals"], w["shape"])
        s.set_samples(burnin, nsamples)
        s.init()
        t, _ = s.time_sweeps(0, n, eval=True)
        out[name] = {"sweeps_per_s": n / t, "test_rmse": s.rmse()[0],
                     "note": "sweeps with test evaluation, captured graph"}
        s.close()
    cores = orc.set_threads(os.cpu_count() or 1)
    m = oracle_model(w, K, alpha, 0)
    t0 = time.perf_counter()
    for it in range(n):
        m.sweep(it, burnin)
    tc = time.perf_counter() - t0
    out["cpu_oracle"] = {"sweeps_per_s": n / tc, "test_rmse": m.rmse()[0], "cores": cores,
                         "kind": "port"}
    out["gpu_fp64_over_cpu"] = out["gpu_fp64"]["sweeps_per_s"] / out["cpu_oracle"]["sweeps_per_s"]
    out["rmse_mixed_minus_oracle"] = out["gpu_mixed"]["test_rmse"] - out["cpu_oracle"]["test_rmse"]
    return out


def precision_sweep(device, Ks=(16, 64, 128), burnin=100, nsamples=100):
    """The Gram precision sweep on the 2,000 x 1,500 uniform matrix (60,000 entries, 10% holdout,
    alpha = 4): for each K and Gram input precision (FP64 path; mixed with BF16, FP16 or TF32
    inputs, FP32 accumulation and factor, FP64 retry), the per-row sample error against the
    FP64 sampler under identical keyed draws from one common state, the retry rate of that
    half-sweep, and the test RMSE after burnin + nsamples sweeps from the initial state."""
    from macau_b200 import _lib, workloads
    w = workloads.bpmf_uniform()
    alpha = 4.0
    variants = (("fp64", _lib.MG_COMPUTE_FP64, 0), ("bf16", _lib.MG_COMPUTE_MIXED, 0),
                ("fp16", _lib.MG_COMPUTE_MIXED, 1), ("tf32", _lib.MG_COMPUTE_MIXED, 2))
    out = {"workload": w["name"], "alpha": alpha, "burnin": burnin, "nsamples": nsamples,
           "error": "max |u - u_fp64| / max |u_fp64| over the rows of one mode-0 half-sweep",
           "results": {}}

    def sampler(K, comp, g):
        s = _lib.Sampler(K, alpha, seed=11, compute=comp, device=device)
        s.set_relation_data(w["rows"], w["cols"], w["vals"], w["shape"])
        s.set_relation_data_test(w["trows"], w["tcols"], w["tvals"], w["shape"])
        if comp == _lib.MG_COMPUTE_MIXED:
            s.set_option("gram_precision", g)
        s.set_samples(burnin, nsamples)
        s.init()
        return s

    for K in Ks:
        rng = np.random.default_rng(K)
        V = rng.normal(scale=0.3, size=(w["shape"][1], K))
        mu = rng.normal(scale=0.1, size=K)
        A = rng.normal(size=(K, K))
        Lam = 2.0 * (A @ A.T / K + np.eye(K))
        res, ref = {}, None
        for name, comp, g in variants:
            s = sampler(K, comp, g)
            s.set_latents(1, V)
            s.set_hyper(0, mu, Lam, None)
            s.sample_latents(0, 0)
            U = s.latents(0)
            st = s.stats()
            s.close()
            if ref is None:
                ref = U
            s = sampler(K, comp, g)
            s.sweeps(0, burnin + nsamples, eval=True)
            rmse = s.rmse()[0]
            s.close()
            res[name] = {"sample_error": float(np.abs(U - ref).max() / np.abs(ref).max()),
                         "retry_rate": st["retries"][0] / max(1, w["shape"][0]),
                         "test_rmse": rmse}
        for name in res:
            res[name]["rmse_minus_fp64"] = res[name]["test_rmse"] - res["fp64"]["test_rmse"]
        out["results"][f"K={K}"] = res
    return out


def batched_legs(device, sweeps=20, single_sweeps=3, autotune=True):
    """512 independent BPMF problems of uneven size (rows U[200, 4000], columns U[100, 1000],
    density U[1%, 5%], K in {8, 16, 32}, noise 0.5, alpha = 4): all chains in one graph per sweep
    (mg_batch, mixed) against one problem at a time with the FP64 single-problem sampler."""
    from macau_b200 import _lib, workloads
    problems, Ks, seeds = workloads.batched_uneven()
    alpha = 4.0
    b = _lib.Batch(problems, Ks, seeds, alpha, device=device)
    b.init(10 ** 6)
    tuning = b.autotune(use_cache=False) if autotune else b.tuning()
    b.time_sweeps(0, 3)
    t = b.time_sweeps(3, sweeps)
    info = b.info()
    b.init(sweeps // 2)
    b.sweeps(0, sweeps, eval=True)
    rm = b.rmse()
    b.close()
    out = {"problems": len(problems), "ntrain": info["nnz"],
           "rows": info["rows"], "cols": info["cols"],
           "K_counts": {str(k): Ks.count(k) for k in sorted(set(Ks))},
           "batched_mixed": {"sweeps_per_s": sweeps / t, "ms_per_sweep": t / sweeps * 1e3,
                             "retries": info["retries"],
                             "mean_test_rmse": float(np.mean(rm[:, 0])),
                             "note": "one sweep = every problem sampled once; rmse after "
                                     f"{sweeps // 2} + {sweeps - sweeps // 2} sweeps",
                             "autotune": tuning}}
    tot = 0.0
    for pr, K, sd in zip(problems, Ks, seeds):
        s = _lib.Sampler(K, alpha, seed=sd, compute=_lib.MG_COMPUTE_FP64, device=device)
        s.set_relation_data(pr["rows"], pr["cols"], pr["vals"], pr["shape"])
        s.set_samples(10 ** 6, 1)
        if autotune:
            s.set_option("autotune", 2)
        s.init()
        s.time_sweeps(0, 1, eval=False)
        tp, _ = s.time_sweeps(1, single_sweeps, eval=False)
        tot += tp / single_sweeps
        s.close()
    out["single_fp64"] = {"sweeps_per_s": 1.0 / tot, "ms_per_sweep": tot * 1e3,
                          "note": "sum over problems of each problem's own FP64 sweep time "
                                  "(captured graph, CUDA events)"}
    out["batched_over_single_fp64"] = out["batched_mixed"]["sweeps_per_s"] * tot
    # one problem at a time with the mixed sampler (default shapes)
    tot_mx = 0.0
    for pr, K, sd in zip(problems, Ks, seeds):
        s = _lib.Sampler(K, alpha, seed=sd, compute=_lib.MG_COMPUTE_MIXED, device=device)
        s.set_relation_data(pr["rows"], pr["cols"], pr["vals"], pr["shape"])
        s.set_samples(10 ** 6, 1)
        s.init()
        s.time_sweeps(0, 1, eval=False)
        tp, _ = s.time_sweeps(1, single_sweeps, eval=False)
        tot_mx += tp / single_sweeps
        s.close()
    out["single_mixed"] = {"sweeps_per_s": 1.0 / tot_mx, "ms_per_sweep": tot_mx * 1e3,
                           "note": "sum over problems of each problem's own mixed sweep time"}
    out["batched_over_single_mixed"] = out["batched_mixed"]["sweeps_per_s"] * tot_mx
    # CPU oracle (FP64, all host cores) on a bounded sample of the problems, scaled to the set
    # by training entries
    from oracle import oracle as orc
    from tests.gpu_helpers import oracle_model
    cores = orc.set_threads(os.cpu_count() or 1)
    t_cpu, nnz_cpu, ncpu = 0.0, 0, 0
    for pr, K, sd in zip(problems, Ks, seeds):
        m = oracle_model(pr, K, alpha, sd)
        m.sweep(0, 10 ** 6)
        t0 = time.perf_counter()
        for it in range(1, 3):
            m.sweep(it, 10 ** 6)
        t_cpu += (time.perf_counter() - t0) / 2
        nnz_cpu += len(pr["vals"])
        ncpu += 1
        if t_cpu > 10.0:
            break
    t_set = t_cpu * info["nnz"] / nnz_cpu
    out["cpu_oracle"] = {"sweeps_per_s": 1.0 / t_set, "cores": cores, "kind": "port",
                         "sample": f"2 FP64 sweeps of each of the first {ncpu} problems, the "
                                   "set's time scaled by its training entries"}
    out["batched_over_cpu"] = out["batched_mixed"]["sweeps_per_s"] * t_set
    return out


def peaks():
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


def cpu_baseline(w, budget_s, sweeps_max):
    """Times the CPU oracle (FP64 restatement, all host cores) on full sweeps of the same data."""
    from oracle import oracle as orc
    from tests.gpu_helpers import oracle_model
    cores = orc.set_threads(os.cpu_count() or 1)
    m = oracle_model(w, K_LATENT, ALPHA, 0)
    t0 = time.perf_counter()
    m.sweep(0, 10 ** 6)
    t1 = time.perf_counter() - t0
    n = int(max(1, min(sweeps_max, math.floor(budget_s / max(t1, 1e-9)) - 1)))
    t0 = time.perf_counter()
    for i in range(n):
        m.sweep(1 + i, 10 ** 6)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{n} full FP64 sweeps (after 1 untimed) of {w['name']}, K=32"}


class Ranks:
    """The multi-process plumbing of a run: one process per GPU, launched by torchrun (RANK,
    LOCAL_RANK, WORLD_SIZE, MASTER_* in the environment).  Each rank runs an independent chain
    (seed 1000 + rank); timings are taken as the maximum over ranks and whole-job rates count
    every rank's work.  backend "nccl" with device "cuda:<local rank>" on GPUs; the CPU tests
    use "gloo" with device "cpu"."""

    def __init__(self, backend="nccl", device=None, timeout_s=600):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.device = device if device is not None else f"cuda:{self.local}"
        self.dist = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            if self.device.startswith("cuda"):
                import torch
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def chain_seed(self):
        return 1000 + self.rank

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x):
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def rate(self, units_per_rank, seconds_max):
        """Whole-job rate: every rank processed `units_per_rank` within `seconds_max`."""
        return self.world * units_per_rank / seconds_max

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


# ------------------------------------------------------------------------ arms
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    w = workload(args.scale, 2)
    from oracle import oracle as orc
    from tests.gpu_helpers import oracle_model
    cores = orc.set_threads(os.cpu_count() or 1)
    m = oracle_model(w, K_LATENT, ALPHA, 0)
    for i in range(args.warmup):
        m.sweep(i, 10 ** 6)
    t0 = time.perf_counter()
    for i in range(args.steps):
        m.sweep(args.warmup + i, 10 ** 6)
    dt = time.perf_counter() - t0
    v = args.steps / dt
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded power-law stand-in, no dataset read)",
            "config": config_dict(w, args, 1), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{args.steps} full FP64 sweeps after {args.warmup} warm-up"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_sharded(args, ranks, w, local, clk_bus):
    """N > 1, --sharding rows: one mixed-precision chain whose half-sweeps are split over the
    ranks by rows (macau_b200/sharded.py): each rank samples an entry-balanced row range, the
    new rows are all-gathered over NCCL into every rank's latent buffer (on the library's
    stream), and every rank updates the hyperparameters itself from the same latents.  `value`
    is that one chain's sweeps/s (the whole job's throughput; strong scaling), timed with CUDA
    events on the library stream and taken as the maximum over ranks."""
    import torch
    from macau_b200 import _lib, sharded
    K, W = args.steps, args.warmup
    world, rank = ranks.world, ranks.rank
    lengths = [np.bincount(w["rows"], minlength=w["shape"][0]),
               np.bincount(w["cols"], minlength=w["shape"][1])]
    dev = torch.device(f"cuda:{local}")
    seed = 1000  # one chain: the same seed on every rank

    def chain_for(s):
        return sharded.ShardedChain(sharded.LibraryBackend(s, dev), ranks.dist, rank, world,
                                    lengths)

    mx = make_sampler(w, _lib.MG_COMPUTE_MIXED, seed, local)
    chain = chain_for(mx)
    for it in range(W):
        chain.sweep(it)
    stream = torch.cuda.ExternalStream(mx.stream(), device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ranks.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(clk_bus) as clk:
        e0.record(stream)
        for it in range(W, W + K):
            chain.sweep(it)
        e1.record(stream)
        e1.synchronize()
    torch.cuda.synchronize(dev)
    t = ranks.max(e0.elapsed_time(e1) * 1e-3)
    st = mx.stats()
    mx.close()
    # e2e: set-up from host buffers, the sharded sweeps with evaluation, result read-back
    ranks.barrier()
    t0 = time.perf_counter()
    s = _lib.Sampler(K_LATENT, ALPHA, seed=seed, compute=_lib.MG_COMPUTE_MIXED, device=local)
    s.set_relation_data(w["rows"], w["cols"], w["vals"], w["shape"])
    s.set_relation_data_test(w["trows"], w["tcols"], w["tvals"], w["shape"])
    s.set_samples(0, K)
    s.init()
    h2d0, d2h0 = s.stats()["h2d_bytes"], s.stats()["d2h_bytes"]
    ch = chain_for(s)
    for it in range(K):
        ch.sweep(it)
        s.eval(it)
        s.rmse()
    preds = s.predictions()
    t_e2e = ranks.max(time.perf_counter() - t0)
    st_e = s.stats()
    rmse = s.rmse()[0]
    s.close()
    del preds
    line = {"metric": METRIC, "value": K / t, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": t / K * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "bf16-gram/f32-chol/f64-hyper",
            "data": "synthetic (seeded power-law stand-in, no dataset read)",
            "config": dict(config_dict(w, args, world),
                           parallelism=f"rows of each half-sweep split over {world} ranks, "
                                       "all-gather of the new rows (NCCL)"),
            "sharding": {"ranges": [ch.ranges[m][rank] for m in (0, 1)],
                         "collective": "all_gather of each half-sweep's latent rows"},
            "test_rmse": {"mixed": rmse},
            "gpu_launches": int(round(st["kernel_launches"] / max(1, st["sweeps"]) * K)),
            "clocks": clk.summary(),
            "e2e": {"value": K / t_e2e, "unit": UNIT,
                    "h2d_bytes_per_step": (st_e["h2d_bytes"] - h2d0) / K,
                    "d2h_bytes_per_step": (st_e["d2h_bytes"] - d2h0) / K,
                    "timed": "C-ABI set-up from host buffers, sharded sweeps with evaluation "
                             "and RMSE read-back, predictions read-back"}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def run_ours(args):
    from macau_b200 import _lib
    ranks = Ranks("nccl")
    world, rank, local = ranks.world, ranks.rank, ranks.local
    barrier, max_over_ranks = ranks.barrier, ranks.max

    import torch
    bus = None
    try:
        props = torch.cuda.get_device_properties(local)
        bus = getattr(props, "pci_bus_id", None)
        if isinstance(bus, int):
            bus = "%02x:00" % bus
    except Exception:
        pass

    seed = ranks.chain_seed()
    K, W = args.steps, args.warmup
    if args.only == "precision":
        print(json.dumps({"only": "precision", "precision_sweep": precision_sweep(local)}),
              flush=True)
        ranks.close()
        return 0
    if args.only == "batched":
        print(json.dumps({"only": "batched",
                          "batched": batched_legs(local, autotune=not args.no_autotune)}),
              flush=True)
        ranks.close()
        return 0
    if args.only in ("macau", "univariate"):
        # one side-information sampler (FP64) on the Macau workload, for profiling
        from macau_b200 import workloads
        ws = workloads.macau_side(scale=args.scale)
        fr, fc, _, shp = ws["side"]
        s = _lib.Sampler(K_LATENT, ALPHA, seed=seed, compute=_lib.MG_COMPUTE_FP64, device=local)
        s.set_relation_data(ws["rows"], ws["cols"], ws["vals"], ws["shape"])
        if args.only == "macau":
            s.set_side(0, fr, fc, None, shp, 5.0, 1e-6)
        else:
            s.set_side_univariate(0, fr, fc, None, shp, 5.0)
        s.set_samples(10 ** 6, 1)
        s.init()
        s.time_sweeps(0, max(W, 1), eval=False)
        t, _ = s.time_sweeps(W, K, eval=False)
        _, ph = s.time_sweeps(W + K, K, eval=False, phase_events=True)
        print(json.dumps({"only": args.only, "workload": ws["name"], "ms_per_step": t / K * 1e3,
                          "phase_ms": [x / K * 1e3 for x in ph], "stats": s.stats()}), flush=True)
        s.close()
        ranks.close()
        return 0
    w = workload(args.scale, 2)
    sharding = args.sharding or ("rows" if world > 1 else "replicas")
    if sharding == "rows" and args.only == "all":
        return run_sharded(args, ranks, w, local, bus)
    if args.only != "all":
        comp = _lib.MG_COMPUTE_MIXED if args.only == "mixed" else _lib.MG_COMPUTE_FP64
        s = make_sampler(w, comp, seed, local, autotune=0 if args.no_autotune else 2)
        s.time_sweeps(0, max(W, 1), eval=False)
        t, _ = s.time_sweeps(W, K, eval=False)
        _, ph = s.time_sweeps(W + K, K, eval=False, phase_events=True)
        print(json.dumps({"only": args.only, "workload": w["name"], "ms_per_step": t / K * 1e3,
                          "phase_ms": [x / K * 1e3 for x in ph], "stats": s.stats()}), flush=True)
        s.close()
        ranks.close()
        return 0
    # ---- mixed-precision batched sampler: headline value ----
    tune = 0 if args.no_autotune else 2
    mx = make_sampler(w, _lib.MG_COMPUTE_MIXED, seed, local, autotune=tune)
    tuning = {"mixed": mx.tuning()}
    mx.time_sweeps(0, max(W, 1), eval=False)
    barrier()
    with ClockSampler(bus) as clk:
        t_mx, _ = mx.time_sweeps(W, K, eval=False)
    t_mx = max_over_ranks(t_mx)
    st_mx = mx.stats()
    kernels_per_sweep = st_mx["kernel_launches"] / max(1, st_mx["sweeps"])
    # per-kernel durations for the roofline (same kernels, un-captured, events between phases)
    _, ph = mx.time_sweeps(W + K, min(K, 50), eval=False, phase_events=True)
    nph = min(K, 50)
    # test RMSE after the chain continues with evaluation (posterior mean over 20 sweeps)
    mx.set_samples(W + K + nph, 20)
    mx.sweeps(W + K + nph, 20, eval=True)
    rmse_mx = mx.rmse()[0]
    retries = st_mx["retries"]
    mx.close()
    # ---- FP64 plain sampler ----
    fp = make_sampler(w, _lib.MG_COMPUTE_FP64, seed, local, autotune=tune)
    tuning["fp64"] = fp.tuning()
    fp.time_sweeps(0, max(W, 1), eval=False)
    barrier()
    t_fp, _ = fp.time_sweeps(W, K, eval=False)
    t_fp = max_over_ranks(t_fp)
    _, ph_fp = fp.time_sweeps(W + K, min(K, 20), eval=False, phase_events=True)
    fp.set_samples(W + K + min(K, 20), 20)
    fp.sweeps(W + K + min(K, 20), 20, eval=True)
    rmse_fp = fp.rmse()[0]
    st_fp = fp.stats()
    fp.close()
    # ---- e2e through the C ABI with host buffers ----
    E = args.e2e_steps or K
    barrier()
    h2d0, d2h0 = st_fp["h2d_bytes"], st_fp["d2h_bytes"]
    t0 = time.perf_counter()
    s = _lib.Sampler(K_LATENT, ALPHA, seed=seed, compute=_lib.MG_COMPUTE_MIXED, device=local)
    if tune:
        s.set_option("autotune", 1)  # the choice of the mixed arm, from the autotuner's cache
    ta = time.perf_counter()
    s.set_relation_data(w["rows"], w["cols"], w["vals"], w["shape"])
    tb = time.perf_counter()
    s.set_relation_data_test(w["trows"], w["tcols"], w["tvals"], w["shape"])
    tc = time.perf_counter()
    s.set_samples(0, E)
    s.init()
    t1 = time.perf_counter()
    tuning["e2e"] = [t["state"] for t in s.tuning()]
    for i in range(E):
        s.sweep(i, eval=True)
        s.rmse()
    t2 = time.perf_counter()
    preds = s.predictions()
    t_e2e = time.perf_counter() - t0
    e2e_split = {"setup_s": t1 - t0, "sweeps_s": t2 - t1, "readback_s": t0 + t_e2e - t2,
                 "setup_parts_s": {"create": ta - t0, "train": tb - ta, "test": tc - tb,
                                   "init": t1 - tc}}
    st_e = s.stats()
    s.close()
    t_e2e = max_over_ranks(t_e2e)
    h2d = st_e["h2d_bytes"] - h2d0
    d2h = st_e["d2h_bytes"] - d2h0
    del preds

    # ---- roofline of the dominant step: the latent sampler (the fused k_gram_tc) ----
    hbm, tflops, src = peaks()
    b = sampler_bytes(st_mx, w, "mixed", 0) + sampler_bytes(st_mx, w, "mixed", 1)
    t_launch = (ph[0] + ph[1]) / (2 * nph)     # mean seconds per half-sweep of the sampler
    achieved = b / 2 / t_launch / 1e9
    traffic = read_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic, "peak_source": src,
                "kernel": "latent sampler half-sweep (fused k_gram_tc: tensor-core Grams and "
                          "the rows' finish), mean of the two modes, CUDA events on the library "
                          "stream",
                "algorithmic_bytes_per_launch": b / 2}
    if ph[5] > 0:
        t_gram = (ph[5] + ph[6]) / (2 * nph)   # mean seconds per k_gram_tc launch
        gflop = sum(st_mx["nnz"][m] * (K_LATENT * (K_LATENT + 1) + 2 * K_LATENT) for m in (0, 1)) / 2
        gathered = sum(st_mx["nnz"][m] for m in (0, 1)) / 2 * K_LATENT * 2
        roofline["gram_kernel"] = {
            "name": "k_gram_tc (fused: Gram + finish)", "ms_per_launch": t_gram * 1e3,
            "share_of_sampler": (ph[5] + ph[6]) / (ph[0] + ph[1]),
            "algorithmic_tflops": gflop / t_gram / 1e12, "tensor_peak_bf16": tflops,
            "tensor_frac": gflop / t_gram / 1e12 / tflops,
            "l2_gather_GBps": gathered / t_gram / 1e9}
    v_mx = ranks.rate(K, t_mx)
    v_fp = ranks.rate(K, t_fp)
    line = {"metric": METRIC, "value": v_mx, "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": t_mx / K * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16-gram/f32-chol/f64-hyper",
            "data": "synthetic (seeded power-law stand-in, no dataset read)",
            "config": config_dict(w, args, world),
            "fp64_value": v_fp, "fp64_ms_per_step": t_fp / K * 1e3,
            "mixed_over_fp64": v_mx / v_fp,
            "test_rmse": {"mixed": rmse_mx, "fp64": rmse_fp,
                          "note": "posterior mean of 20 evaluated sweeps after the timed ones"},
            "phase_ms": {"mixed": [x / nph * 1e3 for x in ph],
                         "fp64": [x / min(K, 20) * 1e3 for x in ph_fp],
                         "order": ["sample0", "sample1", "prior0", "prior1", "eval",
                                   "gram0", "gram1"]},
            "retries_fp64_refactor": retries,
            "gpu_launches": int(round(kernels_per_sweep * K)),
            "clocks": clk.summary(), "roofline": roofline,
            "e2e": {"value": ranks.rate(E, t_e2e), "unit": UNIT, "h2d_bytes_per_step": h2d / E,
                    "d2h_bytes_per_step": d2h / E,
                    "timed": "C-ABI run: data upload + CSR build, init (autotuner choice "
                             "from its cache), sweeps with eval and RMSE read-back, final "
                             "predictions read-back",
                    "split_s": e2e_split},
            "autotune": tuning}
    if rank == 0 and world == 1 and not args.no_side:
        line["side_info"] = side_info_legs(local)
    if rank == 0 and world == 1 and not args.no_precision:
        line["precision_sweep"] = precision_sweep(local)
    if rank == 0 and world == 1 and not args.no_uniform:
        line["uniform_k10"] = uniform_legs(local)
    if rank == 0 and world == 1 and not args.no_batched:
        line["batched"] = batched_legs(local, autotune=not args.no_autotune)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w, args.cpu_seconds, 50)
        line["mixed_over_cpu"] = v_mx / line["cpu_baseline"]["value"]
        line["fp64_over_cpu"] = v_fp / line["cpu_baseline"]["value"]
    if rank == 0:
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
