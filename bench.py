"""Benchmark: first-order density rho1 (+ grad rho1) grid points per second on
the config-2 workload, with the Hartree sum-up measured beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl frpa|reference]

One "step" is one pass of rho1 + grad rho1 over every grid batch of the
config-2 workload (1,000 atoms, 10 basis functions each, 30,000 uneven batches
of 100-300 points with 100-600 active functions, P1 within the batch-active
pattern), synthetic and seeded; FP64 in and out.  Under torchrun (N > 1) every
rank processes its own independently seeded workload of that size (weak
scaling; the batches are independent, so there is no collective on the data
path).  Rank 0 prints one JSON line.

--impl reference times the reference's own CPU implementation of the same
path (its evaluate_first_order_rho.cpp compiled from source into oracle/_ref,
all host threads, batches split across them) on a bounded sample of the same
workload and prints the same metric.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "rho1 grid pts/s: plain FP64 vs grouped split-BF16 @1e-10 rel err; sumup pts/s"
UNIT = "grid pts/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["frpa", "reference"], default="frpa")
    ap.add_argument("--batches", type=int, default=30_000, help="grid batches per rank (config 2: 30000)")
    ap.add_argument("--sumup-points", type=int, default=2_000_000)
    ap.add_argument("--sumup-lmax", type=str, default="4,6,8")
    ap.add_argument("--no-sumup", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="target CPU-baseline sample time")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (default tile shapes)")
    ap.add_argument("--config4-sizes", default="2000",
                    help="config-4 sweep sizes in atoms (comma list; 2000,10000,40000 for the full sweep)")
    ap.add_argument("--no-config4", action="store_true", help="skip the config-4 sweep")
    ap.add_argument("--no-config5", action="store_true", help="skip the adjoint / first-order H timings")
    ap.add_argument("--scaling", choices=["weak", "strong"], default="weak",
                    help="weak: each rank its own config-2 problem; strong: one problem, batches sharded by cost")
    ap.add_argument("--mode", choices=["fp64", "split", "i8"], default=None,
                    help="headline rho1 path (default: split if built, else fp64)")
    return ap.parse_args()


# ------------------------------------------------------------------ ranks


class Ranks:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False

    def init(self, use_gpu: bool):
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            backend = "nccl" if use_gpu else "gloo"
            dist.init_process_group(backend=backend, timeout=datetime.timedelta(minutes=10))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as dist

            dist.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        import torch.distributed as dist

        t = torch.tensor([v], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if not self.pg:
            return v
        import torch
        import torch.distributed as dist

        t = torch.tensor([v], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist

            dist.destroy_process_group()


# ----------------------------------------------------------------- clocks


class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons while a
    timed region runs; summarised as median SM MHz under load."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self._t = None

    def _gpu_id(self):
        try:
            import torch

            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            return uuid if uuid.startswith("GPU-") else "GPU-" + uuid
        except Exception:
            return str(self.dev)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self._gpu_id(), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, util, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
                util.append(float(parts[3]) if parts[3] not in ("[N/A]", "") else 100.0)
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        loaded = [s for s, u in zip(sm, util) if u >= 50] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm), "samples_under_load": len(loaded)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": d.get("hbm_gbs"), "bf16_tflops": d.get("bf16_tflops"),
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained"), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "fallback"}


def profile_traffic(name: str, batches: int = 30_000):
    """DRAM bytes of one step from the committed ncu summary, if present; the
    figures are for the 30,000-batch config-2 step and are scaled to
    `batches` (traffic grows with the batch count)."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            v = json.load(f).get(name)
        return None if v is None else v * batches / 30_000
    return None


# ------------------------------------------------------------ GPU helpers


def _dev(a, dtype=None):
    import torch

    a = np.asarray(a) if dtype is None else np.asarray(a).astype(dtype)
    return torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).cuda()


class Rho1Workload:
    """Config-2 batches with phi / grad phi generated on the device.  With
    ``shard = (rank, world)`` the problem is the same on every rank and this
    rank keeps its cost-balanced share of the batches (strong scaling)."""

    def __init__(self, n_batches: int, seed: int, shard=None):
        import torch

        from fast_rpa_eval_b200 import _lib, parallel, synth

        t0 = time.time()
        self.prob = p = synth.config2(seed=seed, n_batches=n_batches)
        if shard is not None:
            rank, world = shard
            ids = parallel.shard_batches(parallel.rho1_batch_costs(p), world)[rank]
            self.prob = p = parallel.select_batches(p, ids)
        self.t_host = time.time() - t0
        pts = _dev(np.asfortranarray(p.valid_points_xyz.T))
        self.wave = torch.empty(p.wave_len, dtype=torch.float64, device="cuda")
        self.gwave = torch.empty(3 * p.wave_len, dtype=torch.float64, device="cuda")
        _lib.synth_basis_values(p, pts, self.wave, self.gwave, pad_value=0.0)
        del pts
        self.P1 = _dev(p.first_order_density_matrix)
        self.bias = _dev(p.first_order_rho_bias_part2)
        self.gbias = _dev(p.first_order_gradient_rho_bias)
        self.rho = torch.zeros(p.n_full_points * p.T, dtype=torch.float64, device="cuda")
        self.grad = torch.zeros(3 * p.n_max_batch_size * p.n_my_batches_work * p.T, dtype=torch.float64,
                                device="cuda")
        self.plan = _lib.Rho1Plan(p)
        self.n_active = p.j_atom_end - p.j_atom_begin + 1
        self.points = p.total_points() * p.T
        self.flops = p.flops()
        self.bytes = p.algorithmic_bytes()
        torch.cuda.synchronize()

    def step(self, mode: int, stream):
        self.plan.execute(self.n_active, self.wave, self.gwave, self.P1, self.bias, self.gbias, self.rho, self.grad,
                          mode=mode, stream=stream)


def time_device_steps(fn, K: int, W: int, ranks: Ranks, stream):
    """W untimed steps, then K steps between CUDA events on `stream`,
    bracketed by barrier + synchronize; returns ms per step (max over ranks)."""
    import torch

    for _ in range(W):
        fn()
    torch.cuda.synchronize()
    ranks.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(K):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    ranks.barrier()
    return ranks.max(e0.elapsed_time(e1) / K)


def time_e2e(w: Rho1Workload, mode: int, K: int, W: int, ranks: Ranks):
    """The reference-facing call: evaluate_first_order_rho_..._cu_host_ on the
    session (constant arrays resident, phi borrowed in place), with P1 and the
    biases uploaded from pinned host memory and rho1 / grad rho1 downloaded
    every step, as the reference's host-copy mode does."""
    import torch

    from fast_rpa_eval_b200 import _lib

    p = w.prob
    pin = lambda t: t.cpu().pin_memory()  # noqa: E731
    P1, bias, gbias = pin(w.P1), pin(w.bias), pin(w.gbias)
    rho = torch.empty(w.rho.numel(), dtype=torch.float64).pin_memory()
    grad = torch.empty(w.grad.numel(), dtype=torch.float64).pin_memory()
    _lib.set_rho1_mode(mode)
    sess = _lib.Session(p, wave=w.wave, gradient_wave=w.gwave)
    try:
        for _ in range(W):
            sess.rho1(P1=P1, bias=bias, gbias=gbias, rho=rho, grad=grad)
        ranks.barrier()
        t0 = time.perf_counter()
        for _ in range(K):
            sess.rho1(P1=P1, bias=bias, gbias=gbias, rho=rho, grad=grad)
        dt = (time.perf_counter() - t0) / K
        ranks.barrier()
    finally:
        sess.close()
        _lib.set_rho1_mode(0)
    ms = ranks.max(dt * 1e3)
    check = np.asarray(rho.numpy()[: min(1000, rho.numel())])
    h2d = 8 * (P1.numel() + bias.numel() + gbias.numel())
    d2h = 8 * (rho.numel() + grad.numel())
    return ms, h2d, d2h, bool(np.isfinite(check).all())


def time_sumup(L: int, n_points: int, seed: int, K: int, W: int, ranks: Ranks, stream):
    """Config-3 sum-up at l_max = L; L2 flushed before every timed call (the
    inputs are smaller than L2), calls timed one by one with CUDA events."""
    import torch

    from fast_rpa_eval_b200 import _lib, synth

    p = synth.config3(l_max=L, n_points=n_points, seed=seed)
    plan = _lib.SumupPlan(p)
    args = (_dev(p.l_hartree_max_far_distance, np.int32), _dev(p.multipole_radius_sq), _dev(p.outer_potential_radius),
            _dev(p.multipole_moments), _dev(p.spline))
    dv = _dev(p.delta_v_hartree)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2
    for _ in range(W):
        plan.execute(1, *args, dv, stream=stream)
    torch.cuda.synchronize()
    ranks.barrier()
    times = []
    for _ in range(K):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.execute(1, *args, dv, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ranks.barrier()
    ms = ranks.max(sum(times) / K)
    fast = plan.fast
    plan.close()
    return p, ms, fast


def time_config5(K: int, W: int, ranks: Ranks, stream, fp64_peak: float, fma_peak: float):
    """Config 5 (the adjoint check): dL/dP1 and the first-order H with every
    exchange-correlation term on the config-1 recipe at 200 atoms, and dL/dQ
    of the sum-up at 100 atoms, l_max 6, 200,000 points.  Each call is timed
    with CUDA events over K calls after W warm-up calls; FLOPs are the
    contraction's 2 T nc^2 np (FP64 tensor pipe) and, for dQ, the forward's
    2 (L + 1)^2 per evaluated (point, atom) pair (FP64 FMA pipe)."""
    import torch

    from fast_rpa_eval_b200 import _lib, synth

    from fast_rpa_eval_b200 import parallel

    out = {}
    p = synth.make_rho1_problem(T=1, seed=5, n_atoms=200, box=None, density=0.1, n_batches=1600,
                                nc_range=(40, 120), exact_selection=False)
    if ranks.world > 1:  # each rank its cost share of the batches; dP1 summed over ranks (NCCL)
        p = parallel.select_batches(p, parallel.shard_batches(parallel.rho1_batch_costs(p), ranks.world)[ranks.rank])
    plan = _lib.Rho1Plan(p)
    rng = np.random.default_rng(5)
    w, gw = _dev(p.wave), _dev(p.gradient_wave)
    g_rho = _dev(rng.uniform(0.01, 1.0, p.n_full_points) * rng.normal(size=p.n_full_points))
    dP1 = torch.zeros(p.n_basis * p.n_basis, dtype=torch.float64, device="cuda")
    gemm = 2.0 * float(np.sum(p.n_compute_c_batches.astype(np.float64) ** 2 * p.n_point_batches))
    def adjoint_step():
        plan.adjoint_p1(1, w, gw, g_rho, None, dP1, stream=stream)
        if ranks.world > 1:
            parallel.all_reduce_sum(dP1)

    ms = time_device_steps(adjoint_step, K, W, ranks, stream)
    gemm = ranks.sum(gemm)
    out["adjoint_dP1"] = {"ms_per_call": ms, "tflops_fp64": gemm / (ms / 1e3) / 1e12,
                          "frac_of_measured_fp64_mma": gemm / (ms / 1e3) / 1e12 / fp64_peak / ranks.world,
                          "batches_per_rank": int(p.n_my_batches_work), "n_basis": int(p.n_basis),
                          "accumulation": "128-bit fixed point, bit-identical across runs",
                          "ranks": ranks.world,
                          "collective": "NCCL all-reduce of dP1 after each call" if ranks.world > 1 else None}
    xc = {k: _dev(a) for k, a in synth.first_order_h_inputs(p, seed=6).items()}
    vhg, pt = _dev(rng.normal(size=p.n_full_points)), _dev(p.partition_tab)
    av = torch.from_numpy(np.ascontiguousarray(p.atom_valid_n_compute_c_batches.ravel(order="F"),
                                               dtype=np.int32)).cuda()
    H = torch.zeros(p.n_basis * p.n_basis, dtype=torch.float64, device="cuda")
    ms = time_device_steps(lambda: plan.first_order_h(1, p.n_atoms, 1, 1, av, w, gw, xc["hessian_wave"], xc, vhg,
                                                      pt, H, stream=stream), K, W, ranks, stream)
    out["first_order_h"] = {"ms_per_call": ms, "tflops_fp64": gemm / (ms / 1e3) / 1e12,
                            "frac_of_measured_fp64_mma": gemm / (ms / 1e3) / 1e12 / fp64_peak / ranks.world,
                            "terms": "H_prefactor1, v_hartree_gradient, vsigma/gradient terms, v2rho2, v2rhosigma, "
                                     "v2sigma2, Hessian", "device_flags": plan.device_flags()}
    del plan, w, gw, xc, H, dP1
    s = synth.make_sumup_problem(n_atoms=100, n_points=200_000, l_pot_max=6, T=1, seed=9, outer_radius=8.0,
                                 l_hartree_per_species=[6, 5, 4, 6])
    sp = _lib.SumupPlan(s)
    args = (_dev(s.l_hartree_max_far_distance, np.int32), _dev(s.multipole_radius_sq), _dev(s.outer_potential_radius),
            _dev(s.multipole_moments))
    g = _dev(rng.normal(size=s.n_full_points))
    dQ = torch.empty(s.multipole_moments.size, dtype=torch.float64, device="cuda")
    ms = time_device_steps(lambda: sp.adjoint_q(1, *args, g, dQ, stream=stream), K, W, ranks, stream)
    flops = 2.0 * 49 * s.pair_count()
    out["adjoint_dQ"] = {"ms_per_call": ms, "pairs": int(s.pair_count()),
                         "tflops_convention_2L2": flops / (ms / 1e3) / 1e12,
                         "frac_of_measured_fp64_fma": flops / (ms / 1e3) / 1e12 / fma_peak}
    sp.close()
    return out


# ----------------------------------------------------------- CPU baseline


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_rho1_rate(sample, target_s: float, passes: int | None = None):
    """Grid points/s of the reference's own CPU rho1 (oracle/_ref) over
    `sample`, all host threads; repeats the sample up to ~target_s seconds."""
    import oracle

    n = host_threads()
    t0 = time.perf_counter()
    oracle.rho1_reference_threaded(sample, n)
    t1 = time.perf_counter() - t0
    reps = passes if passes is not None else max(0, min(50, int(target_s / max(t1, 1e-3)) - 1))
    tot, cnt = t1, 1
    for _ in range(reps):
        t0 = time.perf_counter()
        oracle.rho1_reference_threaded(sample, n)
        tot += time.perf_counter() - t0
        cnt += 1
    pts = sample.total_points() * sample.T
    return pts * cnt / tot, n, cnt, tot


def cpu_sample_batches(prob, threads: int) -> int:
    # about 4 ms of reference work per batch per thread; aim for ~1 s a pass
    return int(min(prob.n_my_batches_work, max(64, 250 * threads)))


def cpu_sumup_rate(L: int, n_points: int, target_s: float):
    """Points/s of the reference's own CPU sum-up (l_pot_max <= 6 only: its
    near field stops there) on a point sample of the config-3 recipe."""
    import oracle
    from fast_rpa_eval_b200 import synth

    n = host_threads()
    p = synth.config3(l_max=L, n_points=n_points, seed=4)
    t0 = time.perf_counter()
    oracle.sumup_reference_threaded(p, n)
    dt = time.perf_counter() - t0
    return n_points / dt, n, dt


# ---------------------------------------------------------- reference arm


def run_reference(args, ranks: Ranks):
    """The reference's CPU rho1 on the config-2 workload, bounded sample per
    step, all host threads (rank 0 only)."""
    if ranks.rank != 0:
        return None
    import oracle
    from fast_rpa_eval_b200 import synth

    if not oracle.ref_available(1):
        return {"impl": "reference", "unavailable": "oracle/_ref was not built (reference sources absent at build time)"}
    prob = synth.config2(seed=2, n_batches=args.batches)
    threads = host_threads()
    nb = cpu_sample_batches(prob, threads)
    wave, gwave = synth.host_basis_values(prob, nb)
    sample = synth.subset_batches(prob, nb, wave, gwave)
    for _ in range(args.warmup):
        oracle.rho1_reference_threaded(sample, threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.rho1_reference_threaded(sample, threads)
        times.append(time.perf_counter() - t0)
    pts = sample.total_points()
    ms = 1e3 * sum(times) / len(times)
    value = pts / (ms / 1e3)
    desc = f"first {nb} of {prob.n_my_batches_work} config-2 batches ({pts} grid points) per step"
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded config-2 recipe)", "impl": "reference",
        "config": {"workload": "config2: rho1 + grad rho1, 1000 atoms, 30000 batches of 100-300 points, "
                               "n_compute 100-600, T=1 (bounded CPU sample per step)",
                   "sample": desc, "path": "reference evaluate_first_order_rho.cpp (oracle/_ref), OpenBLAS dgemm "
                                           "sequential, batches split over host threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }


# ---------------------------------------------------------------- main arm


def run_frpa(args, ranks: Ranks):
    import torch

    from fast_rpa_eval_b200 import _lib, autotune

    torch.cuda.set_device(ranks.local)
    _lib.set_device(ranks.local)  # the library's own runtime: plans and the session on this rank's GPU
    stream = torch.cuda.current_stream()
    peaks = measured_peaks()
    mode_name = args.mode or "fp64"
    mode = {"split": _lib.RHO1_SPLIT_BF16, "i8": _lib.RHO1_SPLIT_I8}.get(mode_name, _lib.RHO1_FP64)
    out = {}

    if args.scaling == "strong":  # one config-2 problem, its batches shared out by cost
        w = Rho1Workload(args.batches, seed=2, shard=(ranks.rank, ranks.world))
    else:  # every rank its own seeded config-2 problem
        w = Rho1Workload(args.batches, seed=2 + 7919 * ranks.rank)
    p = w.prob
    info = w.plan.info()
    w_points, w_flops, w_bytes = int(p.total_points()), p.flops(), p.algorithmic_bytes()

    fp64_peak = _lib.probe_fp64_tflops("mma")
    fma_peak = _lib.probe_fp64_tflops("fma")

    # the autotuner picks each path's tile shape / schedule on these inputs
    # (results are identical for every candidate); the timed steps replay a
    # CUDA graph of each path's tuned launches
    tuned = {}
    if not args.no_tune:
        for m, nm in ((_lib.RHO1_FP64, "fp64"), (_lib.RHO1_SPLIT_BF16, "split")):
            tuned[nm] = autotune.tune_rho1(w.plan, p, lambda m=m: w.step(m, None), m, reps=2)
        out["autotune"] = {nm: {"choice": r["choice"], "timings_ms": r["timings"]} for nm, r in tuned.items()}
        tuned = {nm: r["choice"] for nm, r in tuned.items()}
    graphs = {m: _lib.capture_graph(lambda m=m: w.step(m, None))
              for m in (_lib.RHO1_FP64, _lib.RHO1_SPLIT_BF16, _lib.RHO1_SPLIT_I8)}

    n_items_tuned = w.plan.info()["n_items"]
    i8_groups = w.plan.i8_info()["groups"]

    # both rho1 paths are timed on the same inputs; the headline is --mode
    clocks = ClockSampler(ranks.local)
    clocks.start()
    ms_fp64 = time_device_steps(lambda: graphs[_lib.RHO1_FP64].replay(), args.steps, args.warmup, ranks, stream)
    ms_split = time_device_steps(lambda: graphs[_lib.RHO1_SPLIT_BF16].replay(), args.steps, args.warmup, ranks,
                                 stream)
    ms_i8 = time_device_steps(lambda: graphs[_lib.RHO1_SPLIT_I8].replay(), args.steps, args.warmup, ranks, stream)
    clk = clocks.stop()
    del graphs
    ms = {_lib.RHO1_FP64: ms_fp64, _lib.RHO1_SPLIT_BF16: ms_split, _lib.RHO1_SPLIT_I8: ms_i8}[mode]

    total_pts = ranks.sum(float(w.points))
    value = total_pts / (ms / 1e3)
    achieved_tf = w.flops / (ms_fp64 / 1e3) / 1e12

    # both split modes against plain FP64 on the full workload, same inputs
    split_out = {}
    for m in (_lib.RHO1_SPLIT_BF16, _lib.RHO1_SPLIT_I8):
        w.step(m, stream)
        torch.cuda.synchronize()
        split_out[m] = (w.rho.clone(), w.grad.clone())
    w.step(_lib.RHO1_FP64, stream)
    torch.cuda.synchronize()
    for m, key in ((_lib.RHO1_SPLIT_BF16, "split_vs_fp64_normwise_rel"),
                   (_lib.RHO1_SPLIT_I8, "split_i8_vs_fp64_normwise_rel")):
        rho_m, grad_m = split_out[m]
        out[key] = {"rho1": float((rho_m - w.rho).abs().max() / w.rho.abs().max()),
                    "grad_rho1": float((grad_m - w.grad).abs().max() / w.grad.abs().max())}
    out["device_flags"] = w.plan.device_flags()
    del split_out
    out["rho1_split_bf16"] = {"pts_per_s": total_pts / (ms_split / 1e3), "ms_per_step": ms_split,
                              "speedup_vs_fp64": ms_fp64 / ms_split,
                              "hbm_gbs_algorithmic": w_bytes / (ms_split / 1e3) / 1e9,
                              "roofline_frac_hbm_algorithmic": w_bytes / (ms_split / 1e3) / 1e9 / peaks["hbm_gbs"],
                              "bf16_equivalent_tflops": 15 * w_flops / (ms_split / 1e3) / 1e12}
    i8_traffic = profile_traffic("rho1_split_i8_step", p.n_my_batches_work)
    out["rho1_split_i8"] = {
        "pts_per_s": total_pts / (ms_i8 / 1e3), "ms_per_step": ms_i8, "speedup_vs_fp64": ms_fp64 / ms_i8,
        "kernels_per_group": "pack A (phi digits), pack B (P1c digits), tcgen05.mma.kind::i8 contraction",
        "groups": i8_groups,
        # roofline: the path's algorithmic bytes over the step time, against the
        # measured copy bandwidth; the DRAM bytes it actually moved (ncu, scaled
        # to this batch count) are reported beside it, not as the fraction
        "roofline": {"bound": "hbm", "achieved_gbs_algorithmic": w_bytes / (ms_i8 / 1e3) / 1e9,
                     "peak_gbs": peaks["hbm_gbs"], "frac": w_bytes / (ms_i8 / 1e3) / 1e9 / peaks["hbm_gbs"],
                     "algorithmic_bytes_per_step": w_bytes, "traffic_bytes_per_step": i8_traffic,
                     "achieved_dram_frac": (i8_traffic / (ms_i8 / 1e3) / 1e9 / peaks["hbm_gbs"])
                     if i8_traffic else None}}
    out["rho1_fp64"] = {"pts_per_s": total_pts / (ms_fp64 / 1e3), "ms_per_step": ms_fp64,
                        "tflops_fp64": achieved_tf, "frac_of_measured_fp64_mma": achieved_tf / fp64_peak,
                        "hbm_gbs_algorithmic": w.bytes / (ms_fp64 / 1e3) / 1e9}

    # the bias producer (generate_first_order_rho_bias_part2) for a 4-atom tile
    # on the same batches, P1 standing in for the ground-state density matrix
    av = torch.from_numpy(np.ascontiguousarray(p.atom_valid_n_compute_c_batches.ravel(order="F"),
                                               dtype=np.int32)).cuda()
    bias4 = torch.zeros(p.n_max_batch_size * p.n_my_batches_work * 4, dtype=torch.float64, device="cuda")
    na = min(4, p.n_atoms)

    def bias_step():
        w.plan.bias_part2(4, p.n_atoms, 1, na, 1, av, w.wave, w.gwave, w.P1, bias4)

    ms_bias = time_device_steps(bias_step, args.steps, args.warmup, ranks, stream)

    # rho1 with the density-matrix bias of atom 1 computed in the same launch,
    # against the two-launch form (bias producer, then plain FP64 rho1)
    bias1 = torch.zeros(p.n_max_batch_size * p.n_my_batches_work, dtype=torch.float64, device="cuda")

    def fused_step():
        w.plan.execute_fused_bias(1, p.n_atoms, 1, 1, av, w.P1, w.wave, w.gwave, w.P1, w.bias, w.gbias, w.rho, w.grad,
                                  stream=stream)

    def two_launch_step():
        w.plan.bias_part2(1, p.n_atoms, 1, 1, 1, av, w.wave, w.gwave, w.P1, bias1, stream=stream)
        w.step(_lib.RHO1_FP64, stream)

    ms_fused = time_device_steps(fused_step, args.steps, args.warmup, ranks, stream)
    ms_two = time_device_steps(two_launch_step, args.steps, args.warmup, ranks, stream)
    out["rho1_fused_bias_1_atom"] = {"ms_fused": ms_fused, "ms_two_launches": ms_two,
                                     "device_flags": w.plan.device_flags(),
                                     "note": "fused: FP64 rho1 + density-matrix bias in one launch; two launches: "
                                             "bias producer then FP64 rho1 (P1 stands in for the density matrix)"}
    del bias1
    out["bias_part2_4_atoms"] = {"ms_per_call": ms_bias, "pts_per_s": total_pts / (ms_bias / 1e3),
                                 "device_flags": w.plan.device_flags()}
    del av, bias4

    # config 5: the adjoints and the first-order H (small; timed beside the headline)
    if not args.no_config5:
        out["config5"] = time_config5(args.steps, args.warmup, ranks, stream, fp64_peak, fma_peak)

    # end to end through the reference-named session entry point
    e2e = None
    if not args.no_e2e:
        ms_e2e, h2d, d2h, finite = time_e2e(w, mode, max(3, args.steps // 2), args.warmup, ranks)
        e2e = {"value": total_pts / (ms_e2e / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e,
               "call": "evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_cu_host_ (pinned host P1, biases, "
                       "outputs; phi resident)", "outputs_finite": finite}
        if mode != _lib.RHO1_SPLIT_I8:  # the same call with the drop-ins switched to split-int8
            ms8, h2d8, d2h8, finite8 = time_e2e(w, _lib.RHO1_SPLIT_I8, max(3, args.steps // 2), args.warmup, ranks)
            out["e2e_split_i8"] = {"value": total_pts / (ms8 / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d8,
                                   "d2h_bytes_per_step": d2h8, "ms_per_step": ms8,
                                   "call": "same entry point after frpa_set_rho1_mode(FRPA_RHO1_SPLIT_I8)",
                                   "outputs_finite": finite8}

    # CPU baseline on rank 0 at N = 1: the reference's CPU code, same batches
    cpu = None
    if not args.no_cpu_baseline and ranks.world == 1:
        import oracle
        from fast_rpa_eval_b200 import synth

        if oracle.ref_available(1):
            nb = cpu_sample_batches(p, host_threads())
            wl = int(p.i_batch_2_wave_offset[nb])
            sample = synth.subset_batches(p, nb, w.wave[:wl].cpu().numpy(), w.gwave[:3 * wl].cpu().numpy())
            rate, cores, passes, secs = cpu_rho1_rate(sample, args.cpu_seconds)
            cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference",
                   "sample": f"first {nb} of {p.n_my_batches_work} config-2 batches ({sample.total_points()} points), "
                             f"{passes} passes in {secs:.1f} s"}
            # parity guard: the GPU's answer on the same batches
            r_ref, g_ref = oracle.rho1_reference_threaded(sample, host_threads())
            q = _lib.Rho1Plan(sample)
            rho_s = torch.zeros(sample.n_full_points, dtype=torch.float64, device="cuda")
            grad_s = torch.zeros(3 * sample.n_max_batch_size * nb, dtype=torch.float64, device="cuda")
            q.execute(1, w.wave, w.gwave, w.P1, _dev(sample.first_order_rho_bias_part2),
                      _dev(sample.first_order_gradient_rho_bias), rho_s, grad_s, mode=mode, stream=stream)
            torch.cuda.synchronize()
            err = float(np.max(np.abs(rho_s.cpu().numpy() - r_ref[:, 0])) / np.max(np.abs(r_ref)))
            errg = float(np.max(np.abs(grad_s.cpu().numpy() - g_ref.ravel(order="F"))) / np.max(np.abs(g_ref)))
            out["parity_vs_reference_on_sample"] = {"rho1_normwise_rel": err, "grad_normwise_rel": errg}

    # sum-up (config 3), per l_max
    sumup = {}
    if not args.no_sumup:
        del w
        torch.cuda.empty_cache()
        for L in [int(x) for x in args.sumup_lmax.split(",") if x]:
            sp, ms_s, fast = time_sumup(L, args.sumup_points, 4 + 7919 * ranks.rank, args.steps, args.warmup, ranks,
                                        stream)
            pairs = sp.pair_count()
            flops = 2.0 * (L + 1) ** 2 * pairs
            ent = {"pts_per_s": ranks.sum(sp.n_valid_points) / (ms_s / 1e3), "ms_per_call": ms_s,
                   "pairs_per_s": ranks.sum(pairs) / (ms_s / 1e3), "fast_path": fast,
                   "tflops_convention_2L2": flops / (ms_s / 1e3) / 1e12,
                   "frac_of_measured_fp64_fma": flops / (ms_s / 1e3) / 1e12 / fma_peak,
                   "hbm_gbs_algorithmic": (32.0 * sp.n_valid_points + 8.0 * ((L + 1) ** 2 + 4) * sp.n_atoms)
                   / (ms_s / 1e3) / 1e9}
            if ranks.world == 1 and not args.no_cpu_baseline and L <= 6:
                import oracle

                if oracle.ref_available(1):
                    rate, cores, secs = cpu_sumup_rate(L, 40_000, args.cpu_seconds)
                    ent["cpu_reference_pts_per_s"] = rate
                    ent["cpu_reference_cores"] = cores
            sumup[f"l{L}"] = ent
            del sp
    out["sumup_config3"] = sumup

    # config 4: the config-1 recipe swept to thousands of atoms (chunked, one
    # graph-captured autotuned launch per chunk and path)
    if not args.no_config4:
        from fast_rpa_eval_b200 import sweep

        w = None  # (the sum-up section may have released it already)
        torch.cuda.empty_cache()
        out["config4_sweep"] = [sweep.run_sweep(int(n), seed=4 + 7919 * ranks.rank, tune=not args.no_tune)
                                for n in args.config4_sizes.split(",") if n.strip()]

    if mode == _lib.RHO1_FP64:
        roofline = {"bound": "tensor", "achieved": achieved_tf, "peak": fp64_peak, "unit": "TFLOP/s",
                    "frac": achieved_tf / fp64_peak, "traffic": profile_traffic("rho1_fp64_kernel", p.n_my_batches_work),
                    "kernel": "rho1_fp64_kernel",
                    "peak_source": "measured on this GPU in this run: FP64 m8n8k4 MMA throughput probe "
                                   "(no FP64 figure in MEASURED_PEAKS.json)",
                    "algorithmic_flops_per_launch": w_flops,
                    "hbm_frac_of_measured": (w_bytes / (ms_fp64 / 1e3) / 1e9) / peaks["hbm_gbs"]}
    elif mode == _lib.RHO1_SPLIT_I8:
        traffic = profile_traffic("rho1_split_i8_step", p.n_my_batches_work)
        gbs = w_bytes / (ms / 1e3) / 1e9
        roofline = {"bound": "hbm", "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": gbs / peaks["hbm_gbs"], "traffic": traffic,
                    "kernel": "split-int8 step (i8_pack_a_kernel, i8_pack_b_kernel, rho1_i8_kernel per group)",
                    "achieved_from": "algorithmic bytes of the step (phi, grad phi, P1c once per batch, outputs) "
                                     "over the CUDA-event time",
                    "peak_source": peaks["source"] + " (MEASURED_PEAKS.json hbm_gbs)",
                    "algorithmic_bytes_per_launch": w_bytes,
                    "achieved_dram_frac": (traffic / (ms / 1e3) / 1e9 / peaks["hbm_gbs"]) if traffic else None}
    else:
        gbs = w_bytes / (ms / 1e3) / 1e9
        roofline = {"bound": "hbm", "achieved": gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": gbs / peaks["hbm_gbs"], "traffic": profile_traffic("rho1_split_kernel", p.n_my_batches_work),
                    "kernel": "rho1_split_kernel", "peak_source": peaks["source"] + " (MEASURED_PEAKS.json hbm_gbs)",
                    "algorithmic_bytes_per_launch": w_bytes,
                    "bf16_equivalent_tflops": 15 * w_flops / (ms / 1e3) / 1e12,
                    "bf16_frac_of_measured": 15 * w_flops / (ms / 1e3) / 1e12 / peaks["bf16_tflops"]}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": args.scaling,
        "vs_baseline": None,
        "dtype": {_lib.RHO1_FP64: "f64",
                  _lib.RHO1_SPLIT_BF16: "f64 in/out, bf16x5 slices -> f32 (tcgen05) contraction",
                  _lib.RHO1_SPLIT_I8: "f64 in/out, int8x5 digit planes -> exact int32 level sums (tcgen05 kind::i8) "
                                      "contraction, f64 recombination and ddots"}[mode],
        "data": "synthetic (seeded config-2 recipe: Gaussian x Y_lm basis, phi generated on the GPU)",
        "config": {"workload": "config2: rho1 + grad rho1, 1000 atoms at 0.1/A^3, 10 functions/atom, "
                               f"{p.n_my_batches_work} batches of 100-300 points, n_compute 100-600, T=1",
                   "path": mode_name, "valid_batches": info["n_valid_batches"], "work_items": n_items_tuned,
                   "launch": ("one persistent grouped launch per step, replayed from a CUDA graph"
                              if mode != _lib.RHO1_SPLIT_I8 else
                              f"row max + {i8_groups} groups x (pack phi, pack P1c, contraction), "
                              "replayed from a CUDA graph"),
                   "tuning": tuned or "defaults (--no-tune)",
                   "grid_points_per_rank": w_points,
                   "l2": "inputs larger than L2 (phi + grad phi = %.1f GB per rank)" % (4 * 8 * p.wave_len / 1e9),
                   "parallelism": (f"weak, {args.gpus} independent config-2 problems" if args.scaling == "weak" else
                                   f"strong, one config-2 problem, batches sharded by cost over {args.gpus} ranks "
                                   "(no collective on the forward path)")},
        "roofline": roofline,
        "clocks": clk,
        "gpu_launches": args.steps * {_lib.RHO1_FP64: 1, _lib.RHO1_SPLIT_BF16: 2,
                                      _lib.RHO1_SPLIT_I8: 1 + 3 * i8_groups}[mode],
        "cpu_baseline": cpu,
        "e2e": e2e,
        "measured_fp64_tflops": {"mma": fp64_peak, "fma": fma_peak},
    }
    line.update(out)
    return line


def main():
    args = parse_args()
    ranks = Ranks()
    if args.impl == "reference":
        ranks.init(use_gpu=False)
        res = run_reference(args, ranks)
        if ranks.rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
        ranks.close()
        return
    ranks.init(use_gpu=True)
    res = run_frpa(args, ranks)
    if ranks.rank == 0:
        print(json.dumps(res), flush=True)
    ranks.close()


if __name__ == "__main__":
    main()
