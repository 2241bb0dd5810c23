"""Config-4 sweep driver: the config-1 recipe at thousands of atoms, processed
as spatially ordered chunks of batches.  Each chunk runs over its own basis
window U (the union of its batches' compute functions) with a dense window of
one global synthetic P1 (frpa_synth_p1_window), as one persistent grouped
launch per path, captured in a CUDA graph, with tile shapes from the
autotuner.  Reports grid points/s of the FP64 and split-BF16 paths and their
mutual error; phi / grad phi come from the device generator."""

from __future__ import annotations

import time

import numpy as np

from . import _lib, autotune, synth


class ChunkRun:
    """Device inputs and plan of one chunk."""

    def __init__(self, geom, b0: int, b1: int, p1_seed: int):
        import torch

        self.prob, U = synth.sweep_chunk_problem(geom, b0, b1)
        p = self.prob
        pts = torch.from_numpy(np.ascontiguousarray(p.valid_points_xyz.T.ravel(order="F"))).cuda()
        self.wave = torch.empty(p.wave_len, dtype=torch.float64, device="cuda")
        self.gwave = torch.empty(3 * p.wave_len, dtype=torch.float64, device="cuda")
        _lib.synth_basis_values(p, pts, self.wave, self.gwave, pad_value=0.0)
        del pts
        self.U = torch.from_numpy(U).cuda()
        n = len(U)
        self.P1 = torch.empty(n * n, dtype=torch.float64, device="cuda")
        scale = 1.0 / np.sqrt(max(1.0, float(np.mean(p.n_compute_c_batches))))
        _lib.synth_p1_window(self.U, n, 1, scale, p1_seed, self.P1)
        nmb, nb = p.n_max_batch_size, p.n_my_batches_work
        self.bias = torch.zeros(nmb * nb, dtype=torch.float64, device="cuda")
        self.gbias = torch.zeros(3 * nmb * nb, dtype=torch.float64, device="cuda")
        self.rho = torch.zeros(p.n_full_points, dtype=torch.float64, device="cuda")
        self.grad = torch.zeros(3 * nmb * nb, dtype=torch.float64, device="cuda")
        self.plan = _lib.Rho1Plan(p)

    def step(self, mode: int):
        self.plan.execute(1, self.wave, self.gwave, self.P1, self.bias, self.gbias, self.rho, self.grad, mode=mode)

    def host_problem(self):
        """The chunk with its device phi / grad phi / P1 window on the host (for
        the oracle)."""
        import dataclasses

        n = self.prob.n_basis
        return dataclasses.replace(
            self.prob, wave=self.wave.cpu().numpy(), gradient_wave=self.gwave.cpu().numpy(),
            first_order_density_matrix=self.P1.cpu().numpy().reshape((n, n, 1), order="F"))


def run_sweep(n_atoms: int, seed: int = 4, reps: int = 3, max_batches: int = 5000, max_window: int = 24000,
              tune: bool = True, p1_seed: int = 12345) -> dict:
    import torch

    t0 = time.time()
    geom = synth.config4_geometry(n_atoms, seed=seed)
    chunks = synth.sweep_chunks(geom, max_batches=max_batches, max_window=max_window)
    t_geom = time.time() - t0
    ms = {_lib.RHO1_FP64: 0.0, _lib.RHO1_SPLIT_BF16: 0.0, _lib.RHO1_SPLIT_I8: 0.0}
    pts = 0
    err = {m: {"rho1": 0.0, "grad_rho1": 0.0} for m in (_lib.RHO1_SPLIT_BF16, _lib.RHO1_SPLIT_I8)}
    choice = {}
    windows = []
    flags = 0
    for ci, (b0, b1) in enumerate(chunks):
        c = ChunkRun(geom, b0, b1, p1_seed)
        windows.append(c.prob.n_basis)
        if tune and ci == 0:
            for m in (_lib.RHO1_FP64, _lib.RHO1_SPLIT_BF16):
                choice.update(autotune.tune_rho1(c.plan, c.prob, lambda m=m: c.step(m), m, reps=1)["choice"])
        elif choice:
            c.plan.set_tuning(**choice)
        out = {}
        for m in ms:
            g = _lib.capture_graph(lambda m=m: c.step(m))
            g.replay()
            torch.cuda.synchronize()
            out[m] = (c.rho.clone(), c.grad.clone())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                g.replay()
            e1.record()
            torch.cuda.synchronize()
            ms[m] += e0.elapsed_time(e1) / reps
            del g
        rf, gf = out[_lib.RHO1_FP64]
        for m, e in err.items():
            rs, gs = out[m]
            e["rho1"] = max(e["rho1"], float((rs - rf).abs().max() / rf.abs().max()))
            e["grad_rho1"] = max(e["grad_rho1"], float((gs - gf).abs().max() / gf.abs().max()))
        flags |= c.plan.device_flags()
        pts += c.prob.total_points()
        del c, out
        torch.cuda.empty_cache()
    return {
        "n_atoms": n_atoms, "n_batches": geom.n_batches, "grid_points": int(pts), "chunks": len(chunks),
        "max_window_functions": int(max(windows)), "tuning": choice or "defaults",
        "fp64": {"ms": ms[_lib.RHO1_FP64], "pts_per_s": pts / (ms[_lib.RHO1_FP64] / 1e3)},
        "split_bf16": {"ms": ms[_lib.RHO1_SPLIT_BF16], "pts_per_s": pts / (ms[_lib.RHO1_SPLIT_BF16] / 1e3)},
        "split_i8": {"ms": ms[_lib.RHO1_SPLIT_I8], "pts_per_s": pts / (ms[_lib.RHO1_SPLIT_I8] / 1e3)},
        "split_vs_fp64_normwise_rel_max_over_chunks": err[_lib.RHO1_SPLIT_BF16],
        "split_i8_vs_fp64_normwise_rel_max_over_chunks": err[_lib.RHO1_SPLIT_I8], "device_flags": flags,
        "host_geometry_s": t_geom}
