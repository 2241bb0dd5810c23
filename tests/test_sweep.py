"""Config-4 sweep: chunking and basis windows on CPU; on the GPU a chunk
through both rho1 paths against the oracle (with the device-generated phi and
P1 window copied back), agreement of P1 windows on shared functions, and a
small end-to-end sweep."""

import numpy as np
import pytest

import oracle
from fast_rpa_eval_b200 import _lib, synth


def _geom():
    return synth.config4_geometry(40, seed=6)


def test_chunks_cover_batches_and_respect_the_window():
    g = _geom()
    chunks = synth.sweep_chunks(g, max_batches=60, max_window=500)
    assert chunks[0][0] == 0 and chunks[-1][1] == g.n_batches
    assert all(a[1] == b[0] for a, b in zip(chunks, chunks[1:]))
    for b0, b1 in chunks:
        window = set().union(*[g.ib[b].tolist() for b in range(b0, b1)])
        assert len(window) <= 500 or b1 - b0 == 1


def test_chunk_problem_maps_back_to_the_global_functions():
    g = _geom()
    b0, b1 = synth.sweep_chunks(g, max_batches=60, max_window=500)[1]
    p, U = synth.sweep_chunk_problem(g, b0, b1)
    for k, b in enumerate(range(b0, b1)):
        nc = p.n_compute_c_batches[k]
        assert np.array_equal(U[p.i_basis_batches[:nc, k] - 1], g.ib[b])
    assert p.n_basis == len(U) and np.all(np.diff(U) > 0)
    assert np.array_equal(p.atoms_xyz[p.basis.atom], g.atoms[g.basis.atom[U]])


@pytest.mark.gpu
@pytest.mark.parametrize("mode,tol", [(_lib.RHO1_FP64, 1e-12), (_lib.RHO1_SPLIT_BF16, 1e-10),
                                      (_lib.RHO1_SPLIT_I8, 1e-10)])
def test_chunk_matches_oracle(mode, tol):
    import torch

    from fast_rpa_eval_b200 import sweep
    from gpu_util import normwise_rel

    g = _geom()
    chunks = synth.sweep_chunks(g, max_batches=60, max_window=500)
    c = sweep.ChunkRun(g, *chunks[0], p1_seed=7)
    c.step(mode)
    torch.cuda.synchronize()
    hp = c.host_problem()
    r_o, g_o = oracle.rho1(hp)
    r = c.rho.cpu().numpy().reshape(r_o.shape, order="F")
    gr = c.grad.cpu().numpy().reshape(g_o.shape, order="F")
    assert normwise_rel(r, r_o) < tol and normwise_rel(gr, g_o) < tol
    assert c.plan.device_flags() == 0


@pytest.mark.gpu
def test_p1_windows_agree_on_shared_functions():
    import torch

    n_all = 60
    U1 = torch.arange(0, 40, dtype=torch.int32, device="cuda")
    U2 = torch.arange(20, n_all, dtype=torch.int32, device="cuda")
    a = torch.empty(40 * 40, dtype=torch.float64, device="cuda")
    b = torch.empty(40 * 40, dtype=torch.float64, device="cuda")
    _lib.synth_p1_window(U1, 40, 1, 0.5, 99, a)
    _lib.synth_p1_window(U2, 40, 1, 0.5, 99, b)
    A = a.cpu().numpy().reshape(40, 40, order="F")
    B = b.cpu().numpy().reshape(40, 40, order="F")
    assert np.array_equal(A, A.T)
    assert np.array_equal(A[20:40, 20:40], B[0:20, 0:20])
    assert 0.3 < A.std() < 0.7


@pytest.mark.gpu
def test_small_sweep_end_to_end():
    from fast_rpa_eval_b200 import sweep

    res = sweep.run_sweep(30, reps=1, max_batches=80, max_window=500)
    assert res["chunks"] >= 2 and res["grid_points"] > 0 and res["device_flags"] == 0
    assert res["split_vs_fp64_normwise_rel_max_over_chunks"]["rho1"] < 1e-10
    assert res["split_i8_vs_fp64_normwise_rel_max_over_chunks"]["rho1"] < 1e-10
