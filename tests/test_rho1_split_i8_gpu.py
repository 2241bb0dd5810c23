"""Split-int8 rho1 (five signed 8-bit digits per operand, tcgen05 kind::i8,
exact int32 level sums, FP64 epilogue) against the oracle.  Stated tolerance:
1e-10 normwise relative, for rho1 and grad rho1 separately."""
import numpy as np
import pytest

import oracle
from fast_rpa_eval_b200 import _lib, synth
from gpu_util import normwise_rel, rho1_device_run

pytestmark = pytest.mark.gpu
TOL_SPLIT = 1e-10


def run_i8(p, scratch_mb=None):
    plan = _lib.Rho1Plan(p)
    if scratch_mb is not None:
        plan.set_tuning(split_i8_scratch_mb=scratch_mb)
    out = rho1_device_run(plan, p, mode=_lib.RHO1_SPLIT_I8)
    assert plan.device_flags() == 0
    return out


def test_i8_small_config1():
    p = synth.config1(seed=1, n_batches=8)
    r, g = run_i8(p)
    r_o, g_o = oracle.rho1(p)
    assert normwise_rel(r, r_o) < TOL_SPLIT, normwise_rel(r, r_o)
    assert normwise_rel(g, g_o) < TOL_SPLIT, normwise_rel(g, g_o)


@pytest.mark.parametrize("T,n_active", [(1, 1), (2, 1), (3, 3)])
def test_i8_matches_oracle_edge_cases(T, n_active):
    p = synth.make_rho1_problem(T=T, seed=40 + T, with_bias=True, extra_full_points=21, empty_batches=3,
                                pad_value=np.nan, n_active=n_active)
    r, g = run_i8(p)
    r_o, g_o = oracle.rho1(p)
    assert not np.isnan(r).any() and not np.isnan(g).any()
    assert normwise_rel(r, r_o) < TOL_SPLIT and normwise_rel(g, g_o) < TOL_SPLIT
    assert np.array_equal(r_o == 0, r == 0)


def test_i8_config2_recipe_uneven_batches():
    p = synth.make_rho1_problem(n_atoms=120, shells="sssf", box=None, density=0.1, n_batches=150,
                                np_range=(100, 300), nc_range=(100, 600), p1_pattern="active",
                                exact_selection=False, seed=12, pad_value=np.nan)
    r, g = run_i8(p)
    r_o, g_o = oracle.rho1(p, n_threads=8)
    assert normwise_rel(r, r_o) < TOL_SPLIT and normwise_rel(g, g_o) < TOL_SPLIT


def test_i8_groups_give_identical_results():
    """A 1 MiB scratch budget packs and contracts the batches in many groups;
    the results are bit-identical to one group."""
    p = synth.make_rho1_problem(n_atoms=60, shells="sssf", box=None, density=0.1, n_batches=40,
                                np_range=(20, 300), nc_range=(16, 400), exact_selection=False, seed=13,
                                with_bias=True, T=2)
    a = run_i8(p)
    b = run_i8(p, scratch_mb=1)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    r_o, g_o = oracle.rho1(p)
    assert normwise_rel(a[0], r_o) < TOL_SPLIT and normwise_rel(a[1], g_o) < TOL_SPLIT


def test_i8_at_n_compute_2048():
    """No FP32 exactness bound: the int32 levels are exact up to K = 26,000,
    so the split-int8 mode covers n_compute up to FRPA_MAX_N_COMPUTE."""
    p = synth.make_rho1_problem(n_atoms=130, seed=21, box=None, density=0.1, n_batches=4, np_range=(20, 70),
                                nc_range=(2048, 2048), with_bias=True, pad_value=np.nan, exact_selection=False)
    assert int(p.n_compute_c_batches.max()) == 2048
    r, g = run_i8(p)
    r_o, g_o = oracle.rho1(p)
    assert normwise_rel(r, r_o) < TOL_SPLIT and normwise_rel(g, g_o) < TOL_SPLIT


def test_i8_deterministic_and_scaled_inputs():
    p = synth.config1(seed=2, n_batches=12, with_bias=True)
    a = run_i8(p)
    b = run_i8(p)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    # rows of very different magnitude: per-point and per-row scales
    p.wave[:] *= 1e-7
    p.gradient_wave[:] *= 1e-7
    p.first_order_density_matrix[:] *= 1e5
    r, g = run_i8(p)
    r_o, g_o = oracle.rho1(p)
    assert normwise_rel(r, r_o) < TOL_SPLIT and normwise_rel(g, g_o) < TOL_SPLIT


@pytest.mark.parametrize("via", ["dropin", "session"])
def test_i8_through_the_reference_entry_points(via):
    """frpa_set_rho1_mode(FRPA_RHO1_SPLIT_I8) switches the reference-named
    entry points (the host drop-in and the session's cu_host twin) to this
    mode; two calls in a row, P1 changed in between."""
    p = synth.make_rho1_problem(T=2, seed=43, with_bias=True, extra_full_points=5, empty_batches=2)
    _lib.set_rho1_mode(_lib.RHO1_SPLIT_I8)
    try:
        if via == "dropin":
            outs = []
            for rep in range(2):
                q = synth.make_rho1_problem(T=2, seed=43, with_bias=True, extra_full_points=5, empty_batches=2)
                q.first_order_density_matrix = np.asfortranarray(q.first_order_density_matrix * (1.0 + rep))
                outs.append((q, _lib.dropin_rho1(q)))
        else:
            outs = []
            with _lib.Session(p) as s:
                for rep in range(2):
                    q = synth.make_rho1_problem(T=2, seed=43, with_bias=True, extra_full_points=5, empty_batches=2)
                    q.first_order_density_matrix = np.asfortranarray(p.first_order_density_matrix * (1.0 + rep))
                    outs.append((q, s.rho1(P1=q.first_order_density_matrix)))
    finally:
        _lib.set_rho1_mode(_lib.RHO1_FP64)
    for q, (r, g) in outs:
        r_o, g_o = oracle.rho1(q)
        assert normwise_rel(r.reshape(r_o.shape, order="F"), r_o) < TOL_SPLIT
        assert normwise_rel(g.reshape(g_o.shape, order="F"), g_o) < TOL_SPLIT
