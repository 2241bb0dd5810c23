"""Split-BF16 rho1 (tcgen05 tensor cores, FP32 accumulation, FP64 epilogue)
against the oracle.  Stated tolerance: 1e-10 normwise relative, for rho1 and
grad rho1 separately."""
import numpy as np
import pytest

import oracle
from fast_rpa_eval_b200 import _lib, synth
from gpu_util import normwise_rel, rho1_device_run

pytestmark = pytest.mark.gpu
TOL_SPLIT = 1e-10


def run_split(p):
    plan = _lib.Rho1Plan(p)
    out = rho1_device_run(plan, p, mode=_lib.RHO1_SPLIT_BF16)
    assert plan.device_flags() == 0
    return out


def test_split_small_config1():
    p = synth.config1(seed=1, n_batches=8)
    r, g = run_split(p)
    r_o, g_o = oracle.rho1(p)
    assert normwise_rel(r, r_o) < TOL_SPLIT, normwise_rel(r, r_o)
    assert normwise_rel(g, g_o) < TOL_SPLIT, normwise_rel(g, g_o)


@pytest.mark.parametrize("T,n_active", [(1, 1), (2, 1), (3, 3)])
def test_split_matches_oracle_edge_cases(T, n_active):
    p = synth.make_rho1_problem(T=T, seed=40 + T, with_bias=True, extra_full_points=21, empty_batches=3,
                                pad_value=np.nan, n_active=n_active)
    r, g = run_split(p)
    r_o, g_o = oracle.rho1(p)
    assert not np.isnan(r).any() and not np.isnan(g).any()
    assert normwise_rel(r, r_o) < TOL_SPLIT and normwise_rel(g, g_o) < TOL_SPLIT
    assert np.array_equal(r_o == 0, r == 0)


def test_split_config2_recipe_uneven_batches():
    p = synth.make_rho1_problem(n_atoms=120, shells="sssf", box=None, density=0.1, n_batches=150,
                                np_range=(100, 300), nc_range=(100, 600), p1_pattern="active",
                                exact_selection=False, seed=12, pad_value=np.nan)
    r, g = run_split(p)
    r_o, g_o = oracle.rho1(p, n_threads=8)
    assert normwise_rel(r, r_o) < TOL_SPLIT and normwise_rel(g, g_o) < TOL_SPLIT


def test_split_deterministic():
    p = synth.config1(seed=2, n_batches=12, with_bias=True)
    a = run_split(p)
    b = run_split(p)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
