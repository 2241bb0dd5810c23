"""rho1 at the largest supported n_compute: 2048 for the plain FP64 path
(FRPA_MAX_N_COMPUTE) and 1024 for split-BF16 (the bound under which its exact
FP32 levels stay exact); one past the split bound is refused before any
launch.  Against the oracle, tolerances as in the other rho1 tests."""

import numpy as np
import pytest

import oracle
from fast_rpa_eval_b200 import _lib, synth

from gpu_util import normwise_rel, rho1_device_run


def _wide(nc, n_atoms, seed):
    return synth.make_rho1_problem(n_atoms=n_atoms, seed=seed, box=None, density=0.1, n_batches=4,
                                   np_range=(20, 70), nc_range=(nc, nc), with_bias=True, pad_value=np.nan,
                                   exact_selection=False)


@pytest.mark.gpu
def test_fp64_at_n_compute_2048():
    p = _wide(2048, 130, seed=21)
    assert int(p.n_compute_c_batches.max()) == 2048
    r, g = rho1_device_run(_lib.Rho1Plan(p), p, mode=_lib.RHO1_FP64)
    r_o, g_o = oracle.rho1(p)
    assert normwise_rel(r, r_o) < 1e-12 and normwise_rel(g, g_o) < 1e-12


@pytest.mark.gpu
def test_split_at_n_compute_1024():
    p = _wide(1024, 60, seed=22)
    assert int(p.n_compute_c_batches.max()) == 1024
    plan = _lib.Rho1Plan(p)
    r, g = rho1_device_run(plan, p, mode=_lib.RHO1_SPLIT_BF16)
    r_o, g_o = oracle.rho1(p)
    assert normwise_rel(r, r_o) < 1e-10 and normwise_rel(g, g_o) < 1e-10
    assert plan.device_flags() == 0


@pytest.mark.gpu
def test_split_refuses_n_compute_1025():
    p = _wide(1025, 60, seed=23)
    plan = _lib.Rho1Plan(p)
    with pytest.raises(_lib.FrpaError) as e:
        rho1_device_run(plan, p, mode=_lib.RHO1_SPLIT_BF16)
    assert e.value.status == _lib.FRPA_ERR_UNSUPPORTED
