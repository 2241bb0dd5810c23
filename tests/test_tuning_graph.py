"""Tunings, the autotuner and CUDA-graph replay of the rho1 plans.

* every tile shape / schedule gives bit-identical rho1 and grad rho1 (the
  tunings only re-cut the work list), FP64 and split-BF16;
* the autotuner leaves a candidate of its space applied and caches it;
* a captured CUDA graph of a plan's launches replays to the same results as
  direct execution, also after the inputs change in place.
"""

import json

import numpy as np
import pytest

import oracle
from fast_rpa_eval_b200 import _lib, autotune, synth


def test_autotune_space_and_key():
    p = synth.config1(seed=2)
    k1 = autotune.geometry_key(p, _lib.RHO1_FP64, "gpu")
    k2 = autotune.geometry_key(p, _lib.RHO1_SPLIT_BF16, "gpu")
    assert k1 != k2 and k1 == autotune.geometry_key(p, _lib.RHO1_FP64, "gpu")
    for mode in (_lib.RHO1_FP64, _lib.RHO1_SPLIT_BF16):
        assert all(set(c) <= set(_lib.TUNINGS) for c in autotune.space(mode))


def _setup(seed=3):
    import torch

    from gpu_util import dev

    p = synth.config2(seed=seed, n_batches=120, eval_phi=True)
    args = dict(wave=dev(p.wave), gwave=dev(p.gradient_wave), P1=dev(p.first_order_density_matrix),
                bias=dev(p.first_order_rho_bias_part2), gbias=dev(p.first_order_gradient_rho_bias),
                rho=torch.zeros(p.n_full_points * p.T, dtype=torch.float64, device="cuda"),
                grad=torch.zeros(3 * p.n_max_batch_size * p.n_my_batches_work * p.T, dtype=torch.float64,
                                 device="cuda"))
    return p, args


def _run(plan, p, a, mode):
    plan.execute(p.j_atom_end - p.j_atom_begin + 1, a["wave"], a["gwave"], a["P1"], a["bias"], a["gbias"],
                 a["rho"], a["grad"], mode=mode)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [_lib.RHO1_FP64, _lib.RHO1_SPLIT_BF16])
def test_every_tuning_gives_identical_results(mode):
    import torch

    p, a = _setup()
    plan = _lib.Rho1Plan(p)
    _run(plan, p, a, mode)
    torch.cuda.synchronize()
    r0, g0 = a["rho"].clone(), a["grad"].clone()
    r_o, _ = oracle.rho1(p)
    tol = 1e-12 if mode == _lib.RHO1_FP64 else 1e-10
    ref = torch.from_numpy(r_o.ravel(order="F")).cuda()
    assert float((r0 - ref).abs().max() / ref.abs().max()) < tol
    for cand in autotune.space(mode):
        plan.set_tuning(**cand)
        assert all(plan.tuning()[k] == v for k, v in cand.items())
        _run(plan, p, a, mode)
        torch.cuda.synchronize()
        assert torch.equal(a["rho"], r0) and torch.equal(a["grad"], g0), cand
    assert plan.device_flags() == 0


@pytest.mark.gpu
def test_tuning_rejects_bad_values():
    p, _ = _setup()
    plan = _lib.Rho1Plan(p)
    for kw in ({"fp64_tile_points": 96}, {"fp64_ctas_per_sm": 4}, {"split_tile_points": 200}, {"order": 3}):
        with pytest.raises(_lib.FrpaError):
            plan.set_tuning(**kw)


@pytest.mark.gpu
def test_autotuner_picks_and_caches(tmp_path):
    p, a = _setup()
    plan = _lib.Rho1Plan(p)
    cache = str(tmp_path / "tune.json")
    res = autotune.tune_rho1(plan, p, lambda: _run(plan, p, a, _lib.RHO1_FP64), _lib.RHO1_FP64, reps=1,
                             cache_path=cache)
    assert not res["cached"] and res["choice"] in autotune.space(_lib.RHO1_FP64)
    assert all(plan.tuning()[k] == v for k, v in res["choice"].items())
    assert len(json.load(open(cache))) == 1
    plan2 = _lib.Rho1Plan(p)
    res2 = autotune.tune_rho1(plan2, p, lambda: _run(plan2, p, a, _lib.RHO1_FP64), _lib.RHO1_FP64,
                              cache_path=cache)
    assert res2["cached"] and res2["choice"] == res["choice"]


@pytest.mark.gpu
@pytest.mark.parametrize("mode,scratch_mb", [(_lib.RHO1_FP64, None), (_lib.RHO1_SPLIT_BF16, None),
                                             (_lib.RHO1_SPLIT_I8, None), (_lib.RHO1_SPLIT_I8, 1)])
def test_graph_replay_matches_direct_execution(mode, scratch_mb):
    """For split-int8 also with a 1 MiB scratch budget: several groups, packed
    on the plan's side stream (captured through event edges) into two
    alternating scratch sets."""
    import torch

    p, a = _setup(seed=5)
    plan = _lib.Rho1Plan(p)
    if scratch_mb is not None:
        plan.set_tuning(split_i8_scratch_mb=scratch_mb)
    g = _lib.capture_graph(lambda: _run(plan, p, a, mode))
    g.replay()
    torch.cuda.synchronize()
    r_graph, g_graph = a["rho"].clone(), a["grad"].clone()
    a["rho"].fill_(3.0)
    _run(plan, p, a, mode)
    torch.cuda.synchronize()
    assert torch.equal(a["rho"], r_graph) and torch.equal(a["grad"], g_graph)
    # new P1 values in the same buffer: the replay sees them
    a["P1"].mul_(-0.5)
    g.replay()
    torch.cuda.synchronize()
    r2 = a["rho"].clone()
    _run(plan, p, a, mode)
    torch.cuda.synchronize()
    assert torch.equal(a["rho"], r2) and not torch.equal(r2, r_graph)
    assert plan.device_flags() == 0
