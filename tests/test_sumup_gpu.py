"""Hartree sum-up on the GPU against the oracle: values within FP64 tolerance
and every branch decision (near / far / skipped, l_atom_max) bit-identical."""
import numpy as np
import pytest
import torch

import oracle
from fast_rpa_eval_b200 import _lib, synth
from gpu_util import dev, host, normwise_rel

pytestmark = pytest.mark.gpu
TOL = 1e-12


def run(plan, p, generic=False, codes=False):
    dv = dev(p.delta_v_hartree)
    c = torch.zeros(p.n_valid_points * p.n_centers_hartree_potential * p.T, dtype=torch.uint8, device="cuda") if codes else None
    plan.execute(p.j_atom_end - p.j_atom_begin + 1, dev(p.l_hartree_max_far_distance, np.int32),
                 dev(p.multipole_radius_sq), dev(p.outer_potential_radius), dev(p.multipole_moments), dev(p.spline),
                 dv, branch_codes=c, force_generic=generic)
    torch.cuda.synchronize()
    out = host(dv, (p.n_full_points, p.T))
    if codes:
        return out, host(c, (p.n_valid_points, p.n_centers_hartree_potential, p.T))
    return out


def delta_rel(out, ref, d0):
    return normwise_rel(out - d0, ref - d0)


@pytest.mark.parametrize("L,T,lh", [(4, 1, None), (6, 1, None), (6, 2, [6, 4, 2, 0]), (8, 1, [8, 7, 5, 3]), (8, 2, None)])
def test_sumup_fast_matches_oracle(L, T, lh):
    p = synth.make_sumup_problem(n_atoms=24, n_points=6000, l_pot_max=L, T=T, seed=50 + L + T,
                                 l_hartree_per_species=lh, extra_full_points=64)
    plan = _lib.SumupPlan(p)
    assert plan.fast
    out, codes = run(plan, p, codes=True)
    ref, rcodes = oracle.sumup(p, branch_codes=True)
    assert np.array_equal(codes, rcodes)
    assert delta_rel(out, ref, p.delta_v_hartree) < TOL
    # untouched full points keep their input value exactly
    untouched = np.setdiff1d(np.arange(p.n_full_points), p.i_valid_point_2_i_full_points_map)
    assert np.array_equal(out[untouched], p.delta_v_hartree[untouched])


@pytest.mark.parametrize("centers", ["identity", "permuted"])
def test_sumup_generic_matches_oracle(centers):
    p = synth.make_sumup_problem(n_atoms=20, n_points=3000, l_pot_max=6, T=2, seed=61, centers=centers,
                                 l_hartree_per_species=[6, 5, 3, 6])
    plan = _lib.SumupPlan(p)
    assert plan.fast == (centers == "identity")
    out, codes = run(plan, p, generic=True, codes=True)
    ref, rcodes = oracle.sumup(p, branch_codes=True)
    assert np.array_equal(codes, rcodes)
    assert delta_rel(out, ref, p.delta_v_hartree) < TOL


@pytest.mark.skipif(not oracle.ref_available(1), reason="reference library not built")
def test_sumup_matches_reference_cpu_code():
    p = synth.make_sumup_problem(n_atoms=30, n_points=8000, l_pot_max=6, T=1, seed=71, l_hartree_per_species=[6, 6, 4, 2])
    out = run(_lib.SumupPlan(p), p)
    ref = oracle.sumup(p, use_reference=True)
    assert delta_rel(out, ref, p.delta_v_hartree) < TOL


def test_sumup_config3_shape_far_field_only():
    # the benchmark recipe at reduced size: no l truncation, near field rare
    p = synth.config3(l_max=8, n_atoms=60, n_points=20000, seed=5)
    out = run(_lib.SumupPlan(p), p)
    ref = oracle.sumup(p, n_threads=8)
    assert delta_rel(out, ref, p.delta_v_hartree) < TOL


def test_sumup_dropin_symbol_matches_oracle():
    p = synth.make_sumup_problem(n_atoms=16, n_points=2000, l_pot_max=6, T=2, seed=81)
    out = _lib.dropin_sumup(p)
    ref = oracle.sumup(p)
    assert delta_rel(out, ref, p.delta_v_hartree) < TOL


def test_sumup_session_cu_host_matches_oracle():
    r = synth.make_rho1_problem(T=1, seed=3, n_batches=8)
    p = synth.make_sumup_problem(n_atoms=16, n_points=1500, l_pot_max=6, T=1, seed=82)
    # share the full-point count (the session holds both paths)
    p.n_full_points = r.n_full_points = max(r.n_full_points, p.n_full_points)
    pad = p.n_full_points - p.coord_points.shape[1]
    p.coord_points = np.asfortranarray(np.concatenate([p.coord_points, np.zeros((3, pad))], axis=1))
    p.delta_v_hartree = np.asfortranarray(np.concatenate([p.delta_v_hartree, np.zeros((pad, 1))], axis=0))
    p.partition_tab = np.concatenate([p.partition_tab, np.ones(pad)])
    r.partition_tab = p.partition_tab
    r.i_valid_point_2_i_full_points_map = np.concatenate(
        [r.i_valid_point_2_i_full_points_map, np.arange(len(r.i_valid_point_2_i_full_points_map), p.n_full_points)]).astype(np.int32)
    with _lib.Session(r, p) as s:
        out = s.sumup()
        ref = oracle.sumup(p)
        assert delta_rel(out, ref, p.delta_v_hartree) < TOL
        out2 = s.sumup(delta_v=out)
        ref2 = oracle.sumup(p, delta_v=ref)
        assert delta_rel(out2, ref2, p.delta_v_hartree) < TOL
