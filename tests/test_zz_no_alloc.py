"""The allocation-free sum-up entry point (frpa_sumup_execute_noalloc), for
callers that cannot let the library allocate device memory, against the
plan-based entry point on the same inputs, over two calls in a row.

Collected last on purpose: if it fails, a run that stops at the first failure
has already run every other test."""
import ctypes

import numpy as np
import pytest
import torch

from fast_rpa_eval_b200 import _lib, synth
from gpu_util import dev, host, normwise_rel

pytestmark = pytest.mark.gpu
TOL = 1e-12  # normwise relative on the accumulated increment, as the other sum-up tests


def _noalloc(p, arrays, dv, stream=0):
    c = ctypes.c_int
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    a = arrays
    return _lib.lib().frpa_sumup_execute_noalloc(
        c(p.T), c(p.j_atom_begin), c(p.j_atom_end), c(p.n_full_points), c(p.l_max_analytic_multipole),
        c(p.index_cc_dim_0), c(p.n_valid_points), c(p.l_pot_max), c(p.n_hartree_grid), c(p.n_centers),
        c(p.n_centers_hartree_potential), c(p.n_atoms), c(p.hartree_force_l_add), c(p.n_species), P(a["species"]),
        P(a["species_center"]), P(a["lhmfd"]), P(a["map"]), P(a["coord"]), P(a["mrs"]), P(a["opr"]), P(a["Q"]),
        P(a["spline"]), P(a["l_hartree"]), P(a["n_grid"]), P(a["ncc"]), P(a["chp"]), P(a["c2a"]), P(a["icc"]),
        P(a["ijk"]), P(a["cc"]), P(a["cxyz"]), P(a["rgm"]), P(a["linc"]), P(dv), ctypes.c_void_p(stream))


def _device_arrays(p):
    i32 = np.int32
    return dict(species=dev(p.species, i32), species_center=dev(p.species_center, i32),
                lhmfd=dev(p.l_hartree_max_far_distance, i32), map=dev(p.i_valid_point_2_i_full_points_map, i32),
                coord=dev(p.coord_points), mrs=dev(p.multipole_radius_sq), opr=dev(p.outer_potential_radius),
                Q=dev(p.multipole_moments), spline=dev(p.spline), l_hartree=dev(p.l_hartree, i32),
                n_grid=dev(p.n_grid, i32), ncc=dev(p.n_cc_lm_ijk, i32), chp=dev(p.centers_hartree_potential, i32),
                c2a=dev(p.center_to_atom, i32), icc=dev(p.index_cc, i32), ijk=dev(p.index_ijk_max_cc, i32),
                cc=dev(p.cc), cxyz=dev(p.coords_center), rgm=dev(p.r_grid_min), linc=dev(p.log_r_grid_inc))


def test_noalloc_sumup_matches_plan_entry_point_twice():
    p = synth.make_sumup_problem(n_atoms=24, n_points=5000, l_pot_max=6, T=2, seed=91,
                                 l_hartree_per_species=[6, 5, 3, 6], extra_full_points=40)
    a = _device_arrays(p)
    plan = _lib.SumupPlan(p)
    dv_plan = dev(p.delta_v_hartree)
    dv_noalloc = dev(p.delta_v_hartree)
    d0 = p.delta_v_hartree.copy()
    shape = (p.n_full_points, p.T)
    for call in range(2):
        plan.execute(p.T, a["lhmfd"], a["mrs"], a["opr"], a["Q"], a["spline"], dv_plan)
        st = _noalloc(p, a, dv_noalloc)
        assert st == 0, _lib.last_error()
        torch.cuda.synchronize()
        ref = host(dv_plan, shape)
        got = host(dv_noalloc, shape)
        assert normwise_rel(got - d0, ref - d0) < TOL, call
    plan.close()


def test_noalloc_sumup_rejects_sizes_beyond_its_scratch():
    p = synth.make_sumup_problem(n_atoms=4, n_points=100, l_pot_max=4, T=1, seed=3)
    a = _device_arrays(p)
    big = synth.make_sumup_problem(n_atoms=4, n_points=100, l_pot_max=4, T=1, seed=3)
    big.n_atoms = 20_000  # index_cc_dim_0 x n_atoms x 8 bytes > 8 MiB
    dv = dev(p.delta_v_hartree)
    st = _noalloc(big, a, dv)
    assert st == _lib.FRPA_ERR_INVALID
    assert "scratch" in _lib.last_error()[1]


def _noalloc_flags():
    f = ctypes.c_int(-1)
    assert _lib.lib().frpa_sumup_noalloc_flags(ctypes.byref(f), ctypes.c_void_p(0)) == 0, _lib.last_error()
    return f.value


def test_noalloc_sumup_partial_atom_tile_matches_plan():
    # tile of 3 perturbations with only 2 active: columns t >= n_active stay untouched
    p = synth.make_sumup_problem(n_atoms=16, n_points=3000, l_pot_max=5, T=3, n_active=2, seed=17,
                                 extra_full_points=25)
    assert p.j_atom_end - p.j_atom_begin + 1 == 2
    a = _device_arrays(p)
    plan = _lib.SumupPlan(p)
    dv_plan, dv_noalloc = dev(p.delta_v_hartree), dev(p.delta_v_hartree)
    d0 = p.delta_v_hartree.copy()
    shape = (p.n_full_points, p.T)
    plan.execute(2, a["lhmfd"], a["mrs"], a["opr"], a["Q"], a["spline"], dv_plan)
    assert _noalloc(p, a, dv_noalloc) == 0, _lib.last_error()
    torch.cuda.synchronize()
    ref, got = host(dv_plan, shape), host(dv_noalloc, shape)
    assert normwise_rel(got[:, :2] - d0[:, :2], ref[:, :2] - d0[:, :2]) < TOL
    assert np.array_equal(got[:, 2], d0[:, 2])
    plan.close()


def test_noalloc_sumup_without_valid_points_leaves_output_unchanged():
    p = synth.make_sumup_problem(n_atoms=6, n_points=200, l_pot_max=4, T=1, seed=5)
    a = _device_arrays(p)
    dv = dev(p.delta_v_hartree)
    p.n_valid_points = 0
    assert _noalloc(p, a, dv) == 0, _lib.last_error()
    torch.cuda.synchronize()
    assert np.array_equal(host(dv, (p.n_full_points, p.T)), p.delta_v_hartree)


def test_noalloc_sumup_reports_clamped_far_distance_l():
    # an l_hartree_max_far_distance entry above l_pot_max is clamped on the
    # device; the flag word keeps it until frpa_sumup_noalloc_flags reads it
    p = synth.make_sumup_problem(n_atoms=10, n_points=1500, l_pot_max=4, T=1, seed=23)
    _noalloc_flags()  # start from a clear flag word
    a = _device_arrays(p)
    bad = p.l_hartree_max_far_distance.copy()
    bad[3, 0] = p.l_pot_max + 2
    a["lhmfd"] = dev(bad, np.int32)
    plan = _lib.SumupPlan(p)
    plan.device_flags()
    dv_plan, dv_noalloc = dev(p.delta_v_hartree), dev(p.delta_v_hartree)
    plan.execute(1, a["lhmfd"], a["mrs"], a["opr"], a["Q"], a["spline"], dv_plan)
    assert _noalloc(p, a, dv_noalloc) == 0, _lib.last_error()
    torch.cuda.synchronize()
    assert plan.device_flags() & 1
    assert _noalloc_flags() & 1
    assert _noalloc_flags() == 0  # read and cleared
    d0 = p.delta_v_hartree
    shape = (p.n_full_points, p.T)
    assert normwise_rel(host(dv_noalloc, shape) - d0, host(dv_plan, shape) - d0) < TOL
    plan.close()
