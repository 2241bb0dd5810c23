"""The oracle itself: pinned against the reference's own CPU sources
(compiled in place into oracle/_ref/) and against the mathematics."""
import json
import os

import numpy as np
import pytest

import oracle
from fast_rpa_eval_b200 import synth, tables
from conftest import needs_reference

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b))))


@needs_reference(1)
@pytest.mark.parametrize("T", [1, 2, 4])
def test_rho1_oracle_matches_reference(T):
    p = synth.make_rho1_problem(T=T, seed=10 + T, with_bias=True, extra_full_points=50, empty_batches=3,
                                pad_value=np.nan, n_active=max(1, T - 1))
    r_o, g_o = oracle.rho1(p)
    r_r, g_r = oracle.rho1(p, use_reference=True)
    assert not np.isnan(r_o).any() and not np.isnan(g_o).any()
    assert rel(r_o, r_r) < 1e-13 and rel(g_o, g_r) < 1e-13


def test_rho1_oracle_threads_identical():
    p = synth.make_rho1_problem(T=1, seed=3, with_bias=True)
    a = oracle.rho1(p, n_threads=1)
    b = oracle.rho1(p, n_threads=4)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@needs_reference(1)
def test_ylm_oracle_matches_reference_sheval():
    rng = np.random.default_rng(0)
    for _ in range(100):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        ab = np.hypot(d[0], d[1])
        st, ct, cp, sp = ab, d[2], d[0] / ab, d[1] / ab
        for l in range(7):
            a = oracle.ylm(l, st * cp, st * sp, ct)
            b = oracle.ylm(l, 0, 0, 0, use_reference=True, trig=(st, ct, sp, cp))
            assert np.max(np.abs(a - b)) < 1e-13


@needs_reference(2)
@pytest.mark.parametrize("T,centers,lh", [(1, "identity", None), (2, "identity", [6, 4, 2, 0]),
                                          (1, "permuted", [6, 5, 3, 6]), (2, "permuted", None)])
def test_sumup_oracle_matches_reference(T, centers, lh):
    p = synth.make_sumup_problem(n_atoms=20, n_points=3000, l_pot_max=6, T=T, seed=5 + T, centers=centers,
                                 l_hartree_per_species=lh, extra_full_points=100)
    o, codes = oracle.sumup(p, branch_codes=True)
    r = oracle.sumup(p, use_reference=True)
    assert np.max(np.abs(o - r)) < 1e-13
    assert ((codes > 0) & (codes < 16)).sum() > 0 and (codes >= 16).sum() > 0  # both branches exercised


def test_index_cc_matches_reference_unrolled_kernel():
    g = json.load(open(os.path.join(GOLDEN, "index_cc_l6.json")))
    ic, cc, n, mx = tables.multipole_tables(6)
    assert ic[:, 2:6].tolist() == g["rows_ijk_nn"]
    assert n.tolist() == g["n_cc_lm_ijk"]
    # counts logged by the reference for l_max_analytic_multipole = 7 (index_cc_dim_0 = 280)
    assert tables.multipole_tables(7)[2].tolist() == [1, 4, 12, 28, 57, 104, 176, 280]


@pytest.mark.parametrize("L", [4, 6, 8])
def test_tables_reproduce_spherical_multipole_field(L):
    p = synth.make_sumup_problem(n_atoms=12, n_points=1500, l_pot_max=L, T=1, seed=40 + L, outer_radius=None,
                                 near_radius=0.3, with_spline=False)
    p.multipole_moments[np.abs(p.multipole_moments) < 1e-10] = 0.0
    d0 = p.delta_v_hartree.copy()
    o, codes = oracle.sumup(p, branch_codes=True)
    ov = (o[:, 0] - d0[:, 0])[p.i_valid_point_2_i_full_points_map]
    far = np.all(codes[:, :, 0] >= 16, axis=1)
    pts = np.asfortranarray(p.coord_points[:, p.i_valid_point_2_i_full_points_map])
    sph = oracle.far_field_spherical(L, pts, p.coords_center, p.multipole_moments[:, :, 0])
    assert far.sum() > 1000
    assert np.max(np.abs(ov - sph)[far]) / np.max(np.abs(sph[far])) < 1e-12


@needs_reference(2)
def test_first_order_h_oracle_matches_reference():
    p = synth.make_rho1_problem(T=2, seed=3, n_atoms=6, n_batches=20, with_bias=True, pad_value=np.nan)
    v = np.asfortranarray(np.random.default_rng(1).normal(size=(p.n_full_points, 2)))
    assert rel(oracle.first_order_h(p, v), oracle.first_order_h(p, v, use_reference=True)) < 1e-13


@needs_reference(2)
@pytest.mark.parametrize("j_coord", [1, 3])
def test_first_order_h_oracle_with_every_term_matches_reference(j_coord):
    p = synth.make_rho1_problem(T=2, seed=5, n_atoms=6, n_batches=16, pad_value=np.nan, n_active=2)
    xc = synth.first_order_h_inputs(p, seed=11, pad_value=np.nan)
    v = np.asfortranarray(np.random.default_rng(3).normal(size=(p.n_full_points, 2)))
    ho = oracle.first_order_h(p, v, xc=xc, j_coord=j_coord)
    hr = oracle.first_order_h(p, v, use_reference=True, xc=xc, j_coord=j_coord)
    assert np.all(np.isfinite(ho)) and np.abs(ho).max() > 0
    assert rel(ho, hr) < 1e-13
    # every term moves the result (the test would not see a dropped term otherwise)
    for k in xc:
        xk = dict(xc)
        xk[k] = np.zeros_like(xc[k])
        assert rel(oracle.first_order_h(p, v, xc=xk, j_coord=j_coord), ho) > 1e-6, k


@needs_reference(4)
def test_bias_producer_oracle_matches_reference():
    p = synth.make_rho1_problem(T=4, seed=4, n_atoms=6, n_batches=20, pad_value=np.nan, n_active=3)
    p.j_atom_begin, p.j_atom_end = 2, 4
    dm = np.random.default_rng(2).normal(size=(p.n_basis, p.n_basis))
    dm = dm + dm.T
    bo = oracle.rho_bias_part2(p, dm, j_coord=2)
    br = oracle.rho_bias_part2(p, dm, use_reference=True, j_coord=2)
    assert rel(bo[:, :, :3], br[:, :, :3]) < 1e-13
