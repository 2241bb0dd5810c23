"""The boundary as the reference's own C++ callers see it.

oracle/_ref/libref_headers_check.so is tests/cxx/reference_headers_check.cpp
compiled against the reference's headers (evaluate_first_order_rho.h,
sum_up_whole_potential.h, evaluate_first_order_H.h, device_data.hpp) together
with include/frpa.h -- it only compiles if both declare every shared entry
point alike -- and linked against libfrpa.so.  Its thin C wrappers call the
entry points the reference declares with C++ linkage (the session functions and
the sum-up's cu_host_ twin) by their C++ symbols, as the reference's runners
do.  Loading it resolves every such symbol against libfrpa.so; the GPU test
runs a session through them against the oracle."""
import ctypes
import os
import types

import numpy as np
import pytest

import oracle
from fast_rpa_eval_b200 import _lib, synth
from gpu_util import normwise_rel

CHECK = os.path.join(os.path.dirname(oracle.__file__), "_ref", "libref_headers_check.so")
needs_check_lib = pytest.mark.skipif(not os.path.exists(CHECK),
                                     reason="reference headers were absent when oracle/_ref was built")
CXX_LINKAGE = ("init_dfpt_device_info", "free_dfpt_device_info", "init_dfpt_device_data", "free_dfpt_device_data",
               "sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_cu_host_")


def _entry():
    _lib.lib()  # libfrpa.so first, so the check library binds to this copy
    L = ctypes.CDLL(CHECK)  # RTLD_NOW: every C++ symbol it uses must resolve in libfrpa.so
    return types.SimpleNamespace(**{n: getattr(L, "hdrchk_" + n) for n in CXX_LINKAGE})


@needs_check_lib
def test_cxx_linkage_symbols_resolve_in_the_library():
    e = _entry()
    assert all(callable(getattr(e, n)) for n in CXX_LINKAGE)


@needs_check_lib
@pytest.mark.gpu
def test_session_through_cxx_linkage_matches_oracle():
    r = synth.make_rho1_problem(T=1, seed=13, n_batches=10, with_bias=True)
    n_r = int(r.n_point_batches_prefix_sum[-1])
    p = synth.make_sumup_problem(n_atoms=12, n_points=n_r + 800, l_pot_max=6, T=1, seed=84)
    # the session holds one full-point set and one valid-point map for both
    # paths (as init_dfpt_device_data does): rho1's points are the first n_r
    # entries of the sum-up's map
    p.n_full_points = r.n_full_points = max(r.n_full_points, p.n_full_points)
    pad = p.n_full_points - p.coord_points.shape[1]
    p.coord_points = np.asfortranarray(np.concatenate([p.coord_points, np.zeros((3, pad))], axis=1))
    p.delta_v_hartree = np.asfortranarray(np.concatenate([p.delta_v_hartree, np.zeros((pad, 1))], axis=0))
    p.partition_tab = np.concatenate([p.partition_tab, np.ones(pad)])
    r.partition_tab = p.partition_tab
    r.i_valid_point_2_i_full_points_map = p.i_valid_point_2_i_full_points_map[:n_r].astype(np.int32).copy()
    with _lib.Session(r, p, entry=_entry()) as s:
        rho, grad = s.rho1()
        r_o, g_o = oracle.rho1(r)
        assert normwise_rel(rho.reshape(r_o.shape, order="F"), r_o) < 1e-12
        assert normwise_rel(grad.reshape(g_o.shape, order="F"), g_o) < 1e-12
        out = s.sumup()
        ref = oracle.sumup(p)
        d0 = p.delta_v_hartree
        assert normwise_rel(out - d0, ref - d0) < 1e-12
