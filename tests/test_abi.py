"""The C-ABI library on the CPU: it loads, exports every symbol include/frpa.h
declares, and rejects bad input before touching a device."""
import ctypes
import os
import re

import numpy as np
import pytest

from fast_rpa_eval_b200 import _lib, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "frpa.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:void|int|char)\s*\*?\s*([A-Za-z_]\w*)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_reference_entry_points():
    names = declared_functions()
    for ref in ("evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_",
                "evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_cu_host_",
                "sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_",
                "sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_cu_host_",
                "generate_first_order_rho_bias_part2_",
                "init_dfpt_device_info", "init_dfpt_device_data", "free_dfpt_device_data", "free_dfpt_device_info"):
        assert ref in names


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_error_state_and_settings():
    L = _lib.lib()
    L.frpa_clear_error()
    assert L.frpa_last_error() == 0
    assert L.frpa_set_atom_tile_size(0) == _lib.FRPA_ERR_INVALID
    assert L.frpa_last_error() == _lib.FRPA_ERR_INVALID
    assert b"tile" in L.frpa_last_error_message()
    assert L.frpa_set_atom_tile_size(4) == 0 and L.frpa_get_atom_tile_size() == 4
    assert L.frpa_set_atom_tile_size(1) == 0
    assert L.frpa_set_rho1_mode(7) == _lib.FRPA_ERR_INVALID


@pytest.mark.parametrize("mutate,needle", [
    (lambda p: p.i_basis_batches.__setitem__((0, 0), 0), "basis index"),
    (lambda p: p.n_point_batches.__setitem__(0, p.n_max_batch_size + 1), "points"),
    (lambda p: p.i_batch_2_wave_offset.__setitem__(1, 10**8), "wave block"),
    (lambda p: p.i_valid_point_2_i_full_points_map.__setitem__(0, -1), "map"),
])
def test_rho1_plan_validation_rejects_bad_metadata(mutate, needle):
    p = synth.make_rho1_problem(T=1, seed=2, n_batches=6)
    mutate(p)
    with pytest.raises(_lib.FrpaError) as e:
        _lib.Rho1Plan(p)
    assert e.value.status == _lib.FRPA_ERR_INVALID and needle in e.value.message


@pytest.mark.parametrize("mutate,needle", [
    (lambda p: p.centers_hartree_potential.__setitem__(0, 10**6), "centers_hartree_potential"),
    (lambda p: p.index_cc.__setitem__((3, 1), 5), "(l, m)"),
    (lambda p: p.l_hartree.__setitem__(0, 99), "l_hartree"),
    (lambda p: p.i_valid_point_2_i_full_points_map.__setitem__(0, 10**9), "map"),
])
def test_sumup_plan_validation_rejects_bad_tables(mutate, needle):
    p = synth.make_sumup_problem(n_atoms=5, n_points=50, l_pot_max=4, seed=1)
    mutate(p)
    with pytest.raises(_lib.FrpaError) as e:
        _lib.SumupPlan(p)
    assert e.value.status == _lib.FRPA_ERR_INVALID and needle in e.value.message


def test_cu_host_without_session_reports_no_session():
    p = synth.make_rho1_problem(T=1, seed=2, n_batches=4)
    with pytest.raises(_lib.FrpaError) as e:
        _lib.Session.rho1(type("S", (), {"rho_prob": p})(), None)
    assert e.value.status == _lib.FRPA_ERR_NO_SESSION
