"""Capture / replay: the reader and writer keep the reference's dump layout.

The fixtures tests/golden/capture_*.bin were written by the reference's own
header-only writers (evaluate_first_order_rho_direct_test.hpp,
sum_up_direct_test.hpp) compiled in oracle/_ref, from the fixed recipe in
oracle/capture_writer.cpp (script: tests/golden/make_capture_golden.sh).
"""

import dataclasses
import os

import numpy as np
import pytest

import oracle
from fast_rpa_eval_b200 import capture, synth

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _dvec(n, start, step):
    return start + np.arange(n) * step


def test_reads_the_reference_rho_dump():
    m = capture.read_rho_meta(os.path.join(GOLD, "capture_rho_meta.bin"))
    assert [m[s] for s in capture.RHO_SCALARS] == [3, 11, 7, 2, 5, 7, 4]
    assert m["basis_atom"].tolist() == [1, 1, 1, 1, 2, 2, 2]
    assert m["batch_sizes"].tolist() == [4, 3, 4]
    assert m["n_point_batches_prefix_sum"].tolist() == [0, 4, 7, 11]
    assert m["i_valid_point_2_i_full_points_map"].tolist() == list(range(10, -1, -1))
    assert m["n_compute_c_batches"].tolist() == [5, 0, 3]
    assert m["i_basis_batches"].tolist() == list(range(1, 22))
    assert m["atom_valid_n_compute_c_batches"].tolist() == list(range(0, 18, 2))
    assert m["i_batch_2_wave_offset"].tolist() == [0, 32, 32, 48]
    capture.check_rho_meta(m)


def test_reads_the_reference_sumup_dump():
    s = capture.read_sumup_data(os.path.join(GOLD, "capture_sumup.bin"))
    assert [s[k] for k in capture.SUMUP_SCALARS] == [1, 2, 6, 2, 12, 5, 1, 9, 10, 3, 3, 3, 1, 2]
    assert s["i_valid_point_2_i_full_points_map"].tolist() == [5, 4, 3, 1, 0]
    assert np.array_equal(s["coord_points"], _dvec(18, -1.5, 0.25))
    assert np.array_equal(s["outer_potential_radius"], _dvec(12, 100.0, -3.0))
    assert np.array_equal(s["multipole_moments"], _dvec(24, 0.125, 0.0625))
    assert s["index_cc"].tolist() == list(range(72))
    assert np.array_equal(s["log_r_grid_inc"], [0.0125, 0.015])
    assert np.array_equal(s["partition_tab"], _dvec(6, 0.1, 0.1))


@pytest.mark.parametrize("name,reader,writer", [
    ("capture_rho_meta.bin", capture.read_rho_meta, capture.write_rho_meta),
    ("capture_sumup.bin", capture.read_sumup_data, capture.write_sumup_data)])
def test_writer_reproduces_the_reference_bytes(tmp_path, name, reader, writer):
    src = os.path.join(GOLD, name)
    out = tmp_path / name
    writer(str(out), reader(src))
    assert out.read_bytes() == open(src, "rb").read()


def test_truncated_and_padded_dumps_are_rejected(tmp_path):
    raw = open(os.path.join(GOLD, "capture_rho_meta.bin"), "rb").read()
    for bad in (raw[:-4], raw + b"\0\0\0\0", raw[:20]):
        p = tmp_path / "bad.bin"
        p.write_bytes(bad)
        with pytest.raises(capture.CaptureError):
            capture.read_rho_meta(str(p))


def test_replayed_rho1_metadata_gives_the_same_density(tmp_path):
    prob = synth.config1(seed=4)
    path = str(tmp_path / "meta.bin")
    capture.write_rho_meta(path, capture.rho_meta_of(prob))
    m = capture.read_rho_meta(path)
    capture.check_rho_meta(m)
    nb, ncb = m["n_my_batches_work"], m["n_centers_basis_I"]
    replay = dataclasses.replace(
        prob, **{s: m[s] for s in capture.RHO_SCALARS},
        basis_atom=m["basis_atom"], batch_sizes=m["batch_sizes"], n_point_batches=m["n_point_batches"],
        n_point_batches_prefix_sum=m["n_point_batches_prefix_sum"],
        i_valid_point_2_i_full_points_map=m["i_valid_point_2_i_full_points_map"],
        n_compute_c_batches=m["n_compute_c_batches"],
        i_basis_batches=m["i_basis_batches"].reshape((ncb, nb), order="F"),
        atom_valid_n_compute_c_batches=m["atom_valid_n_compute_c_batches"].reshape((-1, nb), order="F"),
        i_batch_2_wave_offset=m["i_batch_2_wave_offset"])
    r0, g0 = oracle.rho1(prob)
    r1, g1 = oracle.rho1(replay)
    assert np.array_equal(r0, r1) and np.array_equal(g0, g1)
