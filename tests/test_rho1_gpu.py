"""rho1 / grad rho1 on the GPU against the oracle (and the reference's own CPU code)."""
import numpy as np
import pytest

import oracle
from fast_rpa_eval_b200 import _lib, synth
from gpu_util import dev, host, normwise_rel, rho1_device_run

pytestmark = pytest.mark.gpu
TOL_FP64 = 1e-12  # normwise relative, plain FP64 path


@pytest.mark.parametrize("T,n_active", [(1, 1), (2, 2), (2, 1), (4, 3)])
def test_rho1_fp64_matches_oracle(T, n_active):
    p = synth.make_rho1_problem(T=T, seed=20 + T, with_bias=True, extra_full_points=37, empty_batches=4,
                                pad_value=np.nan, n_active=n_active)
    plan = _lib.Rho1Plan(p)
    r, g = rho1_device_run(plan, p)
    r_o, g_o = oracle.rho1(p)
    assert not np.isnan(r).any() and not np.isnan(g).any()
    assert normwise_rel(r, r_o) < TOL_FP64
    assert normwise_rel(g, g_o) < TOL_FP64
    # every entry the reference leaves at zero is zero here too
    assert np.array_equal(r_o == 0, r == 0)
    assert np.array_equal(g_o == 0, g == 0)


def test_rho1_fp64_deterministic():
    p = synth.make_rho1_problem(T=1, seed=5, with_bias=True)
    plan = _lib.Rho1Plan(p)
    a = rho1_device_run(plan, p)
    b = rho1_device_run(plan, p)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.skipif(not oracle.ref_available(1), reason="reference library not built")
def test_rho1_fp64_matches_reference_cpu_code():
    p = synth.make_rho1_problem(T=1, seed=8, with_bias=True, empty_batches=2, pad_value=np.nan, n_atoms=12,
                                n_batches=120, nc_range=(40, 240))
    r, g = rho1_device_run(_lib.Rho1Plan(p), p)
    r_ref, g_ref = oracle.rho1(p, use_reference=True)
    assert normwise_rel(r, r_ref) < TOL_FP64 and normwise_rel(g, g_ref) < TOL_FP64


def test_rho1_uneven_large_batches():
    # n_compute up to 800 and 400 points: many M tiles, uneven point tiles
    p = synth.make_rho1_problem(T=1, seed=9, n_atoms=60, shells="ssssppdd", box=None, density=0.1, n_batches=40,
                                np_range=(50, 400), nc_range=(50, 800), log_uniform=True, with_bias=True,
                                exact_selection=False, pad_value=np.nan)
    r, g = rho1_device_run(_lib.Rho1Plan(p), p)
    r_o, g_o = oracle.rho1(p, n_threads=8)
    assert normwise_rel(r, r_o) < TOL_FP64 and normwise_rel(g, g_o) < TOL_FP64


def test_rho1_odd_wave_offsets_use_8_byte_path():
    # shift every batch block by one element: no 16-byte alignment
    p = synth.make_rho1_problem(T=1, seed=11, with_bias=True, n_batches=16)
    w = np.concatenate([[0.0], p.wave])
    gw = np.concatenate([[0.0] * 3, p.gradient_wave])
    p.wave, p.gradient_wave = w, gw
    off = p.i_batch_2_wave_offset.astype(np.int64)
    # wave offset +1; gradient offsets are 3x the wave offsets, so +3 lines up
    p.i_batch_2_wave_offset = (off + 1).astype(np.int32)
    r_o, g_o = oracle.rho1(p)
    r, g = rho1_device_run(_lib.Rho1Plan(p), p)
    assert normwise_rel(r, r_o) < TOL_FP64 and normwise_rel(g, g_o) < TOL_FP64


@pytest.mark.parametrize("T", [1, 2])
def test_rho1_dropin_symbol_matches_oracle(T):
    p = synth.make_rho1_problem(T=T, seed=30 + T, with_bias=True, extra_full_points=11, empty_batches=2)
    r, g = _lib.dropin_rho1(p)
    r_o, g_o = oracle.rho1(p)
    assert normwise_rel(r, r_o) < TOL_FP64 and normwise_rel(g, g_o) < TOL_FP64


def test_rho1_session_cu_host_matches_oracle():
    p = synth.make_rho1_problem(T=2, seed=41, with_bias=True, extra_full_points=5)
    with _lib.Session(p) as s:
        for rep in range(2):
            P1 = p.first_order_density_matrix * (1.0 + rep)
            r, g = s.rho1(P1=np.asfortranarray(P1))
            q = synth.make_rho1_problem(T=2, seed=41, with_bias=True, extra_full_points=5)
            q.first_order_density_matrix = np.asfortranarray(P1)
            r_o, g_o = oracle.rho1(q)
            assert normwise_rel(r.reshape(r_o.shape, order="F"), r_o) < TOL_FP64
            assert normwise_rel(g.reshape(g_o.shape, order="F"), g_o) < TOL_FP64


@pytest.mark.parametrize("nb,T,pinned", [(3, 1, False), (64, 2, False), (64, 2, True)])
def test_rho1_session_chunks_equal_one_launch(nb, T, pinned):
    """The host-buffer entry point runs the FP64 step in four batch chunks with
    the bias uploads and grad rho1 downloads overlapped; its outputs equal one
    plan launch bit for bit (3 batches leave a chunk empty; T = 2 splits every
    copy per perturbation; pinned buffers take the asynchronous copy path)."""
    import torch

    p = synth.make_rho1_problem(T=T, seed=43, n_batches=nb, with_bias=True, extra_full_points=3)
    r_d, g_d = rho1_device_run(_lib.Rho1Plan(p), p)

    def host_buf(a):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))
        return torch.from_numpy(a).pin_memory() if pinned else a

    P1, bias, gbias = (host_buf(a) for a in (p.first_order_density_matrix, p.first_order_rho_bias_part2,
                                             p.first_order_gradient_rho_bias))
    rho = host_buf(np.full(p.n_full_points * T, 7.0))
    grad = host_buf(np.full(3 * p.n_max_batch_size * p.n_my_batches_work * T, 7.0))
    with _lib.Session(p) as s:
        for _ in range(2):  # the second call reuses the session's streams and events
            r, g = s.rho1(P1=P1, bias=bias, gbias=gbias, rho=rho, grad=grad)
            r = np.asarray(r).reshape(r_d.shape, order="F")
            g = np.asarray(g).reshape(g_d.shape, order="F")
            assert np.array_equal(r, r_d) and np.array_equal(g, g_d)


def test_library_device_selection():
    """frpa_set_device drives the library's own CUDA runtime (the one plans and
    the session use); a device past the last is rejected with a message."""
    import torch

    _lib.set_device(torch.cuda.current_device())
    assert _lib.get_device() == torch.cuda.current_device()
    with pytest.raises(_lib.FrpaError, match="outside"):
        _lib.set_device(torch.cuda.device_count())
    assert _lib.get_device() == torch.cuda.current_device()


def test_rho1_rejects_bad_input_without_touching_the_gpu_state():
    p = synth.make_rho1_problem(T=1, seed=3, n_batches=8)
    p.i_basis_batches[0, 0] = p.n_basis + 5
    with pytest.raises(_lib.FrpaError) as e:
        _lib.Rho1Plan(p)
    assert e.value.status == _lib.FRPA_ERR_INVALID
    # the library keeps working afterwards
    q = synth.make_rho1_problem(T=1, seed=3, n_batches=8)
    r, g = rho1_device_run(_lib.Rho1Plan(q), q)
    assert normwise_rel(r, oracle.rho1(q)[0]) < TOL_FP64


def test_synth_generator_matches_host_basis_values():
    p = synth.make_rho1_problem(T=1, seed=12, n_batches=10, shells="sspdf")
    plan_pts = dev(np.asfortranarray(p.valid_points_xyz.T))
    import torch
    w = torch.empty(p.wave_len, dtype=torch.float64, device="cuda")
    gw = torch.empty(3 * p.wave_len, dtype=torch.float64, device="cuda")
    _lib.synth_basis_values(p, plan_pts, w, gw, pad_value=0.0)
    torch.cuda.synchronize()
    assert normwise_rel(w.cpu().numpy(), p.wave) < 1e-13
    assert normwise_rel(gw.cpu().numpy(), p.gradient_wave) < 1e-13
