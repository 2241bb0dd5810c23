"""First-order H on the GPU (evaluate_first_order_h_reduce_memory_c_v2_ and
frpa_rho1_first_order_h) against the reference's own CPU code compiled in
oracle/_ref, with every exchange-correlation term non-zero, and the
determinism of the fixed-point accumulation it shares with the rho1 adjoint:
two runs give the same bits."""
import numpy as np
import pytest
import torch

import oracle
from fast_rpa_eval_b200 import _lib, synth
from gpu_util import dev, host, normwise_rel

pytestmark = pytest.mark.gpu
TOL = 1e-12  # normwise relative, FP64 against the reference's FP64


def _case(T, seed, n_atoms=6, n_batches=16, j_begin=1, n_active=None):
    p = synth.make_rho1_problem(T=T, seed=seed, n_atoms=n_atoms, n_batches=n_batches, pad_value=np.nan,
                                n_active=T if n_active is None else n_active)
    p.j_atom_begin = j_begin
    p.j_atom_end = j_begin + (T if n_active is None else n_active) - 1
    xc = synth.first_order_h_inputs(p, seed=seed + 1, pad_value=np.nan)
    v = np.asfortranarray(np.random.default_rng(seed + 2).normal(size=(p.n_full_points, T)))
    return p, xc, v


def _reference(p, v, xc, j_coord, H0):
    return H0 + oracle.first_order_h(p, v, use_reference=oracle.ref_available(p.T), xc=xc, j_coord=j_coord)


@pytest.mark.parametrize("T,j_coord,j_begin", [(1, 1, 1), (2, 2, 1), (2, 3, 3), (4, 1, 2)])
def test_first_order_h_dropin_matches_reference(T, j_coord, j_begin):
    p, xc, v = _case(T, 100 + 7 * T + j_coord, j_begin=j_begin, n_active=min(T, p_atoms(6, j_begin)))
    H0 = np.asfortranarray(np.random.default_rng(9).normal(size=(p.n_basis, p.n_basis, T)))
    got = _lib.dropin_first_order_h(p, v, xc, H=H0, j_coord=j_coord)
    ref = _reference(p, v, xc, j_coord, H0)
    assert np.all(np.isfinite(got))
    assert normwise_rel(got - H0, ref - H0) < TOL


def p_atoms(n_atoms, j_begin):
    return n_atoms - j_begin + 1


def test_first_order_h_partial_tile_leaves_other_perturbations():
    # tile of 3 with 2 atoms active: the third slice of H is left as it was
    p, xc, v = _case(3, 131, n_active=2)
    H0 = np.asfortranarray(np.random.default_rng(4).normal(size=(p.n_basis, p.n_basis, 3)))
    got = _lib.dropin_first_order_h(p, v, xc, H=H0, j_coord=2)
    ref = _reference(p, v, xc, 2, H0)
    assert normwise_rel(got[:, :, :2] - H0[:, :, :2], ref[:, :, :2] - H0[:, :, :2]) < TOL
    assert np.array_equal(got[:, :, 2], H0[:, :, 2])


def _device_inputs(p, xc, v):
    d = {k: dev(a) for k, a in xc.items()}
    return d, dev(v), dev(p.partition_tab), dev(p.atom_valid_n_compute_c_batches, np.int32)


def test_first_order_h_plan_is_bit_identical_across_runs():
    p, xc, v = _case(2, 141, n_atoms=12, n_batches=60)
    plan = _lib.Rho1Plan(p)
    d, vd, pt, av = _device_inputs(p, xc, v)
    w, gw, hw = dev(p.wave), dev(p.gradient_wave), d["hessian_wave"]
    outs = []
    for _ in range(3):
        H = torch.zeros(p.n_basis * p.n_basis * 2, dtype=torch.float64, device="cuda")
        plan.first_order_h(2, p.n_atoms, 1, 1, av, w, gw, hw, d, vd, pt, H)
        torch.cuda.synchronize()
        outs.append(H.clone())
    assert plan.device_flags() == 0
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])
    ref = oracle.first_order_h(p, v, use_reference=oracle.ref_available(2), xc=xc, j_coord=1)
    assert normwise_rel(host(outs[0], ref.shape), ref) < TOL


def test_adjoint_dP1_is_bit_identical_across_runs():
    p = synth.make_rho1_problem(T=2, seed=151, n_atoms=12, n_batches=60, with_bias=True)
    plan = _lib.Rho1Plan(p)
    rng = np.random.default_rng(3)
    g_rho = dev(rng.normal(size=(p.n_full_points, 2)))
    g_grad = dev(rng.normal(size=(3, p.n_max_batch_size, p.n_my_batches_work, 2)))
    w, gw = dev(p.wave), dev(p.gradient_wave)
    outs = []
    for _ in range(3):
        dP1 = torch.zeros(p.n_basis * p.n_basis * 2, dtype=torch.float64, device="cuda")
        plan.adjoint_p1(2, w, gw, g_rho, g_grad, dP1)
        torch.cuda.synchronize()
        outs.append(dP1.clone())
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])
    assert float(outs[0].abs().max()) > 0


def test_first_order_h_flags_a_range_outside_its_batch():
    p, xc, v = _case(1, 161)
    av = p.atom_valid_n_compute_c_batches.copy()
    b = int(np.argmax(p.n_compute_c_batches))
    av[1, b] = p.n_compute_c_batches[b] + 5  # atom 1's range runs past the batch's compute functions
    plan = _lib.Rho1Plan(p)
    d, vd, pt, _ = _device_inputs(p, xc, v)
    H = torch.zeros(p.n_basis * p.n_basis, dtype=torch.float64, device="cuda")
    plan.device_flags()
    plan.first_order_h(1, p.n_atoms, 1, 1, dev(av, np.int32), dev(p.wave), dev(p.gradient_wave),
                       d["hessian_wave"], d, vd, pt, H)
    torch.cuda.synchronize()
    assert plan.device_flags() & 8
    assert torch.isfinite(H).all()
