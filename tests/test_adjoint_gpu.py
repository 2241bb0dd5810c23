"""Adjoints on the GPU: dL/dP1 against the first-order-H integration (the
reference's evaluate_first_order_H with its XC terms zero) and against central
finite differences; dL/dQ_lm of the sum-up against central finite differences."""
import numpy as np
import pytest
import torch

import oracle
from fast_rpa_eval_b200 import _lib, autograd, synth
from gpu_util import dev, host, normwise_rel

pytestmark = pytest.mark.gpu


def _rho1_setup(p):
    plan = _lib.Rho1Plan(p)
    return plan, dev(p.wave), dev(p.gradient_wave), dev(p.first_order_rho_bias_part2), dev(p.first_order_gradient_rho_bias)


@pytest.mark.parametrize("T", [1, 2])
def test_dP1_equals_first_order_h(T):
    p = synth.make_rho1_problem(T=T, seed=70 + T, n_atoms=10, n_batches=40, with_bias=True, pad_value=np.nan)
    v = np.asfortranarray(np.random.default_rng(T).normal(size=(p.n_full_points, T)))
    plan, w, gw, b, gb = _rho1_setup(p)
    g_rho = dev(p.partition_tab[:, None] * v)
    dP1 = torch.zeros(p.n_basis * p.n_basis * T, dtype=torch.float64, device="cuda")
    plan.adjoint_p1(T, w, gw, g_rho, None, dP1)
    torch.cuda.synchronize()
    H = oracle.first_order_h(p, v, use_reference=oracle.ref_available(T))
    assert normwise_rel(host(dP1, H.shape), H) < 1e-12


def _loss_fd(fun, x, idx, h):
    xp = x.clone(); xp[idx] += h
    xm = x.clone(); xm[idx] -= h
    return (fun(xp) - fun(xm)) / (2 * h)


def test_dP1_central_finite_differences_config5_recipe():
    # config 5: config-1 recipe at 200 atoms, L = sum w v rho1, h = 1e-6 on 50 single P1 entries
    p = synth.make_rho1_problem(T=1, seed=5, n_atoms=200, box=None, density=0.1, n_batches=1600,
                                nc_range=(40, 120), exact_selection=False)
    rng = np.random.default_rng(5)
    w = torch.tensor(rng.uniform(0.01, 1.0, p.n_full_points), device="cuda")
    v = torch.tensor(rng.normal(size=p.n_full_points), device="cuda")
    plan, wv, gw, b, gb = _rho1_setup(p)
    P1 = dev(p.first_order_density_matrix).requires_grad_(True)
    rho, grad = autograd.rho1(P1, plan, wv, gw, b, gb, 1)
    L = (w * v * rho).sum()
    L.backward()
    g = P1.grad.detach()

    def loss(P):
        r, _ = autograd.rho1(P, plan, wv, gw, b, gb, 1)
        return float((w * v * r).sum())

    touched = torch.nonzero(g != 0).flatten().cpu().numpy()
    idx = rng.choice(touched, 50, replace=False)
    base = P1.detach()
    errs = [abs(_loss_fd(loss, base, int(i), 1e-6) - float(g[int(i)])) for i in idx]
    assert max(errs) < 1e-7, max(errs)


def test_dP1_with_gradient_outputs_finite_differences():
    p = synth.make_rho1_problem(T=2, seed=6, n_atoms=8, n_batches=24, with_bias=True)
    rng = np.random.default_rng(6)
    plan, wv, gw, b, gb = _rho1_setup(p)
    c_rho = torch.tensor(rng.normal(size=p.n_full_points * 2), device="cuda")
    c_grad = torch.tensor(rng.normal(size=3 * p.n_max_batch_size * p.n_my_batches_work * 2), device="cuda")
    P1 = dev(p.first_order_density_matrix).requires_grad_(True)
    r, g_ = autograd.rho1(P1, plan, wv, gw, b, gb, 1)  # n_active 1 < T: rho1 only for t = 0
    ((c_rho * r).sum() + (c_grad * g_).sum()).backward()
    g = P1.grad.detach()

    def loss(P):
        r, g_ = autograd.rho1(P, plan, wv, gw, b, gb, 1)
        return float((c_rho * r).sum() + (c_grad * g_).sum())

    idx = rng.choice(np.nonzero(g.cpu().numpy())[0], 30, replace=False)
    errs = [abs(_loss_fd(loss, P1.detach(), int(i), 1e-6) - float(g[int(i)])) for i in idx]
    assert max(errs) < 1e-7, max(errs)


def test_dQ_central_finite_differences_config5_recipe():
    # config 5 sum-up: 100 atoms, l_max 6, 200,000 points, h = 1e-6 on Q_lm
    p = synth.make_sumup_problem(n_atoms=100, n_points=200_000, l_pot_max=6, T=1, seed=9, outer_radius=8.0,
                                 l_hartree_per_species=[6, 5, 4, 6])
    rng = np.random.default_rng(9)
    plan = _lib.SumupPlan(p)
    assert plan.fast
    args = (dev(p.l_hartree_max_far_distance, np.int32), dev(p.multipole_radius_sq), dev(p.outer_potential_radius))
    spline = dev(p.spline)
    dv0 = dev(p.delta_v_hartree)
    wg = torch.tensor(rng.uniform(0.01, 1.0, p.n_full_points) * rng.normal(size=p.n_full_points), device="cuda")
    Q = dev(p.multipole_moments).requires_grad_(True)
    dv = autograd.sumup(Q, plan, *args, spline, dv0, 1)
    (wg * dv).sum().backward()
    g = Q.grad.detach()

    def loss(Qx):
        return float((wg * autograd.sumup(Qx, plan, *args, spline, dv0, 1)).sum())

    qv = p.multipole_moments.ravel(order="F")
    cand = np.nonzero(np.abs(qv) > 1e-5)[0]  # away from the 1e-10 threshold at +-h
    idx = rng.choice(cand, 40, replace=False)
    errs = [abs(_loss_fd(loss, Q.detach(), int(i), 1e-6) - float(g[int(i)])) for i in idx]
    scale = max(1.0, float(np.max(np.abs(g.cpu().numpy()[idx]))))
    assert max(errs) / scale < 1e-7, (max(errs), scale)


def test_dQ_is_bit_identical_across_runs():
    p = synth.make_sumup_problem(n_atoms=40, n_points=60_000, l_pot_max=6, T=2, seed=19, outer_radius=8.0)
    plan = _lib.SumupPlan(p)
    rng = np.random.default_rng(19)
    args = (dev(p.l_hartree_max_far_distance, np.int32), dev(p.multipole_radius_sq), dev(p.outer_potential_radius),
            dev(p.multipole_moments))
    g = dev(rng.normal(size=(p.n_full_points, 2)))
    outs = []
    for _ in range(3):
        dQ = torch.empty(p.multipole_moments.size, dtype=torch.float64, device="cuda")
        plan.adjoint_q(2, *args, g, dQ)
        torch.cuda.synchronize()
        outs.append(dQ.clone())
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])
    assert float(outs[0].abs().max()) > 0


def test_dQ_on_the_generic_path_is_reported_unsupported():
    # centres that are not the identity list put the plan on the generic kernel
    p = synth.make_sumup_problem(n_atoms=12, n_points=2000, l_pot_max=4, T=1, seed=21, centers="permuted")
    plan = _lib.SumupPlan(p)
    assert not plan.fast
    args = (dev(p.l_hartree_max_far_distance, np.int32), dev(p.multipole_radius_sq), dev(p.outer_potential_radius),
            dev(p.multipole_moments))
    dQ = torch.empty(p.multipole_moments.size, dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.FrpaError) as e:
        plan.adjoint_q(1, *args, dev(p.delta_v_hartree), dQ)
    assert e.value.status == _lib.FRPA_ERR_UNSUPPORTED and "fast path" in e.value.message
