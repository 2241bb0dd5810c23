"""The bias producer (generate_first_order_rho_bias_part2) on the GPU against
the oracle: plan entry point and reference-named drop-in, every j_coord,
symmetric and non-symmetric density matrices, NaN wave padding.  Stated
tolerance: 1e-12 normwise relative (FP64; the two reference GEMM terms are
summed as one contraction, so rounding differs)."""

import numpy as np
import pytest

import oracle
from fast_rpa_eval_b200 import _lib, synth

TOL = 1e-12


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _problem(seed=4):
    p = synth.make_rho1_problem(T=4, seed=seed, n_atoms=6, n_batches=24, pad_value=np.nan, n_active=3)
    p.j_atom_begin, p.j_atom_end = 2, 4
    return p


@pytest.mark.gpu
@pytest.mark.parametrize("j_coord", [1, 3])
@pytest.mark.parametrize("symmetric", [True, False])
def test_bias_plan_matches_oracle(j_coord, symmetric):
    import torch

    from gpu_util import dev, host

    p = _problem()
    dm = np.random.default_rng(2).normal(size=(p.n_basis, p.n_basis))
    if symmetric:
        dm = dm + dm.T
    ref = oracle.rho_bias_part2(p, dm, j_coord=j_coord)
    plan = _lib.Rho1Plan(p)
    out = torch.zeros(p.n_max_batch_size * p.n_my_batches_work * 4, dtype=torch.float64, device="cuda")
    av = dev(p.atom_valid_n_compute_c_batches, np.int32)
    plan.bias_part2(4, p.n_atoms, p.j_atom_begin, p.j_atom_end, j_coord, av, dev(p.wave), dev(p.gradient_wave),
                    dev(dm), out)
    torch.cuda.synchronize()
    got = host(out, (p.n_max_batch_size, p.n_my_batches_work, 4))
    assert rel(got[:, :, :3], ref[:, :, :3]) < TOL
    assert np.all(got[:, :, 3] == 0.0)
    assert plan.device_flags() == 0


@pytest.mark.gpu
def test_bias_dropin_matches_reference_entry_semantics():
    p = _problem(seed=7)
    dm = np.random.default_rng(5).normal(size=(p.n_basis, p.n_basis))
    init = np.full((p.n_max_batch_size, p.n_my_batches_work, 4), 9.0)
    got = _lib.dropin_bias_part2(p, dm, j_coord=2, bias=init)
    ref = oracle.rho_bias_part2(p, dm, j_coord=2)
    # written: points of batches with compute functions, atoms j_atom_begin..j_atom_end;
    # everything else keeps the caller's values, as in the reference
    written = np.zeros(got.shape, dtype=bool)
    for b in range(p.n_my_batches_work):
        if p.n_compute_c_batches[b] > 0:
            written[: p.n_point_batches[b], b, :3] = True
    assert rel(np.where(written, got, 0.0), np.where(written, ref, 0.0)) < TOL
    assert np.all(got[~written] == 9.0)


@pytest.mark.gpu
def test_bias_flags_a_range_outside_the_batch():
    import torch

    from gpu_util import dev

    p = _problem()
    av = np.array(p.atom_valid_n_compute_c_batches, dtype=np.int32, order="F").copy()
    b = int(np.argmax(p.n_compute_c_batches))
    av[p.j_atom_begin, b] = p.n_compute_c_batches[b] + 5  # atom j_atom_begin's range leaves batch b
    plan = _lib.Rho1Plan(p)
    out = torch.zeros(p.n_max_batch_size * p.n_my_batches_work * 4, dtype=torch.float64, device="cuda")
    plan.bias_part2(4, p.n_atoms, p.j_atom_begin, p.j_atom_end, 1, dev(av, np.int32), dev(p.wave),
                    dev(p.gradient_wave), dev(np.eye(p.n_basis)), out)
    torch.cuda.synchronize()
    assert plan.device_flags() & 8


@pytest.mark.gpu
@pytest.mark.parametrize("j_coord", [1, 2])
def test_fused_bias_equals_rho1_plus_bias_part2(j_coord):
    """frpa_rho1_execute_fused_bias: rho1 with the density-matrix bias computed
    in the same launch equals the two-launch form (rho1 plus the oracle's
    bias part 2 for the active perturbations); grad rho1 is unchanged."""
    import torch

    from gpu_util import dev, host

    p = synth.make_rho1_problem(T=4, seed=9, n_atoms=6, n_batches=24, pad_value=np.nan, n_active=3,
                                with_bias=True)
    p.j_atom_begin, p.j_atom_end = 2, 4
    dm = np.random.default_rng(5).normal(size=(p.n_basis, p.n_basis))  # not symmetric: both gathers matter
    plan = _lib.Rho1Plan(p)
    args = [dev(p.wave), dev(p.gradient_wave), dev(p.first_order_density_matrix), dev(p.first_order_rho_bias_part2),
            dev(p.first_order_gradient_rho_bias)]
    n_rho, n_grad = p.n_full_points * 4, 3 * p.n_max_batch_size * p.n_my_batches_work * 4
    rho, grad = (torch.zeros(n, dtype=torch.float64, device="cuda") for n in (n_rho, n_grad))
    rho0, grad0 = (torch.zeros(n, dtype=torch.float64, device="cuda") for n in (n_rho, n_grad))
    plan.execute_fused_bias(3, p.n_atoms, 2, j_coord, dev(p.atom_valid_n_compute_c_batches, np.int32), dev(dm),
                            *args, rho, grad)
    plan.execute(3, *args, rho0, grad0, mode=_lib.RHO1_FP64)
    torch.cuda.synchronize()
    assert plan.device_flags() == 0
    bias2 = oracle.rho_bias_part2(p, dm, j_coord=j_coord)  # (nmb, nb, 4)
    want = host(rho0, (p.n_full_points, 4)).copy()
    pre, pmap = p.n_point_batches_prefix_sum, p.i_valid_point_2_i_full_points_map
    for b in range(p.n_my_batches_work):
        if p.n_compute_c_batches[b] <= 0:
            continue
        pts = pmap[pre[b]:pre[b + 1]]
        want[pts, :3] += bias2[:len(pts), b, :3]
    got = host(rho, (p.n_full_points, 4))
    assert rel(got, want) < TOL
    assert np.array_equal(got[:, 3], want[:, 3])  # perturbation 4 is not active
    assert torch.equal(grad, grad0)


@pytest.mark.gpu
def test_fused_bias_same_bits_for_both_tile_widths():
    """The fused-bias launch at 128-point work items (the FP64 tile tuning)
    gives the same bits as at 64-point items: per point, both sum the row
    tiles and the lanes of a warp in the same order."""
    import torch

    from gpu_util import dev

    p = synth.make_rho1_problem(T=2, seed=19, n_atoms=6, n_batches=20, with_bias=True, np_range=(60, 250))
    dm = np.random.default_rng(6).normal(size=(p.n_basis, p.n_basis))
    plan = _lib.Rho1Plan(p)
    args = [dev(p.wave), dev(p.gradient_wave), dev(p.first_order_density_matrix), dev(p.first_order_rho_bias_part2),
            dev(p.first_order_gradient_rho_bias)]
    n_rho, n_grad = p.n_full_points * 2, 3 * p.n_max_batch_size * p.n_my_batches_work * 2
    outs = []
    for tile in (64, 128):
        plan.set_tuning(fp64_tile_points=tile)
        rho, grad = (torch.zeros(n, dtype=torch.float64, device="cuda") for n in (n_rho, n_grad))
        plan.execute_fused_bias(2, p.n_atoms, 1, 1, dev(p.atom_valid_n_compute_c_batches, np.int32), dev(dm), *args,
                                rho, grad)
        torch.cuda.synchronize()
        outs.append((rho, grad))
    assert plan.device_flags() == 0
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
