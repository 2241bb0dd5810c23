"""Helpers shared by the GPU tests: move Fortran-ordered numpy arrays to the
device as flat tensors and back."""
import numpy as np
import torch


def dev(a, dtype=None):
    a = np.asarray(a)
    if dtype is not None:
        a = a.astype(dtype)
    return torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).cuda()


def host(t, shape):
    return t.cpu().numpy().reshape(shape, order="F")


def normwise_rel(a, b):
    return float(np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b))))


def rho1_device_run(plan, prob, mode=0, n_active=None, wave=None, gwave=None):
    T = prob.T
    w = dev(prob.wave) if wave is None else wave
    gw = dev(prob.gradient_wave) if gwave is None else gwave
    rho = torch.full((prob.n_full_points * T,), 7.0, dtype=torch.float64, device="cuda")
    grad = torch.full((3 * prob.n_max_batch_size * prob.n_my_batches_work * T,), 7.0, dtype=torch.float64,
                      device="cuda")
    na = prob.j_atom_end - prob.j_atom_begin + 1 if n_active is None else n_active
    plan.execute(na, w, gw, dev(prob.first_order_density_matrix), dev(prob.first_order_rho_bias_part2),
                 dev(prob.first_order_gradient_rho_bias), rho, grad, mode=mode)
    torch.cuda.synchronize()
    return (host(rho, (prob.n_full_points, T)),
            host(grad, (3, prob.n_max_batch_size, prob.n_my_batches_work, T)))
