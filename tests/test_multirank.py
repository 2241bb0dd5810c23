"""Multi-rank plumbing on CPU: two gloo ranks shard the config-1 rho1 batches and
the sum-up points, evaluate their shards with the oracle, and reassemble.

* rho1 / grad rho1 from the shards equal the unsharded result bit for bit
  (batches are independent);
* dL/dP1 (first-order H) summed over ranks by the all-reduce equals the
  unsharded integral to rounding;
* the sum-up from point shards equals the unsharded result bit for bit;
* dL/dQ_lm of the sum-up from point shards, summed by the all-reduce, equals
  the unsharded one to rounding.
"""

import dataclasses
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from fast_rpa_eval_b200 import parallel, synth


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problems():
    prob = synth.config1(seed=11)
    sp = synth.make_sumup_problem(n_atoms=12, n_points=3000, l_pot_max=4, T=1, seed=5)
    return prob, sp


def _dq_by_linearity(sp, g):
    """dQ_lm(a) = sum_p g(p) d delta_v(p)/dQ_lm(a) for the moments the forward
    keeps (|Q| > 1e-10): the sum-up is linear in them, so each column is one
    oracle call with a unit moment and the near field (spline) off."""
    L2 = (sp.l_pot_max + 1) ** 2
    zero_spline = np.zeros_like(sp.spline)
    zero_dv = np.zeros_like(sp.delta_v_hartree)
    dQ = np.zeros((L2, sp.n_atoms))
    for a in range(sp.n_atoms):
        for lm in range(L2):
            if abs(sp.multipole_moments[lm, a, 0]) <= 1e-10:
                continue
            Q = np.zeros_like(sp.multipole_moments)
            Q[lm, a, 0] = 1.0
            one = dataclasses.replace(sp, multipole_moments=Q, spline=zero_spline, delta_v_hartree=zero_dv)
            dQ[lm, a] = float(np.dot(g, oracle.sumup(one)[:, 0]))
    return dQ


def _worker(rank: int, world: int, port: int, out_dir: str):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        prob, sp = _problems()
        shards = parallel.shard_batches(parallel.rho1_batch_costs(prob), world)
        sub = parallel.select_batches(prob, shards[rank])
        r, g = oracle.rho1(sub)
        parts = [None] * world
        dist.all_gather_object(parts, (shards[rank], r, g))
        # adjoint: this rank's share of dL/dP1, summed over ranks
        v = np.random.default_rng(3).standard_normal((prob.n_full_points, prob.T))
        H = torch.from_numpy(np.ascontiguousarray(oracle.first_order_h(sub, v)))
        parallel.all_reduce_sum(H)
        # sum-up by point shards
        sl = parallel.shard_points(sp.n_valid_points, world, rank)
        dv = oracle.sumup(parallel.select_points(sp, sl))
        dparts = [None] * world
        dist.all_gather_object(dparts, (sl, dv))
        # sum-up adjoint: this rank's points' share of dL/dQ, summed over ranks
        gq = np.random.default_rng(7).standard_normal(sp.n_full_points)
        dQ = torch.from_numpy(_dq_by_linearity(parallel.select_points(sp, sl), gq))
        parallel.all_reduce_sum(dQ)
        if rank == 0:
            rho, grad = parallel.merge_rho1(prob, parts)
            dv_all = np.array(sp.delta_v_hartree, dtype=np.float64).reshape((sp.n_full_points, sp.T), order="F").copy()
            for s, d in dparts:
                pts = sp.i_valid_point_2_i_full_points_map[s]
                dv_all[pts, :] = d[pts, :]
            np.savez(os.path.join(out_dir, "merged.npz"), rho=rho, grad=grad, H=H.numpy(), dv=dv_all, dQ=dQ.numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_shard_batches_covers_every_batch_once_and_balances():
    rng = np.random.default_rng(0)
    costs = rng.uniform(1, 100, 997)
    costs[::13] = 0.0
    for world in (1, 2, 3, 8):
        shards = parallel.shard_batches(costs, world)
        allb = np.sort(np.concatenate(shards))
        assert np.array_equal(allb, np.arange(len(costs)))
        loads = np.array([costs[s].sum() for s in shards])
        assert loads.max() - loads.min() <= costs.max()


def test_shard_points_partition():
    for n, world in ((10, 3), (7, 8), (1000, 2)):
        cover = np.concatenate([np.arange(n)[parallel.shard_points(n, world, r)] for r in range(world)])
        assert np.array_equal(cover, np.arange(n))


def test_select_batches_roundtrip_single_rank():
    prob, _ = _problems()
    ids = np.arange(prob.n_my_batches_work)[::-1]
    r, g = oracle.rho1(parallel.select_batches(prob, ids))
    rho, grad = parallel.merge_rho1(prob, [(ids, r, g)])
    r0, g0 = oracle.rho1(prob)
    assert np.array_equal(rho, r0) and np.array_equal(grad, g0)


def test_two_gloo_ranks_reassemble_the_unsharded_results(tmp_path):
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    got = np.load(tmp_path / "merged.npz")
    prob, sp = _problems()
    r0, g0 = oracle.rho1(prob)
    assert np.array_equal(got["rho"], r0)
    assert np.array_equal(got["grad"], g0)
    v = np.random.default_rng(3).standard_normal((prob.n_full_points, prob.T))
    H0 = oracle.first_order_h(prob, v)
    assert np.max(np.abs(got["H"] - H0)) <= 1e-13 * np.max(np.abs(H0))
    assert np.array_equal(got["dv"], oracle.sumup(sp))
    dQ0 = _dq_by_linearity(sp, np.random.default_rng(7).standard_normal(sp.n_full_points))
    assert np.abs(dQ0).max() > 0
    assert np.max(np.abs(got["dQ"] - dQ0)) <= 1e-12 * np.max(np.abs(dQ0))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_gpu_shards_merge_to_the_unsharded_gpu_result(mode):
    """Each shard through its own plan (as each rank would on its GPU), merged:
    identical to one plan over all batches, for the FP64 and split paths."""
    from fast_rpa_eval_b200 import _lib
    from gpu_util import rho1_device_run

    prob, _ = _problems()
    full = rho1_device_run(_lib.Rho1Plan(prob), prob, mode=mode)
    parts = []
    for ids in parallel.shard_batches(parallel.rho1_batch_costs(prob), 3):
        sub = parallel.select_batches(prob, ids)
        r, g = rho1_device_run(_lib.Rho1Plan(sub), sub, mode=mode)
        parts.append((ids, r, g))
    rho, grad = parallel.merge_rho1(prob, parts)
    assert np.array_equal(rho, full[0]) and np.array_equal(grad, full[1])
