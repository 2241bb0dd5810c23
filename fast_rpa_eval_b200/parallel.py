"""Sharding the rho1 / sum-up work over ranks (one process per GPU).

The grid batches of evaluate_first_order_rho are independent and their outputs
disjoint (rho1 is scattered through i_valid_point_2_i_full_points_map, grad rho1
is indexed by batch), so the forward pass needs no collective: each rank
evaluates a cost-balanced subset of the batches on its own GPU and the slices
are merged (or simply left where the caller wants them).  The sum-up is
independent per grid point the same way.  The adjoints are sums over batches
(dL/dP1) and over points (dL/dQ_lm): one all-reduce each.

    shards = shard_batches(rho1_batch_costs(prob), world_size)
    sub = select_batches(prob, shards[rank])      # a standalone problem
    ...run sub on this rank's GPU...
    rho, grad = merge_rho1(prob, [(shards[r], rho_r, grad_r) for r in ranks])

Host-side logic only; the GPU work goes through the C ABI (`_lib`).
"""

from __future__ import annotations

import dataclasses

import numpy as np


def rho1_batch_costs(prob) -> np.ndarray:
    """Work estimate per batch: T (nc^2 np + 4 nc np), the contraction plus the
    phi / grad-phi streams; 0 for batches without compute functions."""
    nc = prob.n_compute_c_batches.astype(np.float64)
    npb = prob.n_point_batches.astype(np.float64)
    c = prob.T * (nc * nc * npb + 4.0 * nc * npb)
    c[prob.n_compute_c_batches <= 0] = 0.0
    return c


def shard_batches(costs, world_size: int) -> list[np.ndarray]:
    """Partition batch indices into ``world_size`` sets of near-equal total
    cost (longest-processing-time greedy, deterministic); each set sorted."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    costs = np.asarray(costs, dtype=np.float64)
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(world_size)
    owner = np.empty(len(costs), dtype=np.int64)
    for b in order:
        r = int(np.argmin(load))
        owner[b] = r
        load[r] += costs[b]
    return [np.flatnonzero(owner == r) for r in range(world_size)]


def select_batches(prob, batch_ids) -> object:
    """The batches ``batch_ids`` of ``prob`` as a standalone problem: the same
    n_full_points and point map values (so rho1 lands at the caller's full-
    point indices), batch arrays and phi blocks re-packed in the given order."""
    ids = np.asarray(batch_ids, dtype=np.int64)
    pre, off = prob.n_point_batches_prefix_sum, prob.i_batch_2_wave_offset
    npb = prob.n_point_batches[ids].astype(np.int32)
    new_pre = np.zeros(len(ids) + 1, dtype=np.int32)
    new_pre[1:] = np.cumsum(npb)
    blk = (off[ids + 1] - off[ids]).astype(np.int64)
    new_off = np.zeros(len(ids) + 1, dtype=np.int64)
    new_off[1:] = np.cumsum(blk)
    pmap = np.concatenate([prob.i_valid_point_2_i_full_points_map[pre[b]:pre[b + 1]] for b in ids]) if len(ids) \
        else np.zeros(0, dtype=np.int32)
    wave = gwave = xyz = None
    if prob.valid_points_xyz is not None:  # the points' coordinates, for a device phi generator
        xyz = np.concatenate([prob.valid_points_xyz[pre[b]:pre[b + 1]] for b in ids]) if len(ids) \
            else np.zeros((0, 3))
    if prob.wave is not None:
        wave = np.concatenate([prob.wave[off[b]:off[b + 1]] for b in ids]) if len(ids) else np.zeros(0)
        gwave = np.concatenate([prob.gradient_wave[3 * off[b]:3 * off[b + 1]] for b in ids]) if len(ids) \
            else np.zeros(0)
    return dataclasses.replace(
        prob, n_my_batches_work=len(ids), batch_sizes=prob.batch_sizes[ids].copy(), n_point_batches=npb,
        n_point_batches_prefix_sum=new_pre, i_valid_point_2_i_full_points_map=pmap.astype(np.int32),
        n_compute_c_batches=prob.n_compute_c_batches[ids].copy(),
        i_basis_batches=np.asfortranarray(prob.i_basis_batches[:, ids]),
        atom_valid_n_compute_c_batches=np.asfortranarray(prob.atom_valid_n_compute_c_batches[:, ids]),
        i_batch_2_wave_offset=new_off.astype(np.int32), wave=wave, gradient_wave=gwave,
        first_order_rho_bias_part2=np.asfortranarray(prob.first_order_rho_bias_part2[:, ids, :]),
        first_order_gradient_rho_bias=np.asfortranarray(prob.first_order_gradient_rho_bias[:, :, ids, :]),
        valid_points_xyz=xyz)


def merge_rho1(prob, parts):
    """Full (rho1 (n_full_points, T), grad rho1 (3, n_max_batch_size,
    n_batches, T)) from per-shard results [(batch_ids, rho, grad), ...] of
    problems made by select_batches."""
    T = prob.T
    rho = np.zeros((prob.n_full_points, T))
    grad = np.zeros((3, prob.n_max_batch_size, prob.n_my_batches_work, T), order="F")
    pre, pmap = prob.n_point_batches_prefix_sum, prob.i_valid_point_2_i_full_points_map
    for ids, r, g in parts:
        ids = np.asarray(ids, dtype=np.int64)
        g = np.asarray(g).reshape((3, prob.n_max_batch_size, len(ids), T), order="F")
        r = np.asarray(r).reshape((prob.n_full_points, T), order="F")
        for k, b in enumerate(ids):
            if prob.n_compute_c_batches[b] <= 0:
                continue
            pts = pmap[pre[b]:pre[b + 1]]
            rho[pts, :] = r[pts, :]
            grad[:, :, b, :] = g[:, :, k, :]
    return rho, grad


def shard_points(n_valid_points: int, world_size: int, rank: int) -> slice:
    """Contiguous, near-equal range of valid points for ``rank``."""
    base, extra = divmod(int(n_valid_points), world_size)
    lo = rank * base + min(rank, extra)
    return slice(lo, lo + base + (1 if rank < extra else 0))


def select_points(sumup_prob, points: slice):
    """The sum-up restricted to the valid points ``points`` (same full-point
    arrays; only those points are accumulated)."""
    pmap = sumup_prob.i_valid_point_2_i_full_points_map[points]
    return dataclasses.replace(sumup_prob, n_valid_points=len(pmap),
                               i_valid_point_2_i_full_points_map=np.ascontiguousarray(pmap, dtype=np.int32))


def all_reduce_sum(tensor, group=None):
    """In-place sum over ranks (the one collective of the adjoints: dL/dP1 or
    dL/dQ_lm).  A torch tensor on the rank's device (NCCL) or on the CPU (gloo)."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(tensor, op=dist.ReduceOp.SUM, group=group)
    return tensor
