"""Seeded synthetic workloads in the reference's exact array layouts.

The reference is driven by captured FHI-aims metadata plus ``setRandom`` bulk
arrays (fast_rap_src_dfpt_gpu_eval/direct_test/evaluate_first_order_rho_run.cpp:13-65,
.../sum_up_run.cpp:13-40); the captures are absent, so workloads are built
here from a physical recipe instead:

* atoms in a box, Gaussian basis functions  phi = R_lm(r - R_A) exp(-a |r - R_A|^2)
  (R_lm = r^l Y_lm, the real solid harmonic, so phi and grad phi are smooth and
  analytic), a log-uniform in [0.1, 10];
* grid batches of points drawn in a ball around an atom;
* per batch the n_compute functions with the largest max |phi| over the
  batch (the reference's cutoff |phi| > 1e-8 activates nearly every function
  with these exponents, so the n_compute ranges of each workload are imposed
  by drawing n_compute and keeping the strongest functions);
* arrays in Fortran (column-major) order with the reference's 1-based basis /
  species / centre indices and 0-based full-point indices.

Nothing here is on the product path; the library only consumes the arrays.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import tables

# --------------------------------------------------------------------------
# Basis functions
# --------------------------------------------------------------------------

SHELL_L = {"s": 0, "p": 1, "d": 2, "f": 3, "g": 4}


def _solid_monomials(l: int, m: int):
    norm, poly = tables.solid_harmonic(l, m)
    mons = [(norm * float(c), a, b, cc) for (a, b, cc), c in poly.items()]
    return mons


_MONO_CACHE: dict = {}


def solid_harmonic_value_grad(l: int, m: int, x, y, z):
    """R_lm and its gradient at arrays x, y, z (reference Y_lm convention)."""
    key = (l, m)
    if key not in _MONO_CACHE:
        _MONO_CACHE[key] = _solid_monomials(l, m)
    v = np.zeros_like(x)
    gx = np.zeros_like(x)
    gy = np.zeros_like(x)
    gz = np.zeros_like(x)
    for c, a, b, k in _MONO_CACHE[key]:
        xa, yb, zk = x**a, y**b, z**k
        v += c * xa * yb * zk
        if a:
            gx += c * a * x ** (a - 1) * yb * zk
        if b:
            gy += c * b * xa * y ** (b - 1) * zk
        if k:
            gz += c * k * xa * yb * z ** (k - 1)
    return v, gx, gy, gz


@dataclass
class Basis:
    """Per basis function: owning atom (0-based), l, m, Gaussian exponent."""

    atom: np.ndarray
    l: np.ndarray
    m: np.ndarray
    alpha: np.ndarray

    @property
    def n(self) -> int:
        return int(self.atom.shape[0])


def make_basis(n_atoms: int, shells: str, rng: np.random.Generator) -> Basis:
    """Functions numbered atom-major (so each batch's 1-based i_basis list,
    sorted ascending, groups functions by atom as atom_valid_n_compute_c_batches
    assumes).  Each shell gets its own log-uniform exponent in [0.1, 10]."""
    atom, ls, ms, al = [], [], [], []
    for a in range(n_atoms):
        for sh in shells:
            l = SHELL_L[sh]
            alpha = float(np.exp(rng.uniform(np.log(0.1), np.log(10.0))))
            for m in range(-l, l + 1):
                atom.append(a)
                ls.append(l)
                ms.append(m)
                al.append(alpha)
    return Basis(np.array(atom, np.int32), np.array(ls, np.int32), np.array(ms, np.int32), np.array(al))


def eval_basis(basis: Basis, funcs: np.ndarray, atoms_xyz: np.ndarray, pts: np.ndarray):
    """phi (nf, np) and grad phi (nf, 3, np) for functions `funcs` at points (np, 3)."""
    nf, npt = len(funcs), pts.shape[0]
    phi = np.zeros((nf, npt))
    gphi = np.zeros((nf, 3, npt))
    if nf == 0 or npt == 0:
        return phi, gphi
    rel = pts[None, :, :] - atoms_xyz[basis.atom[funcs]][:, None, :]
    x, y, z = rel[..., 0], rel[..., 1], rel[..., 2]
    r2 = x * x + y * y + z * z
    g = np.exp(-basis.alpha[funcs][:, None] * r2)
    for lm in set(zip(basis.l[funcs].tolist(), basis.m[funcs].tolist())):
        sel = np.nonzero((basis.l[funcs] == lm[0]) & (basis.m[funcs] == lm[1]))[0]
        v, gx, gy, gz = solid_harmonic_value_grad(lm[0], lm[1], x[sel], y[sel], z[sel])
        a2 = 2.0 * basis.alpha[funcs][sel][:, None]
        gs = g[sel]
        phi[sel] = v * gs
        gphi[sel, 0] = (gx - a2 * x[sel] * v) * gs
        gphi[sel, 1] = (gy - a2 * y[sel] * v) * gs
        gphi[sel, 2] = (gz - a2 * z[sel] * v) * gs
    return phi, gphi


def place_atoms(n_atoms: int, rng: np.random.Generator, box: float | None = None, density: float | None = None,
                min_dist: float = 1.0) -> np.ndarray:
    """Uniform positions, rejection-sampled to keep pairs >= min_dist apart."""
    if box is None:
        box = (n_atoms / density) ** (1.0 / 3.0)
    pos = np.zeros((n_atoms, 3))
    cell = max(min_dist, 1e-6)
    grid: dict = {}
    k = 0
    tries = 0
    while k < n_atoms:
        tries += 1
        if tries > 200 * n_atoms + 1000:
            raise RuntimeError("could not place atoms without overlap")
        p = rng.uniform(0.0, box, 3)
        key = tuple((p // cell).astype(int))
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for q in grid.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                        if np.sum((pos[q] - p) ** 2) < min_dist * min_dist:
                            ok = False
        if ok:
            pos[k] = p
            grid.setdefault(key, []).append(k)
            k += 1
    return pos


# --------------------------------------------------------------------------
# rho1 workloads
# --------------------------------------------------------------------------


@dataclass
class Rho1Problem:
    """All arguments of evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_
    (fast_rap_src_dfpt_gpu_eval/evaluate_first_order_rho.h:3-35), Fortran order."""

    T: int
    j_atom_begin: int
    j_atom_end: int
    j_coord: int
    n_my_batches_work: int
    n_full_points: int
    n_basis: int
    n_atoms: int
    n_max_compute_ham: int
    n_centers_basis_I: int
    n_max_batch_size: int
    batch_sizes: np.ndarray
    n_point_batches: np.ndarray
    n_point_batches_prefix_sum: np.ndarray
    i_valid_point_2_i_full_points_map: np.ndarray
    n_compute_c_batches: np.ndarray
    i_basis_batches: np.ndarray  # (n_centers_basis_I, n_batches) F
    atom_valid_n_compute_c_batches: np.ndarray  # (n_atoms + 1, n_batches) F
    i_batch_2_wave_offset: np.ndarray
    wave: np.ndarray | None
    gradient_wave: np.ndarray | None
    first_order_density_matrix: np.ndarray  # (n_basis, n_basis, T) F
    first_order_rho_bias_part2: np.ndarray  # (n_max_batch_size, n_batches, T) F
    first_order_gradient_rho_bias: np.ndarray  # (3, n_max_batch_size, n_batches, T) F
    basis_atom: np.ndarray
    partition_tab: np.ndarray
    density_matrix: np.ndarray | None
    # generator geometry (not part of the reference interface)
    atoms_xyz: np.ndarray = field(repr=False, default=None)
    basis: Basis = field(repr=False, default=None)
    valid_points_xyz: np.ndarray = field(repr=False, default=None)  # (n_valid, 3)

    @property
    def n_valid_points(self) -> int:
        return int(self.n_point_batches_prefix_sum[-1])

    @property
    def wave_len(self) -> int:
        return int(self.i_batch_2_wave_offset[self.n_my_batches_work])

    def total_points(self) -> int:
        return int(np.sum(self.n_point_batches[self.n_compute_c_batches > 0]))

    def flops(self, with_grad: bool = True) -> float:
        """FP64-equivalent flops: 2 T nc^2 np + 2 T nc np (+ 6 T nc np)."""
        nc = self.n_compute_c_batches.astype(np.float64)
        npt = self.n_point_batches.astype(np.float64)
        per = 2 * nc * nc * npt + (8 if with_grad else 2) * nc * npt
        return float(self.T * np.sum(per[nc > 0]))

    def algorithmic_bytes(self, with_grad: bool = True) -> float:
        """8 (nc np (1 + 3) + T nc^2 + T np (2 + 6)) + 4 (nc + np) per batch."""
        nc = self.n_compute_c_batches.astype(np.float64)
        npt = self.n_point_batches.astype(np.float64)
        g = 3 if with_grad else 0
        per = 8 * (nc * npt * (1 + g) + self.T * nc * nc + self.T * npt * (2 + (6 if with_grad else 0))) + 4 * (nc + npt)
        return float(np.sum(per[nc > 0]))


def make_rho1_problem(
    n_atoms: int = 8,
    shells: str = "ssssppdd",
    box: float | None = 6.0,
    density: float | None = None,
    n_batches: int = 64,
    np_range=(100, 200),
    nc_range=(40, 120),
    log_uniform: bool = False,
    T: int = 1,
    seed: int = 1,
    point_radius: float = 3.0,
    with_bias: bool = False,
    extra_full_points: int = 0,
    empty_batches: int = 0,
    pad_value: float = 0.0,
    p1_pattern: str = "dense",
    eval_phi: bool = True,
    n_active: int | None = None,
    exact_selection: bool | None = None,
    min_atom_dist: float = 1.0,
) -> Rho1Problem:
    """Build a rho1 workload.

    Config 1 of the benchmark suite is the default (8 atoms in a 6 A cube,
    20 functions per atom = 4 s + 2 p + 2 d, 64 batches of 100-200 points,
    n_compute 40-120, T = 1).  ``eval_phi=False`` leaves wave/gradient_wave
    unset so that a device generator can fill them.  ``pad_value`` fills the
    rows n_compute..n_compute_padding-1 of every batch (the reference never
    reads them; NaN there proves a kernel does not either).
    """
    rng = np.random.default_rng(seed)
    atoms = place_atoms(n_atoms, rng, box=box, density=density, min_dist=min_atom_dist)
    basis = make_basis(n_atoms, shells, rng)
    n_basis = basis.n

    def draw(lo, hi, size):
        if log_uniform:
            return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), size))).astype(np.int64).clip(lo, hi)
        return rng.integers(lo, hi + 1, size)

    npts = draw(np_range[0], np_range[1], n_batches)
    ncs = np.minimum(draw(nc_range[0], nc_range[1], n_batches), n_basis)
    if empty_batches:
        ncs[rng.choice(n_batches, size=empty_batches, replace=False)] = 0

    if exact_selection is None:
        exact_selection = n_basis * int(npts.mean()) <= 200_000

    # points of each batch: uniform in a ball around a random atom
    centre_atom = rng.integers(0, n_atoms, n_batches)
    tot = int(npts.sum())
    u = rng.normal(size=(tot, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    r = point_radius * rng.uniform(0, 1, tot) ** (1.0 / 3.0)
    owner = np.repeat(np.arange(n_batches), npts)
    all_pts = atoms[centre_atom[owner]] + u * r[:, None]
    starts = np.zeros(n_batches + 1, np.int64)
    starts[1:] = np.cumsum(npts)
    pts_list = [all_pts[starts[b]:starts[b + 1]] for b in range(n_batches)]

    # n_compute selection: the strongest functions over the batch
    atom_of = basis.atom
    ib_list = [None] * n_batches
    if exact_selection:
        for b in range(n_batches):
            nc = int(ncs[b])
            if nc == 0:
                ib_list[b] = np.zeros(0, np.int64)
                continue
            phi, _ = eval_basis(basis, np.arange(n_basis), atoms, pts_list[b])
            score = np.max(np.abs(phi), axis=1)
            ib_list[b] = np.sort(np.argpartition(-score, nc - 1)[:nc])
    else:
        # radial envelope max of r^l exp(-a r^2) over the batch ball, for the
        # functions of the atoms nearest the batch centre
        fpa = max(1, n_basis // n_atoms)
        k_near = int(min(n_atoms, max(8, 4 * int(ncs.max()) // fpa + 8)))
        funcs_of_atom = np.arange(n_basis).reshape(n_atoms, fpa) if n_basis == n_atoms * fpa else None
        chunk = 2048
        for b0 in range(0, n_batches, chunk):
            b1 = min(n_batches, b0 + chunk)
            c = atoms[centre_atom[b0:b1]]
            d_atom = np.linalg.norm(c[:, None, :] - atoms[None, :, :], axis=2)
            near = np.argpartition(d_atom, k_near - 1, axis=1)[:, :k_near]
            for bi, b in enumerate(range(b0, b1)):
                nc = int(ncs[b])
                if nc == 0:
                    ib_list[b] = np.zeros(0, np.int64)
                    continue
                cand = funcs_of_atom[near[bi]].ravel() if funcs_of_atom is not None else np.nonzero(np.isin(atom_of, near[bi]))[0]
                d = d_atom[bi, atom_of[cand]]
                lo, hi = np.maximum(d - point_radius, 0.0), d + point_radius
                lv = basis.l[cand].astype(np.float64)
                al = basis.alpha[cand]
                rstar = np.clip(np.sqrt(lv / (2 * al)), lo, hi)
                score_c = rstar**lv * np.exp(-al * rstar * rstar)
                nc = min(nc, len(cand))
                ncs[b] = nc
                ib_list[b] = np.sort(cand[np.argpartition(-score_c, nc - 1)[:nc]])

    n_max_compute_ham = int(max(1, ncs.max()))
    n_centers_basis_I = n_basis if n_basis * n_batches <= 50_000_000 else n_max_compute_ham
    i_basis = np.zeros((n_centers_basis_I, n_batches), np.int32, order="F")
    avn = np.zeros((n_atoms + 1, n_batches), np.int32, order="F")
    for b in range(n_batches):
        ib = ib_list[b]
        i_basis[: len(ib), b] = ib + 1
        counts = np.bincount(atom_of[ib], minlength=n_atoms) if len(ib) else np.zeros(n_atoms, np.int64)
        avn[1:, b] = np.cumsum(counts)

    prefix = np.zeros(n_batches + 1, np.int32)
    prefix[1:] = np.cumsum(npts)
    n_valid = int(prefix[-1])
    n_full = n_valid + extra_full_points
    perm = rng.permutation(n_full).astype(np.int32)
    vmap = perm[:n_valid].copy()
    # the rho entry point sizes this map n_full_points (evaluate_first_order_rho.cpp:63)
    map_full = np.concatenate([vmap, perm[n_valid:]]).astype(np.int32)
    valid_xyz = np.concatenate(pts_list, axis=0) if n_valid else np.zeros((0, 3))

    ncp = ((ncs + 3) // 4) * 4
    off = np.zeros(n_batches + 1, np.int64)
    off[1:] = np.cumsum(ncp * npts)
    if off[-1] >= 2**31:
        raise ValueError("wave offsets overflow int32 (the reference's index type)")
    off = off.astype(np.int32)

    wave = gwave = None
    if eval_phi:
        wave = np.full(int(off[-1]), pad_value)
        gwave = np.full(3 * int(off[-1]), pad_value)
        for b in range(n_batches):
            nc, npb = int(ncs[b]), int(npts[b])
            if nc == 0:
                continue
            phi, gphi = eval_basis(basis, ib_list[b], atoms, pts_list[b])
            w = wave[off[b] : off[b] + ncp[b] * npb].reshape(npb, ncp[b])  # (np, ncp) C = (ncp, np) F
            w[:, :nc] = phi.T
            gw = gwave[3 * off[b] : 3 * off[b] + 3 * ncp[b] * npb].reshape(npb, 3, ncp[b])
            gw[:, :, :nc] = np.transpose(gphi, (2, 1, 0))

    # first-order density matrix: symmetric, N(0,1)/sqrt(scale)
    P1 = np.zeros((n_basis, n_basis, T), order="F")
    if p1_pattern == "dense":
        scale = math.sqrt(n_basis)
        for t in range(T):
            a = rng.normal(size=(n_basis, n_basis)) / scale
            P1[:, :, t] = np.triu(a) + np.triu(a, 1).T
    else:  # within the batch-active pattern
        mask = np.zeros((n_atoms, n_atoms), bool)
        for b in range(n_batches):
            at = np.unique(atom_of[ib_list[b]])
            mask[at[:, None], at[None, :]] = True
        scale = math.sqrt(max(1.0, float(ncs[ncs > 0].mean())))
        full_mask = mask[np.ix_(atom_of, atom_of)]
        for t in range(T):
            a = rng.standard_normal(size=(n_basis, n_basis))
            a *= 1.0 / scale
            a = np.triu(a)
            a += np.triu(a, 1).T
            a[~full_mask] = 0.0
            P1[:, :, t] = a

    nmb = int(npts.max()) if n_batches else 1
    if with_bias:
        bias = np.asfortranarray(rng.uniform(-1, 1, (nmb, n_batches, T)))
        gbias = np.asfortranarray(rng.uniform(-1, 1, (3, nmb, n_batches, T)))
    else:
        bias = np.zeros((nmb, n_batches, T), order="F")
        gbias = np.zeros((3, nmb, n_batches, T), order="F")
    if n_active is None:
        n_active = T
    return Rho1Problem(
        T=T, j_atom_begin=1, j_atom_end=n_active, j_coord=1,
        n_my_batches_work=n_batches, n_full_points=n_full, n_basis=n_basis, n_atoms=n_atoms,
        n_max_compute_ham=n_max_compute_ham, n_centers_basis_I=n_centers_basis_I, n_max_batch_size=nmb,
        batch_sizes=npts.astype(np.int32), n_point_batches=npts.astype(np.int32),
        n_point_batches_prefix_sum=prefix, i_valid_point_2_i_full_points_map=map_full,
        n_compute_c_batches=ncs.astype(np.int32), i_basis_batches=i_basis, atom_valid_n_compute_c_batches=avn,
        i_batch_2_wave_offset=off, wave=wave, gradient_wave=gwave, first_order_density_matrix=P1,
        first_order_rho_bias_part2=bias, first_order_gradient_rho_bias=gbias,
        basis_atom=(basis.atom + 1).astype(np.int32), partition_tab=rng.uniform(0.01, 1.0, n_full),
        density_matrix=None, atoms_xyz=atoms, basis=basis, valid_points_xyz=valid_xyz,
    )


def first_order_h_inputs(prob: Rho1Problem, seed: int = 7, pad_value: float = 0.0) -> dict:
    """Seeded stand-ins for the exchange-correlation inputs of the first-order
    H integration (evaluate_first_order_H.cpp:13-53), in the reference's
    layouts: vsigma (3, nmb, nb), gradient_rho (3, n_full), hessian_wave
    (6 wave_len, rows past n_compute set to pad_value), H_prefactor1
    (nmb, nb, T), first_order_gradient_rho (3, nmb, nb, T), first_order_rho
    (n_full, T), v2rho2 (3, nmb, nb), v2rhosigma (6, nmb, nb), v2sigma2
    (6, nmb, nb).  Only their values matter for parity, so they are drawn
    N(0, 1) with mild scales rather than from a functional."""
    rng = np.random.default_rng(seed)
    nb, nmb, nf, T = prob.n_my_batches_work, prob.n_max_batch_size, prob.n_full_points, prob.T
    hess = rng.normal(size=6 * prob.wave_len)
    for b in range(nb):  # the padding rows of every (component, point) column
        nc, npb = int(prob.n_compute_c_batches[b]), int(prob.n_point_batches[b])
        ncp = (nc + 3) // 4 * 4
        if nc > 0 and ncp > nc:
            blk = hess[6 * int(prob.i_batch_2_wave_offset[b]):][: 6 * ncp * npb].reshape((ncp, 6 * npb), order="F")
            blk[nc:, :] = pad_value
    f = lambda *shape: np.asfortranarray(rng.normal(size=shape))  # noqa: E731
    return dict(vsigma=0.5 * f(3, nmb, nb), gradient_rho=f(3, nf), hessian_wave=hess,
                H_prefactor1=f(nmb, nb, T), first_order_gradient_rho=f(3, nmb, nb, T),
                first_order_rho=f(nf, T), v2rho2=0.3 * f(3, nmb, nb), v2rhosigma=0.2 * f(6, nmb, nb),
                v2sigma2=0.1 * f(6, nmb, nb))


def config1(seed: int = 1, **kw) -> Rho1Problem:
    """Benchmark config 1: the CPU-runnable plain FP64 case."""
    return make_rho1_problem(seed=seed, **kw)


def config2(seed: int = 2, n_batches: int = 30_000, eval_phi: bool = False, **kw) -> Rho1Problem:
    """Benchmark config 2: 1,000 atoms at 0.1 / A^3, 10 functions per atom
    (shells s, s, s, f so that l = 3 is exercised), 30,000 batches of 100-300
    points, n_compute 100-600, P1 within the batch-active pattern."""
    args = dict(n_atoms=1000, shells="sssf", box=None, density=0.1, n_batches=n_batches, np_range=(100, 300),
                nc_range=(100, 600), p1_pattern="active", eval_phi=eval_phi, exact_selection=False)
    args.update(kw)
    return make_rho1_problem(seed=seed, **args)


# --------------------------------------------------------------------------
# Sum-up workloads
# --------------------------------------------------------------------------


@dataclass
class SumupProblem:
    """All arguments of sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_
    (fast_rap_src_dfpt_gpu_eval/sum_up_whole_potential.h:3-48), Fortran order."""

    T: int
    j_atom_begin: int
    j_atom_end: int
    n_full_points: int
    l_max_analytic_multipole: int
    index_cc_dim_0: int
    n_valid_points: int
    l_pot_max: int
    n_max_radial: int
    n_hartree_grid: int
    n_centers: int
    n_centers_hartree_potential: int
    n_atoms: int
    hartree_force_l_add: int
    n_species: int
    n_radial: np.ndarray
    species: np.ndarray
    species_center: np.ndarray
    l_hartree_max_far_distance: np.ndarray  # (n_atoms, T)
    i_valid_point_2_i_full_points_map: np.ndarray
    coord_points: np.ndarray  # (3, n_full_points)
    multipole_radius_sq: np.ndarray  # (n_atoms, T)
    outer_potential_radius: np.ndarray  # (l_pot_max + 1, n_atoms, T)
    multipole_moments: np.ndarray  # ((l_pot_max+1)^2, n_atoms, T)
    spline: np.ndarray  # ((l_pot_max+1)^2, 2, n_hartree_grid, n_atoms, T)
    l_hartree: np.ndarray
    n_grid: np.ndarray
    n_cc_lm_ijk: np.ndarray
    centers_hartree_potential: np.ndarray
    center_to_atom: np.ndarray
    index_cc: np.ndarray  # (index_cc_dim_0, 6)
    index_ijk_max_cc: np.ndarray  # (3, l_max_analytic_multipole + 1)
    cc: np.ndarray
    coords_center: np.ndarray  # (3, n_centers)
    r_grid_min: np.ndarray
    log_r_grid_inc: np.ndarray
    scale_radial: np.ndarray
    partition_tab: np.ndarray
    delta_v_hartree: np.ndarray  # (n_full_points, T), accumulated into

    def pair_count(self) -> int:
        return self.n_valid_points * self.n_centers_hartree_potential * max(0, min(self.T, self.j_atom_end - self.j_atom_begin + 1))


def make_sumup_problem(
    n_atoms: int = 20,
    n_points: int = 2000,
    l_pot_max: int = 6,
    T: int = 1,
    seed: int = 3,
    density: float = 0.1,
    near_radius: float = 2.0,
    outer_radius: float | None = 6.0,
    l_hartree_per_species=None,
    n_species: int = 4,
    n_hartree_grid: int = 1301,
    extra_full_points: int = 0,
    centers: str = "identity",
    hartree_force_l_add: int = 1,
    margin: float = 3.0,
    n_active: int | None = None,
    spline_scale: float = 1.0,
    with_spline: bool = True,
    min_atom_dist: float = 1.0,
) -> SumupProblem:
    """Build a sum-up workload.  Config 3 of the benchmark suite is
    n_atoms=500, n_points=2e6, l_pot_max in {4, 6, 8}, outer_radius=None
    (no l truncation: l_atom_max = l_max), near_radius = 2 A."""
    rng = np.random.default_rng(seed)
    L = l_pot_max
    L2 = (L + 1) ** 2
    lma = L + 1
    index_cc, cc, n_cc, ijk_max = (np.array(a, order="F", copy=True) for a in tables.multipole_tables(lma))
    atoms = place_atoms(n_atoms, rng, density=density, min_dist=min_atom_dist)
    box = (n_atoms / density) ** (1.0 / 3.0)
    n_full = n_points + extra_full_points
    coords = np.asfortranarray(rng.uniform(-margin, box + margin, (3, n_full)))
    perm = rng.permutation(n_full).astype(np.int32)
    vmap = perm[:n_points].copy()

    species = rng.integers(1, n_species + 1, n_atoms).astype(np.int32)
    if l_hartree_per_species is None:
        l_hartree = np.full(n_species, L, np.int32)
    else:
        l_hartree = np.asarray(l_hartree_per_species, np.int32)
    n_grid = np.full(n_species, n_hartree_grid, np.int32)
    r_grid_min = np.full(n_species, 1e-4) * rng.uniform(0.5, 2.0, n_species)
    log_r_grid_inc = np.log(1e6) / (n_hartree_grid - 1) * rng.uniform(0.95, 1.05, n_species)

    if centers == "identity":
        n_centers = n_atoms
        center_to_atom = np.arange(1, n_atoms + 1, dtype=np.int32)
        chp = np.arange(1, n_atoms + 1, dtype=np.int32)
    elif centers == "permuted":
        # more centres than atoms (periodic images) and a permuted subset with
        # potential, which exercises the reference's use of the loop slot in
        # the far field (sum_up_whole_potential.cpp:161-162,183)
        n_centers = n_atoms + n_atoms // 2
        center_to_atom = np.concatenate([np.arange(1, n_atoms + 1), rng.integers(1, n_atoms + 1, n_centers - n_atoms)]).astype(np.int32)
        chp = (rng.permutation(n_centers)[: n_atoms] + 1).astype(np.int32)
    else:
        raise ValueError(centers)
    coords_center = np.asfortranarray(atoms[center_to_atom - 1].T.copy())
    if centers == "permuted":
        coords_center[:, n_atoms:] += rng.uniform(-5, 5, (3, n_centers - n_atoms))
    species_center = species[center_to_atom - 1].copy()

    lhmfd = np.asfortranarray(np.repeat(l_hartree[species - 1][:, None], T, axis=1).astype(np.int32))
    mrs = np.asfortranarray(np.full((n_atoms, T), near_radius**2) * rng.uniform(0.9, 1.1, (n_atoms, T)))
    if outer_radius is None:
        opr = np.full((L + 1, n_atoms, T), 1e30, order="F")
    else:
        base = outer_radius * rng.uniform(0.8, 1.2, (1, n_atoms, T))
        opr = np.asfortranarray((base / (1.0 + 0.15 * np.arange(L + 1))[:, None, None]) ** 2)
    q = np.zeros((L2, n_atoms, T), order="F")
    for l in range(L + 1):
        q[l * l : (l + 1) * (l + 1)] = rng.normal(size=(2 * l + 1, n_atoms, T)) * 10.0**-l
    # a few moments below the reference's 1e-10 threshold
    tiny = rng.random(q.shape) < 0.02
    q[tiny] = 1e-12
    if with_spline:
        spline = np.asfortranarray(rng.uniform(-1, 1, (L2, 2, n_hartree_grid, n_atoms, T)) * spline_scale)
    else:
        spline = np.zeros((L2, 2, n_hartree_grid, n_atoms, T), order="F")
    dv = np.asfortranarray(rng.uniform(-1, 1, (n_full, T)))
    if n_active is None:
        n_active = T
    return SumupProblem(
        T=T, j_atom_begin=1, j_atom_end=n_active, n_full_points=n_full, l_max_analytic_multipole=lma,
        index_cc_dim_0=int(n_cc[lma]), n_valid_points=n_points, l_pot_max=L, n_max_radial=n_hartree_grid,
        n_hartree_grid=n_hartree_grid, n_centers=n_centers, n_centers_hartree_potential=len(chp),
        n_atoms=n_atoms, hartree_force_l_add=hartree_force_l_add, n_species=n_species,
        n_radial=np.full(n_species, n_hartree_grid, np.int32), species=species, species_center=species_center,
        l_hartree_max_far_distance=lhmfd, i_valid_point_2_i_full_points_map=vmap, coord_points=coords,
        multipole_radius_sq=mrs, outer_potential_radius=opr, multipole_moments=q, spline=spline,
        l_hartree=l_hartree, n_grid=n_grid, n_cc_lm_ijk=n_cc, centers_hartree_potential=chp,
        center_to_atom=center_to_atom, index_cc=index_cc, index_ijk_max_cc=ijk_max, cc=cc,
        coords_center=coords_center, r_grid_min=r_grid_min, log_r_grid_inc=log_r_grid_inc,
        scale_radial=np.ones(n_species), partition_tab=rng.uniform(0.01, 1.0, n_full), delta_v_hartree=dv,
    )


def config3(l_max: int = 6, seed: int = 4, n_atoms: int = 500, n_points: int = 2_000_000, **kw) -> SumupProblem:
    """Benchmark config 3: 500 atoms, 2e6 points, l_max in {4, 6, 8}."""
    args = dict(outer_radius=None, near_radius=2.0, spline_scale=1e-2)
    args.update(kw)
    return make_sumup_problem(n_atoms=n_atoms, n_points=n_points, l_pot_max=l_max, seed=seed, **args)


def subset_batches(prob: Rho1Problem, n_batches: int, wave=None, gradient_wave=None) -> Rho1Problem:
    """The first ``n_batches`` batches of ``prob`` as a standalone problem whose
    points are renumbered 0..n-1 (the identity valid-to-full map).  ``wave`` /
    ``gradient_wave`` default to prob's arrays cut to the subset's extent."""
    nb = int(min(n_batches, prob.n_my_batches_work))
    pre = prob.n_point_batches_prefix_sum[: nb + 1].astype(np.int32).copy()
    off = prob.i_batch_2_wave_offset[: nb + 1].astype(np.int32).copy()
    n_valid, wl = int(pre[-1]), int(off[-1])
    w = (prob.wave if wave is None else wave)[:wl]
    gw = (prob.gradient_wave if gradient_wave is None else gradient_wave)[: 3 * wl]
    T = prob.T
    return Rho1Problem(
        T=T, j_atom_begin=prob.j_atom_begin, j_atom_end=prob.j_atom_end, j_coord=prob.j_coord, n_my_batches_work=nb,
        n_full_points=max(1, n_valid), n_basis=prob.n_basis, n_atoms=prob.n_atoms,
        n_max_compute_ham=prob.n_max_compute_ham, n_centers_basis_I=prob.n_centers_basis_I,
        n_max_batch_size=prob.n_max_batch_size, batch_sizes=prob.batch_sizes[:nb].copy(),
        n_point_batches=prob.n_point_batches[:nb].copy(), n_point_batches_prefix_sum=pre,
        i_valid_point_2_i_full_points_map=np.arange(max(1, n_valid), dtype=np.int32),
        n_compute_c_batches=prob.n_compute_c_batches[:nb].copy(),
        i_basis_batches=np.asfortranarray(prob.i_basis_batches[:, :nb]),
        atom_valid_n_compute_c_batches=np.asfortranarray(prob.atom_valid_n_compute_c_batches[:, :nb]),
        i_batch_2_wave_offset=off, wave=np.ascontiguousarray(w), gradient_wave=np.ascontiguousarray(gw),
        first_order_density_matrix=prob.first_order_density_matrix,
        first_order_rho_bias_part2=np.asfortranarray(prob.first_order_rho_bias_part2[:, :nb, :]),
        first_order_gradient_rho_bias=np.asfortranarray(prob.first_order_gradient_rho_bias[:, :, :nb, :]),
        basis_atom=prob.basis_atom, partition_tab=np.ones(max(1, n_valid)), density_matrix=None,
        atoms_xyz=prob.atoms_xyz, basis=prob.basis,
        valid_points_xyz=None if prob.valid_points_xyz is None else prob.valid_points_xyz[:n_valid],
    )


def host_basis_values(prob: Rho1Problem, n_batches: int | None = None, pad_value: float = 0.0):
    """Host (numpy) wave / gradient_wave for the first ``n_batches`` batches."""
    nb = prob.n_my_batches_work if n_batches is None else int(n_batches)
    wl = int(prob.i_batch_2_wave_offset[nb])
    wave = np.full(wl, pad_value)
    gwave = np.full(3 * wl, pad_value)
    pre, off = prob.n_point_batches_prefix_sum, prob.i_batch_2_wave_offset
    for b in range(nb):
        nc, npb = int(prob.n_compute_c_batches[b]), int(prob.n_point_batches[b])
        if nc == 0 or npb == 0:
            continue
        ncp = (nc + 3) // 4 * 4
        ib = prob.i_basis_batches[:nc, b] - 1
        phi, gphi = eval_basis(prob.basis, ib, prob.atoms_xyz, prob.valid_points_xyz[pre[b]:pre[b] + npb])
        wave[off[b]:off[b] + ncp * npb].reshape(npb, ncp)[:, :nc] = phi.T
        gwave[3 * off[b]:3 * off[b] + 3 * ncp * npb].reshape(npb, 3, ncp)[:, :, :nc] = np.transpose(gphi, (2, 1, 0))
    return wave, gwave


# --------------------------------------------------------------------------
# Config 4: the config-1 recipe swept to thousands of atoms
# --------------------------------------------------------------------------


@dataclass
class SweepGeometry:
    """Atoms, basis and batches of a config-4 sweep.  Batches are ordered so
    that consecutive ones sit near each other (6 A cells), which keeps the
    basis window of a chunk of batches small."""

    atoms: np.ndarray  # (n_atoms, 3)
    basis: Basis
    centre: np.ndarray  # centre atom of each batch
    npts: np.ndarray
    ncs: np.ndarray
    ib: list  # selected functions (global, sorted) per batch
    seed: int
    point_radius: float = 3.0

    @property
    def n_batches(self) -> int:
        return int(len(self.centre))


def config4_geometry(n_atoms: int, seed: int = 4, batches_per_atom: int = 8, np_range=(50, 400),
                     nc_range=(50, 800), density: float = 8 / 216.0, shells: str = "ssssppdd") -> SweepGeometry:
    """Config 4: the config-1 recipe (20 functions per atom: 4 s + 2 p + 2 d,
    Gaussian radials, density of config 1) at ``n_atoms`` atoms, 8 batches per
    atom, points per batch and n_compute log-uniform over 50-400 and 50-800
    (n_compute chosen as the strongest functions by radial envelope over the
    batch ball among the nearest atoms)."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    atoms = place_atoms(n_atoms, rng, density=density, min_dist=1.0)
    basis = make_basis(n_atoms, shells, rng)
    fpa = basis.n // n_atoms
    centre = np.repeat(np.arange(n_atoms), batches_per_atom)
    cell = np.floor(atoms[centre] / 6.0).astype(np.int64)
    centre = centre[np.lexsort((cell[:, 2], cell[:, 1], cell[:, 0]))]
    nb = len(centre)

    def logu(lo, hi):
        return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), nb))).astype(np.int64).clip(lo, hi)

    npts, ncs = logu(*np_range), logu(*nc_range)
    k_near = int(min(n_atoms, 2 * int(ncs.max()) // fpa + 8))
    tree = cKDTree(atoms)
    ib = [None] * nb
    funcs_of_atom = np.arange(basis.n).reshape(n_atoms, fpa)
    radius = 3.0
    for b0 in range(0, nb, 4096):
        b1 = min(nb, b0 + 4096)
        d_near, near = tree.query(atoms[centre[b0:b1]], k=k_near)
        for k, b in enumerate(range(b0, b1)):
            cand = funcs_of_atom[near[k]].ravel()
            d = np.repeat(d_near[k], fpa)
            lo, hi = np.maximum(d - radius, 0.0), d + radius
            lv = basis.l[cand].astype(np.float64)
            al = basis.alpha[cand]
            rstar = np.clip(np.sqrt(lv / (2 * al)), lo, hi)
            score = rstar**lv * np.exp(-al * rstar * rstar)
            nc = int(min(ncs[b], len(cand)))
            ncs[b] = nc
            ib[b] = np.sort(cand[np.argpartition(-score, nc - 1)[:nc]])
    return SweepGeometry(atoms=atoms, basis=basis, centre=centre, npts=npts, ncs=ncs, ib=ib, seed=seed,
                         point_radius=radius)


def sweep_chunks(geom: SweepGeometry, max_batches: int = 5000, max_window: int = 24000):
    """Consecutive batch ranges [b0, b1) whose basis window (union of their
    compute functions) has at most max_window functions."""
    chunks, b0 = [], 0
    nb = geom.n_batches
    while b0 < nb:
        seen = set()
        b1 = b0
        while b1 < nb and b1 - b0 < max_batches:
            new = seen.union(geom.ib[b1].tolist())
            if len(new) > max_window and b1 > b0:
                break
            seen = new
            b1 += 1
        chunks.append((b0, b1))
        b0 = b1
    return chunks


def sweep_chunk_problem(geom: SweepGeometry, b0: int, b1: int) -> tuple[Rho1Problem, np.ndarray]:
    """Batches [b0, b1) of a sweep as a standalone rho1 problem over its basis
    window U (returned as the global 0-based indices of the window's
    functions): points drawn per batch from a generator keyed by (seed, b0),
    phi / grad phi left to the device generator, P1 left to
    frpa_synth_p1_window over U, biases zero, T = 1."""
    ids = np.arange(b0, b1)
    U = np.unique(np.concatenate([geom.ib[b] for b in ids]))
    atoms_u = np.unique(geom.basis.atom[U])
    basis_u = Basis(np.searchsorted(atoms_u, geom.basis.atom[U]).astype(np.int32), geom.basis.l[U],
                    geom.basis.m[U], geom.basis.alpha[U])
    rng = np.random.default_rng([geom.seed, b0])
    npts = geom.npts[ids].astype(np.int64)
    ncs = geom.ncs[ids].astype(np.int64)
    tot = int(npts.sum())
    u = rng.normal(size=(tot, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    r = geom.point_radius * rng.uniform(0, 1, tot) ** (1.0 / 3.0)
    owner = np.repeat(np.arange(len(ids)), npts)
    pts = geom.atoms[geom.centre[ids][owner]] + u * r[:, None]
    nb = len(ids)
    nmc = int(max(1, ncs.max()))
    i_basis = np.zeros((nmc, nb), np.int32, order="F")
    avn = np.zeros((len(atoms_u) + 1, nb), np.int32, order="F")
    for k, b in enumerate(ids):
        loc = np.searchsorted(U, geom.ib[b])
        i_basis[: len(loc), k] = loc + 1
        avn[1:, k] = np.cumsum(np.bincount(basis_u.atom[loc], minlength=len(atoms_u)))
    prefix = np.zeros(nb + 1, np.int32)
    prefix[1:] = np.cumsum(npts)
    ncp = ((ncs + 3) // 4) * 4
    off = np.zeros(nb + 1, np.int64)
    off[1:] = np.cumsum(ncp * npts)
    if off[-1] >= 2**31:
        raise ValueError("chunk too large for int32 wave offsets")
    nmb = int(npts.max())
    prob = Rho1Problem(
        T=1, j_atom_begin=1, j_atom_end=1, j_coord=1, n_my_batches_work=nb, n_full_points=max(1, tot),
        n_basis=len(U), n_atoms=len(atoms_u), n_max_compute_ham=nmc, n_centers_basis_I=nmc, n_max_batch_size=nmb,
        batch_sizes=npts.astype(np.int32), n_point_batches=npts.astype(np.int32), n_point_batches_prefix_sum=prefix,
        i_valid_point_2_i_full_points_map=np.arange(max(1, tot), dtype=np.int32),
        n_compute_c_batches=ncs.astype(np.int32), i_basis_batches=i_basis, atom_valid_n_compute_c_batches=avn,
        i_batch_2_wave_offset=off.astype(np.int32), wave=None, gradient_wave=None,
        first_order_density_matrix=np.zeros((1, 1, 1), order="F"),
        first_order_rho_bias_part2=np.zeros((nmb, nb, 1), order="F"),
        first_order_gradient_rho_bias=np.zeros((3, nmb, nb, 1), order="F"),
        basis_atom=(basis_u.atom + 1).astype(np.int32), partition_tab=np.ones(max(1, tot)), density_matrix=None,
        atoms_xyz=geom.atoms[atoms_u], basis=basis_u, valid_points_xyz=pts)
    return prob, U.astype(np.int32)
