"""CPU parity oracle bindings (TEST INFRASTRUCTURE).

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg, as the checker.  Two back ends:

* ``liboracle.so``: this project's plain-C restatement (frpa_oracle.c);
* ``_ref/libref_tN.so``: the reference's own CPU sources compiled in place
  for ATOM_TILE_SIZE = N (see Makefile).  ``ref_available()`` says whether
  they were built.

All functions take the problem dataclasses of fast_rpa_eval_b200.synth and
return fresh numpy arrays in the reference's Fortran layouts.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lock = threading.Lock()
_libs: dict = {}

c_int = ctypes.c_int
c_int_p = ctypes.POINTER(ctypes.c_int)
c_dbl_p = ctypes.POINTER(ctypes.c_double)
c_u8_p = ctypes.POINTER(ctypes.c_ubyte)


def reference_tree() -> str:
    """The reference checkout: $FR_REF, else the directory `reference` beside
    this repository (the layout the build container has)."""
    return os.environ.get("FR_REF") or os.path.join(os.path.dirname(os.path.dirname(_HERE)), "reference")


def build(with_reference: bool | None = None) -> None:
    """Compile liboracle.so (and the reference libraries where the reference
    tree is present)."""
    targets = ["oracle"]
    ref = reference_tree()
    if with_reference is None:
        with_reference = os.path.isdir(os.path.join(ref, "fast_rap_src_dfpt_gpu_eval"))
    if with_reference:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", _HERE, "FR_REF=" + os.path.abspath(ref)] + targets, check=True)


def _load(name: str):
    with _lock:
        if name not in _libs:
            path = os.path.join(_HERE, name)
            if not os.path.exists(path):
                if name == "liboracle.so":
                    build(with_reference=False)
                else:
                    raise FileNotFoundError(path)
            _libs[name] = ctypes.CDLL(path)
        return _libs[name]


def ref_available(T: int = 1) -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", f"libref_t{T}.so"))


def _i(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel(order="F"))
    return a, a.ctypes.data_as(c_int_p)


def _d(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))
    return a, a.ctypes.data_as(c_dbl_p)


class _Args:
    """Keeps converted arrays alive for the duration of a call."""

    def __init__(self):
        self.keep = []

    def i(self, a):
        arr, p = _i(a)
        self.keep.append(arr)
        return p

    def d(self, a):
        arr, p = _d(a)
        self.keep.append(arr)
        return p


# --------------------------------------------------------------------------
# rho1
# --------------------------------------------------------------------------


def rho1(prob, n_threads: int = 1, use_reference: bool = False):
    """(first_order_rho (n_full, T), first_order_gradient_rho (3, nmb, nb, T))."""
    T = prob.T
    rho = np.zeros(prob.n_full_points * T)
    grad = np.zeros(3 * prob.n_max_batch_size * prob.n_my_batches_work * T)
    A = _Args()
    if not use_reference:
        lib = _load("liboracle.so")
        lib.oracle_rho1(
            c_int(T), c_int(prob.n_my_batches_work), c_int(prob.j_atom_begin), c_int(prob.j_atom_end),
            c_int(prob.n_full_points), c_int(prob.n_basis), c_int(prob.n_atoms), c_int(prob.n_max_compute_ham),
            c_int(prob.n_centers_basis_I), c_int(prob.n_max_batch_size), A.i(prob.batch_sizes),
            A.i(prob.n_point_batches), A.i(prob.n_point_batches_prefix_sum),
            A.i(prob.i_valid_point_2_i_full_points_map), A.i(prob.n_compute_c_batches), A.i(prob.i_basis_batches),
            A.i(prob.i_batch_2_wave_offset), A.d(prob.wave), A.d(prob.gradient_wave),
            A.d(prob.first_order_density_matrix), rho.ctypes.data_as(c_dbl_p), A.d(prob.first_order_rho_bias_part2),
            grad.ctypes.data_as(c_dbl_p), A.d(prob.first_order_gradient_rho_bias), c_int(n_threads))
    else:
        lib = _load(os.path.join("_ref", f"libref_t{T}.so"))
        ints = [prob.n_my_batches_work, prob.j_atom_begin, prob.j_atom_end, prob.j_coord, prob.n_full_points,
                prob.n_basis, prob.n_atoms, prob.n_max_compute_ham, prob.n_centers_basis_I, prob.n_max_batch_size]
        scal = [ctypes.byref(c_int(int(v))) for v in ints]
        dm = prob.density_matrix if prob.density_matrix is not None else np.zeros(1)
        lib.evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_(
            *scal, A.i(prob.batch_sizes), A.i(prob.n_point_batches), A.i(prob.n_point_batches_prefix_sum),
            A.i(prob.i_valid_point_2_i_full_points_map), A.i(prob.n_compute_c_batches), A.i(prob.i_basis_batches),
            A.i(prob.atom_valid_n_compute_c_batches), A.i(prob.i_batch_2_wave_offset), A.d(prob.wave),
            A.d(prob.gradient_wave), A.d(prob.first_order_density_matrix), rho.ctypes.data_as(c_dbl_p),
            A.d(prob.first_order_rho_bias_part2), grad.ctypes.data_as(c_dbl_p),
            A.d(prob.first_order_gradient_rho_bias), A.i(prob.basis_atom), A.d(prob.partition_tab), A.d(dm))
    return (rho.reshape((prob.n_full_points, T), order="F"),
            grad.reshape((3, prob.n_max_batch_size, prob.n_my_batches_work, T), order="F"))


# --------------------------------------------------------------------------
# sum-up
# --------------------------------------------------------------------------


def sumup(prob, n_threads: int = 1, use_reference: bool = False, branch_codes: bool = False, delta_v=None):
    """delta_v_hartree after the reference's accumulation, starting from
    ``delta_v`` (default prob.delta_v_hartree).  With branch_codes=True also
    returns the per-(valid point, centre slot, tile) branch codes."""
    T = prob.T
    dv = np.array(prob.delta_v_hartree if delta_v is None else delta_v, dtype=np.float64).ravel(order="F").copy()
    A = _Args()
    codes = None
    if not use_reference:
        lib = _load("liboracle.so")
        codes_p = None
        if branch_codes:
            codes = np.zeros(prob.n_valid_points * prob.n_centers_hartree_potential * T, np.uint8)
            codes_p = codes.ctypes.data_as(c_u8_p)
        lib.oracle_sumup(
            c_int(T), c_int(prob.j_atom_begin), c_int(prob.j_atom_end), c_int(prob.n_full_points),
            c_int(prob.l_max_analytic_multipole), c_int(prob.index_cc_dim_0), c_int(prob.n_valid_points),
            c_int(prob.l_pot_max), c_int(prob.n_hartree_grid), c_int(prob.n_centers),
            c_int(prob.n_centers_hartree_potential), c_int(prob.n_atoms), c_int(prob.hartree_force_l_add),
            c_int(prob.n_species), A.i(prob.species), A.i(prob.species_center),
            A.i(prob.l_hartree_max_far_distance), A.i(prob.i_valid_point_2_i_full_points_map),
            A.d(prob.coord_points), A.d(prob.multipole_radius_sq), A.d(prob.outer_potential_radius),
            A.d(prob.multipole_moments), A.d(prob.spline), A.i(prob.l_hartree), A.i(prob.n_grid),
            A.i(prob.n_cc_lm_ijk), A.i(prob.centers_hartree_potential), A.i(prob.center_to_atom),
            A.i(prob.index_cc), A.i(prob.index_ijk_max_cc), A.d(prob.cc), A.d(prob.coords_center),
            A.d(prob.r_grid_min), A.d(prob.log_r_grid_inc), dv.ctypes.data_as(c_dbl_p), codes_p, c_int(n_threads))
    else:
        lib = _load(os.path.join("_ref", f"libref_t{T}.so"))
        ints = [prob.j_atom_begin, prob.j_atom_end, prob.n_full_points, prob.l_max_analytic_multipole,
                prob.index_cc_dim_0, prob.n_valid_points, prob.l_pot_max, prob.n_max_radial, prob.n_hartree_grid,
                prob.n_centers, prob.n_centers_hartree_potential, prob.n_atoms, prob.hartree_force_l_add,
                prob.n_species]
        scal = [ctypes.byref(c_int(int(v))) for v in ints]
        lib.sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_(
            *scal, A.i(prob.n_radial), A.i(prob.species), A.i(prob.species_center),
            A.i(prob.l_hartree_max_far_distance), A.i(prob.i_valid_point_2_i_full_points_map),
            A.d(prob.coord_points), A.d(prob.multipole_radius_sq), A.d(prob.outer_potential_radius),
            A.d(prob.multipole_moments), A.d(prob.spline), A.i(prob.l_hartree), A.i(prob.n_grid),
            A.i(prob.n_cc_lm_ijk), A.i(prob.centers_hartree_potential), A.i(prob.center_to_atom),
            A.i(prob.index_cc), A.i(prob.index_ijk_max_cc), A.d(prob.cc), A.d(prob.coords_center),
            A.d(prob.r_grid_min), A.d(prob.log_r_grid_inc), A.d(prob.scale_radial), A.d(prob.partition_tab),
            dv.ctypes.data_as(c_dbl_p))
    out = dv.reshape((prob.n_full_points, T), order="F")
    if branch_codes:
        return out, codes.reshape((prob.n_valid_points, prob.n_centers_hartree_potential, T), order="F")
    return out


def ylm(l_max: int, x: float, y: float, z: float, use_reference: bool = False, trig=None):
    """Real Y_lm (l*l + l + m).  The reference variant takes (sin t, cos t,
    sin p, cos p) through ``trig``."""
    out = np.zeros((l_max + 1) ** 2)
    if use_reference:
        lib = _load(os.path.join("_ref", "libref_t1.so"))
        st, ct, sp, cp = trig
        lib.ref_sheval(c_int(l_max), ctypes.c_double(st), ctypes.c_double(ct), ctypes.c_double(sp),
                       ctypes.c_double(cp), out.ctypes.data_as(c_dbl_p))
    else:
        lib = _load("liboracle.so")
        lib.oracle_ylm(c_int(l_max), ctypes.c_double(x), ctypes.c_double(y), ctypes.c_double(z),
                       out.ctypes.data_as(c_dbl_p))
    return out


def far_field_spherical(l_max: int, points_3xn, atoms_3xn, Q_lm_by_atom):
    lib = _load("liboracle.so")
    A = _Args()
    n_points = points_3xn.shape[1]
    out = np.zeros(n_points)
    lib.oracle_far_field_spherical(c_int(l_max), c_int(n_points), A.d(points_3xn), c_int(atoms_3xn.shape[1]),
                                   A.d(atoms_3xn), A.d(Q_lm_by_atom), out.ctypes.data_as(c_dbl_p))
    return out


# --------------------------------------------------------------------------
# first-order H (the rho1 adjoint with XC terms zero) and the bias producer
# --------------------------------------------------------------------------


def first_order_h(prob, v, use_reference: bool = False, w=None, xc=None, j_coord: int | None = None):
    """H (n_basis, n_basis, T) accumulated from 0 by the first-order-H
    integration (evaluate_first_order_H.cpp:13-222).  ``v`` is
    v_hartree_gradient (n_full_points, T); ``w`` defaults to
    prob.partition_tab.  ``xc`` (optional) holds the other inputs in the
    reference's layouts: vsigma (3, nmb, nb), gradient_rho (3, n_full),
    hessian_wave (6 wave_len), H_prefactor1 (nmb, nb, T),
    first_order_gradient_rho (3, nmb, nb, T), first_order_rho (n_full, T),
    v2rho2 (3, nmb, nb), v2rhosigma (6, nmb, nb), v2sigma2 (6, nmb, nb);
    absent ones are zero."""
    T = prob.T
    w = prob.partition_tab if w is None else w
    jc = prob.j_coord if j_coord is None else j_coord
    nb, nmb, nfull = prob.n_my_batches_work, prob.n_max_batch_size, prob.n_full_points
    xc = dict(xc or {})
    shapes = dict(vsigma=3 * nmb * nb, gradient_rho=3 * nfull, hessian_wave=6 * prob.wave_len,
                  H_prefactor1=nmb * nb * T, first_order_gradient_rho=3 * nmb * nb * T, first_order_rho=nfull * T,
                  v2rho2=3 * nmb * nb, v2rhosigma=6 * nmb * nb, v2sigma2=6 * nmb * nb)
    arr = {k: (np.asarray(xc[k], dtype=np.float64).ravel(order="F") if k in xc else np.zeros(max(1, n)))
           for k, n in shapes.items()}
    H = np.zeros(prob.n_basis * prob.n_basis * T)
    A = _Args()
    if not use_reference:
        lib = _load("liboracle.so")
        lib.oracle_first_order_h(
            c_int(T), c_int(nb), c_int(prob.j_atom_begin), c_int(prob.j_atom_end), c_int(nfull), c_int(jc),
            c_int(prob.n_basis), c_int(nmb), c_int(prob.n_centers_basis_I), A.i(prob.n_point_batches),
            A.i(prob.n_compute_c_batches), A.i(prob.i_basis_batches), A.i(prob.atom_valid_n_compute_c_batches),
            c_int(prob.n_atoms), A.i(prob.n_point_batches_prefix_sum), A.i(prob.i_valid_point_2_i_full_points_map),
            A.d(arr["vsigma"]), A.d(arr["gradient_rho"]), A.i(prob.i_batch_2_wave_offset), A.d(prob.wave),
            A.d(prob.gradient_wave), A.d(arr["hessian_wave"]), A.d(arr["H_prefactor1"]),
            A.d(arr["first_order_gradient_rho"]), A.d(v), A.d(arr["first_order_rho"]), A.d(arr["v2rho2"]),
            A.d(arr["v2rhosigma"]), A.d(arr["v2sigma2"]), A.d(w), H.ctypes.data_as(c_dbl_p))
    else:
        lib = _load(os.path.join("_ref", f"libref_t{T}.so"))
        ints = [prob.j_atom_begin, prob.j_atom_end, nfull, jc, prob.n_basis, prob.n_atoms,
                prob.n_max_compute_ham, nmb, nb, prob.n_centers_basis_I]
        scal = [ctypes.byref(c_int(int(v_))) for v_ in ints]
        not_use = c_int(0)
        z = lambda n: np.zeros(max(1, n))  # noqa: E731
        lib.evaluate_first_order_h_reduce_memory_c_v2_(
            *scal, A.i(prob.n_point_batches), A.i(prob.n_compute_c_batches), A.i(prob.i_basis_batches),
            A.i(prob.atom_valid_n_compute_c_batches), A.i(prob.n_point_batches_prefix_sum),
            A.i(prob.i_valid_point_2_i_full_points_map),
            A.d(z(nmb * nb)), A.d(arr["vsigma"]), A.d(arr["gradient_rho"]),
            A.d(z(prob.wave_len)), A.i(prob.i_batch_2_wave_offset), A.d(prob.wave), A.d(prob.gradient_wave),
            A.d(arr["hessian_wave"]), H.ctypes.data_as(c_dbl_p), A.d(arr["H_prefactor1"]),
            A.d(arr["first_order_gradient_rho"]), A.d(v), A.d(arr["first_order_rho"]), A.d(arr["v2rho2"]),
            A.d(arr["v2rhosigma"]), A.d(arr["v2sigma2"]), A.d(w), ctypes.byref(not_use))
    return H.reshape((prob.n_basis, prob.n_basis, T), order="F")


def rho_bias_part2(prob, density_matrix, T: int = 4, use_reference: bool = False, j_coord: int = 1):
    """first_order_rho_bias_part2 (n_max_batch_size, n_batches, T); the
    reference producer fixes T = 4."""
    nmb, nb = prob.n_max_batch_size, prob.n_my_batches_work
    out = np.zeros(nmb * nb * T)
    A = _Args()
    if not use_reference:
        lib = _load("liboracle.so")
        lib.oracle_rho_bias_part2(
            c_int(T), c_int(nb), c_int(prob.j_atom_begin), c_int(prob.j_atom_end), c_int(j_coord),
            c_int(prob.n_basis), c_int(prob.n_atoms), c_int(prob.n_centers_basis_I), c_int(nmb),
            A.i(prob.n_point_batches), A.i(prob.n_compute_c_batches), A.i(prob.i_basis_batches),
            A.i(prob.atom_valid_n_compute_c_batches), A.i(prob.i_batch_2_wave_offset), A.d(prob.wave),
            A.d(prob.gradient_wave), A.d(density_matrix), out.ctypes.data_as(c_dbl_p))
    else:
        assert T == 4
        lib = _load(os.path.join("_ref", "libref_bias.so"))
        ints = [nb, prob.j_atom_begin, prob.j_atom_end, j_coord, prob.n_full_points, prob.n_basis, prob.n_atoms,
                prob.n_max_compute_ham, prob.n_centers_basis_I, nmb]
        scal = [ctypes.byref(c_int(int(v_))) for v_ in ints]
        lib.generate_first_order_rho_bias_part2_(
            *scal, A.i(prob.batch_sizes), A.i(prob.n_point_batches), A.i(prob.n_compute_c_batches),
            A.i(prob.i_basis_batches), A.i(prob.atom_valid_n_compute_c_batches), A.i(prob.i_batch_2_wave_offset),
            A.d(prob.wave), A.d(prob.gradient_wave), out.ctypes.data_as(c_dbl_p), A.d(prob.partition_tab),
            A.d(density_matrix))
    return out.reshape((nmb, nb, T), order="F")


# --------------------------------------------------------------------------
# CPU baseline: the reference's rho1 over all host threads
# --------------------------------------------------------------------------


def _openblas_single_thread():
    """The reference links a sequential BLAS (MKL sequential); pin the shared
    OpenBLAS to one thread so batch-parallel threads do not oversubscribe."""
    import glob

    import numpy

    libdir = os.path.realpath(os.path.join(os.path.dirname(numpy.__file__), "..", "numpy.libs"))
    for path in glob.glob(os.path.join(libdir, "libscipy_openblas*")):
        try:
            ob = ctypes.CDLL(path)
            for name in ("scipy_openblas_set_num_threads64_", "scipy_openblas_set_num_threads_64_"):
                if hasattr(ob, name):
                    getattr(ob, name)(c_int(1))
                    return True
        except OSError:
            pass
    return False


def rho1_reference_threaded(prob, n_threads: int):
    """Runs the reference's evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_
    (oracle/_ref, T = 1) over prob's batches split into n_threads contiguous,
    cost-balanced slices, one host thread per slice (the reference itself is
    single-threaded).  Returns (rho, grad) assembled from the slices."""
    import concurrent.futures as cf

    assert prob.T == 1, "threaded baseline slices the batch axis; T = 1 only"
    _openblas_single_thread()
    lib = _load(os.path.join("_ref", "libref_t1.so"))
    nb, nmb = prob.n_my_batches_work, prob.n_max_batch_size
    cost = prob.n_compute_c_batches.astype(np.float64) ** 2 * prob.n_point_batches
    cum = np.concatenate([[0.0], np.cumsum(cost)])
    cuts = [0] + [int(np.searchsorted(cum, cum[-1] * k / n_threads)) for k in range(1, n_threads)] + [nb]
    cuts = sorted(set(min(max(c, 0), nb) for c in cuts))
    A = _Args()
    arr = dict(
        bs=_i(prob.batch_sizes)[0], npb=_i(prob.n_point_batches)[0], pre=_i(prob.n_point_batches_prefix_sum)[0],
        map=_i(prob.i_valid_point_2_i_full_points_map)[0], ncb=_i(prob.n_compute_c_batches)[0],
        ib=_i(prob.i_basis_batches)[0], avn=_i(prob.atom_valid_n_compute_c_batches)[0],
        off=_i(prob.i_batch_2_wave_offset)[0], wave=_d(prob.wave)[0], gwave=_d(prob.gradient_wave)[0],
        P1=_d(prob.first_order_density_matrix)[0], bias=_d(prob.first_order_rho_bias_part2)[0],
        gbias=_d(prob.first_order_gradient_rho_bias)[0], ba=_i(prob.basis_atom)[0], pt=_d(prob.partition_tab)[0])
    grad = np.zeros(3 * nmb * nb)
    rhos = []

    def ip(a, off=0):
        return ctypes.cast(a.ctypes.data + 4 * off, c_int_p)

    def dp(a, off=0):
        return ctypes.cast(a.ctypes.data + 8 * off, c_dbl_p)

    def run(s0, s1):
        rho = np.zeros(prob.n_full_points)
        scal = [ctypes.byref(c_int(int(v))) for v in (
            s1 - s0, prob.j_atom_begin, prob.j_atom_end, prob.j_coord, prob.n_full_points, prob.n_basis,
            prob.n_atoms, prob.n_max_compute_ham, prob.n_centers_basis_I, nmb)]
        lib.evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_(
            *scal, ip(arr["bs"], s0), ip(arr["npb"], s0), ip(arr["pre"], s0), ip(arr["map"]), ip(arr["ncb"], s0),
            ip(arr["ib"], s0 * prob.n_centers_basis_I), ip(arr["avn"], s0 * (prob.n_atoms + 1)), ip(arr["off"], s0),
            dp(arr["wave"]), dp(arr["gwave"]), dp(arr["P1"]), rho.ctypes.data_as(c_dbl_p), dp(arr["bias"], s0 * nmb),
            dp(grad, 3 * nmb * s0), dp(arr["gbias"], 3 * nmb * s0), ip(arr["ba"]), dp(arr["pt"]), dp(arr["P1"]))
        return rho

    with cf.ThreadPoolExecutor(max_workers=max(1, len(cuts) - 1)) as ex:
        rhos = list(ex.map(lambda ab: run(*ab), zip(cuts[:-1], cuts[1:])))
    del A
    rho = np.sum(rhos, axis=0) if rhos else np.zeros(prob.n_full_points)
    return rho.reshape((prob.n_full_points, 1), order="F"), grad.reshape((3, nmb, nb, 1), order="F")


def sumup_reference_threaded(prob, n_threads: int):
    """The reference's sum-up (oracle/_ref) with the valid points split into
    n_threads contiguous slices, one host thread each (outputs are disjoint
    full points).  Returns the accumulated delta_v_hartree."""
    import concurrent.futures as cf

    T = prob.T
    lib = _load(os.path.join("_ref", f"libref_t{T}.so"))
    dv = np.array(prob.delta_v_hartree, dtype=np.float64).ravel(order="F").copy()
    A = _Args()
    ptrs = dict(
        nr=A.i(prob.n_radial), sp=A.i(prob.species), spc=A.i(prob.species_center),
        lh=A.i(prob.l_hartree_max_far_distance), xyz=A.d(prob.coord_points), mrs=A.d(prob.multipole_radius_sq),
        opr=A.d(prob.outer_potential_radius), q=A.d(prob.multipole_moments), spl=A.d(prob.spline),
        lhs=A.i(prob.l_hartree), ng=A.i(prob.n_grid), ncc=A.i(prob.n_cc_lm_ijk),
        chp=A.i(prob.centers_hartree_potential), c2a=A.i(prob.center_to_atom), icc=A.i(prob.index_cc),
        ijk=A.i(prob.index_ijk_max_cc), cc=A.d(prob.cc), cxyz=A.d(prob.coords_center), rgm=A.d(prob.r_grid_min),
        linc=A.d(prob.log_r_grid_inc), scl=A.d(prob.scale_radial), pt=A.d(prob.partition_tab))
    vmap = np.ascontiguousarray(prob.i_valid_point_2_i_full_points_map, dtype=np.int32)
    n = prob.n_valid_points
    cuts = [n * k // n_threads for k in range(n_threads + 1)]

    def run(a, b):
        scal = [ctypes.byref(c_int(int(v))) for v in (
            prob.j_atom_begin, prob.j_atom_end, prob.n_full_points, prob.l_max_analytic_multipole,
            prob.index_cc_dim_0, b - a, prob.l_pot_max, prob.n_max_radial, prob.n_hartree_grid, prob.n_centers,
            prob.n_centers_hartree_potential, prob.n_atoms, prob.hartree_force_l_add, prob.n_species)]
        p = ptrs
        lib.sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_(
            *scal, p["nr"], p["sp"], p["spc"], p["lh"], ctypes.cast(vmap.ctypes.data + 4 * a, c_int_p), p["xyz"],
            p["mrs"], p["opr"], p["q"], p["spl"], p["lhs"], p["ng"], p["ncc"], p["chp"], p["c2a"], p["icc"],
            p["ijk"], p["cc"], p["cxyz"], p["rgm"], p["linc"], p["scl"], p["pt"], dv.ctypes.data_as(c_dbl_p))

    with cf.ThreadPoolExecutor(max_workers=n_threads) as ex:
        list(ex.map(lambda ab: run(*ab), [(cuts[k], cuts[k + 1]) for k in range(n_threads) if cuts[k + 1] > cuts[k]]))
    del A
    return dv.reshape((prob.n_full_points, T), order="F")
