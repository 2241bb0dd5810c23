"""ctypes bindings over the C ABI of libfrpa.so (include/frpa.h).

The library is the product; this module only marshals arguments.  Loading
fails loudly if the shared library has not been built (there is no CPU or
PyTorch fallback): run ``python -m fast_rpa_eval_b200.build``.
"""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# FRPA_LIB overrides the library path (e.g. an alternative build of the same sources)
LIB_PATH = os.environ.get("FRPA_LIB") or os.path.join(_HERE, "lib", "libfrpa.so")

FRPA_OK = 0
FRPA_ERR_INVALID = 1
FRPA_ERR_CUDA = 2
FRPA_ERR_NO_SESSION = 3
FRPA_ERR_OOM = 4
FRPA_ERR_UNSUPPORTED = 5
RHO1_FP64 = 0
RHO1_SPLIT_BF16 = 1
RHO1_SPLIT_I8 = 2
# frpa_rho1_plan_set_tuning keys
TUNE_FP64_TILE_POINTS = 1
TUNE_FP64_CTAS_PER_SM = 2
TUNE_SPLIT_TILE_POINTS = 3
TUNE_ORDER = 4
TUNE_SPLIT_I8_SCRATCH_MB = 5
TUNINGS = {"fp64_tile_points": TUNE_FP64_TILE_POINTS, "fp64_ctas_per_sm": TUNE_FP64_CTAS_PER_SM,
           "split_tile_points": TUNE_SPLIT_TILE_POINTS, "order": TUNE_ORDER,
           "split_i8_scratch_mb": TUNE_SPLIT_I8_SCRATCH_MB}

c_int = ctypes.c_int
c_ll = ctypes.c_longlong
c_void_p = ctypes.c_void_p
c_int_p = ctypes.POINTER(ctypes.c_int)
c_dbl_p = ctypes.POINTER(ctypes.c_double)


class FrpaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"frpa status {status}: {message}")
        self.status = status
        self.message = message


_lock = threading.Lock()
_lib = None


def lib():
    """The loaded libfrpa.so (raises if it was not built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise FileNotFoundError(
                    f"{LIB_PATH} is missing: build the CUDA library with `python -m fast_rpa_eval_b200.build`")
            L = ctypes.CDLL(LIB_PATH)
            L.frpa_last_error_message.restype = ctypes.c_char_p
            _lib = L
        return _lib


def last_error():
    L = lib()
    return L.frpa_last_error(), L.frpa_last_error_message().decode()


def check(status: int):
    if status != FRPA_OK:
        raise FrpaError(status, lib().frpa_last_error_message().decode())


def check_void_call():
    """For the reference's void entry points: raise if the call failed."""
    st, msg = last_error()
    if st != FRPA_OK:
        raise FrpaError(st, msg)


# ----------------------------------------------------------- descriptors


class Rho1Desc(ctypes.Structure):
    _fields_ = [
        ("atom_tile_size", c_int), ("n_my_batches_work", c_int), ("n_full_points", c_int), ("n_basis", c_int),
        ("n_centers_basis_I", c_int), ("n_max_batch_size", c_int),
        ("n_point_batches", c_int_p), ("n_point_batches_prefix_sum", c_int_p),
        ("i_valid_point_2_i_full_points_map", c_int_p), ("n_compute_c_batches", c_int_p),
        ("i_basis_batches", c_int_p), ("i_batch_2_wave_offset", c_int_p), ("wave_alloc_len", c_ll),
    ]


class SumupDesc(ctypes.Structure):
    _fields_ = [
        ("atom_tile_size", c_int), ("n_full_points", c_int), ("l_max_analytic_multipole", c_int),
        ("index_cc_dim_0", c_int), ("n_valid_points", c_int), ("l_pot_max", c_int), ("n_hartree_grid", c_int),
        ("n_centers", c_int), ("n_centers_hartree_potential", c_int), ("n_atoms", c_int),
        ("hartree_force_l_add", c_int), ("n_species", c_int),
        ("species", c_int_p), ("species_center", c_int_p), ("i_valid_point_2_i_full_points_map", c_int_p),
        ("coord_points", c_dbl_p),
        ("l_hartree", c_int_p), ("n_grid", c_int_p), ("n_cc_lm_ijk", c_int_p), ("centers_hartree_potential", c_int_p),
        ("center_to_atom", c_int_p), ("index_cc", c_int_p), ("index_ijk_max_cc", c_int_p),
        ("cc", c_dbl_p), ("coords_center", c_dbl_p), ("r_grid_min", c_dbl_p), ("log_r_grid_inc", c_dbl_p),
    ]


class _Keep:
    """Holds the host arrays a descriptor points into."""

    def __init__(self):
        self.arrays = []

    def i(self, a):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel(order="F"))
        self.arrays.append(a)
        return a.ctypes.data_as(c_int_p)

    def d(self, a):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))
        self.arrays.append(a)
        return a.ctypes.data_as(c_dbl_p)


def rho1_desc(prob, keep: _Keep, T: int | None = None) -> Rho1Desc:
    d = Rho1Desc()
    d.atom_tile_size = prob.T if T is None else T
    d.n_my_batches_work = prob.n_my_batches_work
    d.n_full_points = prob.n_full_points
    d.n_basis = prob.n_basis
    d.n_centers_basis_I = prob.n_centers_basis_I
    d.n_max_batch_size = prob.n_max_batch_size
    d.n_point_batches = keep.i(prob.n_point_batches)
    d.n_point_batches_prefix_sum = keep.i(prob.n_point_batches_prefix_sum)
    d.i_valid_point_2_i_full_points_map = keep.i(prob.i_valid_point_2_i_full_points_map)
    d.n_compute_c_batches = keep.i(prob.n_compute_c_batches)
    d.i_basis_batches = keep.i(prob.i_basis_batches)
    d.i_batch_2_wave_offset = keep.i(prob.i_batch_2_wave_offset)
    d.wave_alloc_len = 0
    return d


def sumup_desc(prob, keep: _Keep) -> SumupDesc:
    d = SumupDesc()
    for name in ("n_full_points", "l_max_analytic_multipole", "index_cc_dim_0", "n_valid_points", "l_pot_max",
                 "n_hartree_grid", "n_centers", "n_centers_hartree_potential", "n_atoms", "hartree_force_l_add",
                 "n_species"):
        setattr(d, name, int(getattr(prob, name)))
    d.atom_tile_size = prob.T
    for name in ("species", "species_center", "i_valid_point_2_i_full_points_map", "l_hartree", "n_grid",
                 "n_cc_lm_ijk", "centers_hartree_potential", "center_to_atom", "index_cc", "index_ijk_max_cc"):
        setattr(d, name, keep.i(getattr(prob, name)))
    for name in ("coord_points", "cc", "coords_center", "r_grid_min", "log_r_grid_inc"):
        setattr(d, name, keep.d(getattr(prob, name)))
    return d


def _ptr(t):
    """Device (or host) address of a torch tensor / numpy array, or None."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return c_void_p(t.data_ptr())
    return c_void_p(t.ctypes.data)


def _stream(stream):
    """cudaStream_t for a torch stream, an integer handle, or None (torch's
    current stream, so that calls inside a CUDA-graph capture are captured)."""
    if stream is None:
        try:
            import torch

            if torch.cuda.is_available() and torch.cuda.is_initialized():
                return c_void_p(torch.cuda.current_stream().cuda_stream)
        except ImportError:
            pass
        return c_void_p(0)
    if hasattr(stream, "cuda_stream"):
        return c_void_p(stream.cuda_stream)
    return c_void_p(int(stream))


# ------------------------------------------------------------------ plans


class Rho1Plan:
    """Device work list for one rho1 batch structure (frpa_rho1_plan)."""

    def __init__(self, prob, T: int | None = None):
        self._keep = _Keep()
        self.desc = rho1_desc(prob, self._keep, T)
        self.T = self.desc.atom_tile_size
        self.handle = c_void_p()
        check(lib().frpa_rho1_plan_create(ctypes.byref(self.handle), ctypes.byref(self.desc)))

    def info(self):
        out = (c_ll * 3)()
        check(lib().frpa_rho1_plan_info(self.handle, out))
        return {"n_items": out[0], "n_valid_batches": out[1], "n_valid_points": out[2]}

    def i8_info(self):
        """Split-int8 grouping: groups (three launches each), work items,
        packed P1c tiles, largest per-group A + B scratch in bytes."""
        out = (c_ll * 4)()
        check(lib().frpa_rho1_plan_i8_info(self.handle, out))
        return {"groups": out[0], "items": out[1], "b_tiles": out[2], "scratch_bytes": out[3]}

    def execute(self, n_active, wave, gwave, P1, bias, gbias, rho, grad, mode=RHO1_FP64, stream=None):
        check(lib().frpa_rho1_execute(self.handle, c_int(mode), c_int(n_active), _ptr(wave), _ptr(gwave), _ptr(P1),
                                      _ptr(bias), _ptr(gbias), _ptr(rho), _ptr(grad), _stream(stream)))

    def execute_fused_bias(self, n_active, n_atoms, j_atom_begin, j_coord, atom_valid, density_matrix, wave, gwave,
                           P1, bias, gbias, rho, grad, stream=None):
        """frpa_rho1_execute_fused_bias: FP64 rho1 with the density-matrix bias
        computed in the same launch."""
        check(lib().frpa_rho1_execute_fused_bias(
            self.handle, c_int(n_active), c_int(n_atoms), c_int(j_atom_begin), c_int(j_coord), _ptr(atom_valid),
            _ptr(density_matrix), _ptr(wave), _ptr(gwave), _ptr(P1), _ptr(bias), _ptr(gbias), _ptr(rho), _ptr(grad),
            _stream(stream)))

    def device_flags(self) -> int:
        f = c_int(0)
        check(lib().frpa_rho1_device_flags(self.handle, ctypes.byref(f)))
        return f.value

    def bias_part2(self, T, n_atoms, j_atom_begin, j_atom_end, j_coord, atom_valid, wave, gwave, density_matrix,
                   out, stream=None):
        """first_order_rho_bias_part2 (n_max_batch_size, n_batches, T) on the device
        (generate_first_order_rho_bias_part2.cpp:11-168); atom_valid is the int32
        (n_atoms + 1, n_batches) array of 0-based compute ranges."""
        check(lib().frpa_rho1_bias_part2(self.handle, c_int(T), c_int(n_atoms), c_int(j_atom_begin),
                                         c_int(j_atom_end), c_int(j_coord), _ptr(atom_valid), _ptr(wave),
                                         _ptr(gwave), _ptr(density_matrix), _ptr(out), _stream(stream)))

    def set_tuning(self, **kw):
        """fp64_tile_points (64 | 128), fp64_ctas_per_sm (0..3),
        split_tile_points (16..128), order (0 largest first | 1 batch order |
        2 locality order, the default),
        split_i8_scratch_mb (>= 1: packed-operand scratch per group of batches)."""
        for k, v in kw.items():
            check(lib().frpa_rho1_plan_set_tuning(self.handle, c_int(TUNINGS[k]), c_int(int(v))))

    def tuning(self) -> dict:
        out = {}
        for k, key in TUNINGS.items():
            v = c_int(0)
            check(lib().frpa_rho1_plan_get_tuning(self.handle, c_int(key), ctypes.byref(v)))
            out[k] = v.value
        return out

    def first_order_h(self, n_active, n_atoms, j_atom_begin, j_coord, atom_valid, wave, gwave, hwave, xc, vhg,
                      partition_tab, H, stream=None):
        """frpa_rho1_first_order_h: accumulates into H (device); ``xc`` maps
        the names of synth.first_order_h_inputs to device tensors."""
        check(lib().frpa_rho1_first_order_h(
            self.handle, c_int(n_active), c_int(n_atoms), c_int(j_atom_begin), c_int(j_coord), _ptr(atom_valid),
            _ptr(wave), _ptr(gwave), _ptr(hwave), _ptr(xc["vsigma"]), _ptr(xc["gradient_rho"]),
            _ptr(xc["H_prefactor1"]), _ptr(xc["first_order_gradient_rho"]), _ptr(vhg), _ptr(xc["first_order_rho"]),
            _ptr(xc["v2rho2"]), _ptr(xc["v2rhosigma"]), _ptr(xc["v2sigma2"]), _ptr(partition_tab), _ptr(H),
            _stream(stream)))

    def adjoint_p1(self, n_active, wave, gwave, g_rho, g_grad, dP1, stream=None):
        check(lib().frpa_rho1_adjoint_p1(self.handle, c_int(n_active), _ptr(wave), _ptr(gwave), _ptr(g_rho),
                                         _ptr(g_grad), _ptr(dP1), _stream(stream)))

    def close(self):
        if self.handle:
            lib().frpa_rho1_plan_destroy(self.handle)
            self.handle = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SumupPlan:
    """Constant sum-up inputs resident on the device (frpa_sumup_plan)."""

    def __init__(self, prob):
        self._keep = _Keep()
        self.desc = sumup_desc(prob, self._keep)
        self.handle = c_void_p()
        check(lib().frpa_sumup_plan_create(ctypes.byref(self.handle), ctypes.byref(self.desc)))

    @property
    def fast(self) -> bool:
        return bool(lib().frpa_sumup_plan_fast(self.handle))

    def execute(self, n_active, lhmfd, mrs, opr, Q, spline, dv, branch_codes=None, force_generic=False,
                stream=None):
        check(lib().frpa_sumup_execute(self.handle, c_int(n_active), c_int(1 if force_generic else 0), _ptr(lhmfd),
                                       _ptr(mrs), _ptr(opr), _ptr(Q), _ptr(spline), _ptr(dv), _ptr(branch_codes),
                                       _stream(stream)))

    def adjoint_q(self, n_active, lhmfd, mrs, opr, Q, g, dQ, stream=None):
        check(lib().frpa_sumup_adjoint_q(self.handle, c_int(n_active), _ptr(lhmfd), _ptr(mrs), _ptr(opr), _ptr(Q),
                                         _ptr(g), _ptr(dQ), _stream(stream)))

    def device_flags(self) -> int:
        f = c_int(0)
        check(lib().frpa_sumup_device_flags(self.handle, ctypes.byref(f)))
        return f.value

    def close(self):
        if self.handle:
            lib().frpa_sumup_plan_destroy(self.handle)
            self.handle = c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def synth_basis_values(prob, points_dev, wave_dev, gwave_dev, pad_value=0.0, stream=None):
    """Fill device wave arrays of `prob` analytically (frpa_synth_basis_values)."""
    keep = _Keep()
    desc = rho1_desc(prob, keep)
    b = prob.basis
    atoms = np.asfortranarray(prob.atoms_xyz.T)
    check(lib().frpa_synth_basis_values(ctypes.byref(desc), _ptr(points_dev), c_int(prob.n_atoms), keep.d(atoms),
                                        keep.i(b.atom), keep.i(b.l), keep.i(b.m), keep.d(b.alpha),
                                        ctypes.c_double(pad_value), _ptr(wave_dev), _ptr(gwave_dev), _stream(stream)))


def synth_p1_window(global_index, n: int, T: int, scale: float, seed: int, out, stream=None):
    """Device window (n, n, T) of a symmetric synthetic P1 keyed by global basis
    indices (frpa_synth_p1_window); global_index: int32 device tensor."""
    check(lib().frpa_synth_p1_window(_ptr(global_index), c_int(n), c_int(T), ctypes.c_double(scale),
                                     ctypes.c_ulonglong(seed), _ptr(out), _stream(stream)))


def set_atom_tile_size(T: int):
    check(lib().frpa_set_atom_tile_size(c_int(T)))


def set_device(device: int):
    """frpa_set_device: the GPU the library's own (static) CUDA runtime makes
    current on this thread; plans and the session created afterwards use it.
    Call it with torch's device when that is not device 0."""
    check(lib().frpa_set_device(c_int(device)))


def get_device() -> int:
    d = c_int(-1)
    check(lib().frpa_get_device(ctypes.byref(d)))
    return d.value


def set_rho1_mode(mode: int):
    check(lib().frpa_set_rho1_mode(c_int(mode)))


# ------------------------------------------------------- reference drop-ins


def _iref(v):
    return ctypes.byref(c_int(int(v)))


def dropin_rho1(prob, symbol: str = "evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_",
                rho=None, grad=None):
    """Calls a reference-named rho1 entry point with host numpy arrays and
    returns (first_order_rho, first_order_gradient_rho)."""
    T = prob.T
    set_atom_tile_size(T)
    k = _Keep()
    rho = np.zeros(prob.n_full_points * T) if rho is None else rho
    grad = np.zeros(3 * prob.n_max_batch_size * prob.n_my_batches_work * T) if grad is None else grad
    dm = prob.density_matrix if prob.density_matrix is not None else np.zeros(1)
    fn = getattr(lib(), symbol)
    lib().frpa_clear_error()
    fn(_iref(prob.n_my_batches_work), _iref(prob.j_atom_begin), _iref(prob.j_atom_end), _iref(prob.j_coord),
       _iref(prob.n_full_points), _iref(prob.n_basis), _iref(prob.n_atoms), _iref(prob.n_max_compute_ham),
       _iref(prob.n_centers_basis_I), _iref(prob.n_max_batch_size), k.i(prob.batch_sizes), k.i(prob.n_point_batches),
       k.i(prob.n_point_batches_prefix_sum), k.i(prob.i_valid_point_2_i_full_points_map),
       k.i(prob.n_compute_c_batches), k.i(prob.i_basis_batches), k.i(prob.atom_valid_n_compute_c_batches),
       k.i(prob.i_batch_2_wave_offset), k.d(prob.wave), k.d(prob.gradient_wave), k.d(prob.first_order_density_matrix),
       _ptr(rho), k.d(prob.first_order_rho_bias_part2), _ptr(grad), k.d(prob.first_order_gradient_rho_bias),
       k.i(prob.basis_atom), k.d(prob.partition_tab), k.d(dm))
    check_void_call()
    return (np.asarray(rho).reshape((prob.n_full_points, T), order="F"),
            np.asarray(grad).reshape((3, prob.n_max_batch_size, prob.n_my_batches_work, T), order="F"))


def dropin_first_order_h(prob, v_hartree_gradient, xc, H=None, j_coord: int | None = None):
    """evaluate_first_order_h_reduce_memory_c_v2_ with host arrays: ``xc`` as
    synth.first_order_h_inputs, H (n_basis, n_basis, T) accumulated into
    (zeros if None); returns H."""
    T = prob.T
    set_atom_tile_size(T)
    k = _Keep()
    Hf = (np.zeros(prob.n_basis * prob.n_basis * T) if H is None
          else np.array(H, dtype=np.float64).ravel(order="F").copy())
    jc = prob.j_coord if j_coord is None else j_coord
    z = np.zeros(1)
    lib().frpa_clear_error()
    lib().evaluate_first_order_h_reduce_memory_c_v2_(
        _iref(prob.j_atom_begin), _iref(prob.j_atom_end), _iref(prob.n_full_points), _iref(jc), _iref(prob.n_basis),
        _iref(prob.n_atoms), _iref(prob.n_max_compute_ham), _iref(prob.n_max_batch_size),
        _iref(prob.n_my_batches_work), _iref(prob.n_centers_basis_I), k.i(prob.n_point_batches),
        k.i(prob.n_compute_c_batches), k.i(prob.i_basis_batches), k.i(prob.atom_valid_n_compute_c_batches),
        k.i(prob.n_point_batches_prefix_sum), k.i(prob.i_valid_point_2_i_full_points_map), k.d(z),
        k.d(xc["vsigma"]), k.d(xc["gradient_rho"]), k.d(z), k.i(prob.i_batch_2_wave_offset), k.d(prob.wave),
        k.d(prob.gradient_wave), k.d(xc["hessian_wave"]), _ptr(Hf), k.d(xc["H_prefactor1"]),
        k.d(xc["first_order_gradient_rho"]), k.d(v_hartree_gradient), k.d(xc["first_order_rho"]), k.d(xc["v2rho2"]),
        k.d(xc["v2rhosigma"]), k.d(xc["v2sigma2"]), k.d(prob.partition_tab), _iref(0))
    check_void_call()
    return Hf.reshape((prob.n_basis, prob.n_basis, T), order="F")


def dropin_sumup(prob, delta_v=None):
    """sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_ with host
    arrays; returns the accumulated delta_v_hartree."""
    set_atom_tile_size(prob.T)
    k = _Keep()
    dv = np.array(prob.delta_v_hartree if delta_v is None else delta_v, dtype=np.float64).ravel(order="F").copy()
    ints = [prob.j_atom_begin, prob.j_atom_end, prob.n_full_points, prob.l_max_analytic_multipole,
            prob.index_cc_dim_0, prob.n_valid_points, prob.l_pot_max, prob.n_max_radial, prob.n_hartree_grid,
            prob.n_centers, prob.n_centers_hartree_potential, prob.n_atoms, prob.hartree_force_l_add, prob.n_species]
    lib().frpa_clear_error()
    lib().sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_(
        *[_iref(v) for v in ints], k.i(prob.n_radial), k.i(prob.species), k.i(prob.species_center),
        k.i(prob.l_hartree_max_far_distance), k.i(prob.i_valid_point_2_i_full_points_map), k.d(prob.coord_points),
        k.d(prob.multipole_radius_sq), k.d(prob.outer_potential_radius), k.d(prob.multipole_moments),
        k.d(prob.spline), k.i(prob.l_hartree), k.i(prob.n_grid), k.i(prob.n_cc_lm_ijk),
        k.i(prob.centers_hartree_potential), k.i(prob.center_to_atom), k.i(prob.index_cc),
        k.i(prob.index_ijk_max_cc), k.d(prob.cc), k.d(prob.coords_center), k.d(prob.r_grid_min),
        k.d(prob.log_r_grid_inc), k.d(prob.scale_radial), k.d(prob.partition_tab), _ptr(dv))
    check_void_call()
    return dv.reshape((prob.n_full_points, prob.T), order="F")


class Session:
    """The reference's device session: init_dfpt_device_info /
    init_dfpt_device_data, the *_cu_host_ twins, free_*.  Holds references to
    every host array passed in so they outlive the calls."""

    def __init__(self, rho_prob, sumup_prob=None, wave=None, gradient_wave=None, entry=None):
        """``wave`` / ``gradient_wave`` (device tensors) replace the problem's
        host arrays; the session then uses them in place.  ``entry``: an object
        whose attributes replace the library's entry points of the same names
        (e.g. callables that reach the C++-linkage exports the way the
        reference's C++ callers bind them); default: the C-linkage exports."""
        self._entry = entry
        self.rho_prob, self.sumup_prob = rho_prob, sumup_prob
        T = rho_prob.T
        if sumup_prob is not None and sumup_prob.T != T:
            raise ValueError("rho1 and sum-up problems must share ATOM_TILE_SIZE")
        set_atom_tile_size(T)
        L = lib()
        L.frpa_clear_error()
        self._fn("init_dfpt_device_info")()
        check_void_call()
        k = self._k = _Keep()
        r, s = rho_prob, sumup_prob
        z = np.zeros(1)
        zi = np.zeros(1, np.int32)
        if s is not None:
            sc = dict(n_valid=s.n_valid_points, n_atoms=s.n_atoms, l_pot_max=s.l_pot_max, n_max_radial=s.n_max_radial,
                      n_hartree_grid=s.n_hartree_grid, n_centers=s.n_centers,
                      n_chp=s.n_centers_hartree_potential, hfla=s.hartree_force_l_add, n_species=s.n_species,
                      lma=s.l_max_analytic_multipole, icc=s.index_cc_dim_0)
            if s.n_full_points != r.n_full_points:
                raise ValueError("rho1 and sum-up problems must share n_full_points")
        else:
            sc = dict(n_valid=0, n_atoms=r.n_atoms, l_pot_max=0, n_max_radial=0, n_hartree_grid=0, n_centers=0,
                      n_chp=0, hfla=0, n_species=0, lma=0, icc=0)
        g = (lambda name, kind: (k.i if kind == "i" else k.d)(getattr(s, name)) if s is not None else
             (k.i(zi) if kind == "i" else k.d(z)))
        dm = r.density_matrix if r.density_matrix is not None else np.zeros(1)
        self._fn("init_dfpt_device_data")(
            _iref(r.n_my_batches_work), _iref(r.n_full_points), _iref(sc["n_valid"]), _iref(r.n_basis),
            _iref(sc["n_atoms"]), _iref(r.n_max_compute_ham), _iref(r.n_centers_basis_I), _iref(r.n_max_batch_size),
            _iref(sc["l_pot_max"]), _iref(sc["n_max_radial"]), _iref(sc["n_hartree_grid"]), _iref(sc["n_centers"]),
            _iref(sc["n_chp"]), _iref(sc["hfla"]), _iref(sc["n_species"]), _iref(sc["lma"]), _iref(sc["icc"]),
            k.i(r.basis_atom), k.i(r.batch_sizes), k.i(r.n_point_batches), k.i(r.n_point_batches_prefix_sum),
            k.i(r.i_valid_point_2_i_full_points_map if s is None else s.i_valid_point_2_i_full_points_map),
            k.i(r.n_compute_c_batches), k.i(r.i_basis_batches), k.i(r.atom_valid_n_compute_c_batches),
            k.i(r.i_batch_2_wave_offset), _ptr(wave) if wave is not None else k.d(r.wave),
            _ptr(gradient_wave) if gradient_wave is not None else k.d(r.gradient_wave), k.d(dm),
            g("n_radial", "i"), g("species", "i"), g("species_center", "i"), g("coord_points", "d"),
            g("l_hartree", "i"), g("n_grid", "i"), g("n_cc_lm_ijk", "i"), g("centers_hartree_potential", "i"),
            g("center_to_atom", "i"), g("index_cc", "i"), g("index_ijk_max_cc", "i"), g("cc", "d"),
            g("coords_center", "d"), g("r_grid_min", "d"), g("log_r_grid_inc", "d"), g("scale_radial", "d"),
            k.d(r.partition_tab), k.d(r.first_order_density_matrix), k.d(np.zeros(1)),
            k.d(r.first_order_rho_bias_part2), k.d(np.zeros(1)), k.d(r.first_order_gradient_rho_bias),
            g("l_hartree_max_far_distance", "i"), g("multipole_radius_sq", "d"), g("outer_potential_radius", "d"),
            g("multipole_moments", "d"), g("spline", "d"), g("delta_v_hartree", "d"))
        check_void_call()

    def rho1(self, P1=None, bias=None, gbias=None, rho=None, grad=None):
        """evaluate_first_order_rho_..._cu_host_: uploads P1 and the biases
        (host arrays), returns the host outputs."""
        r = self.rho_prob
        k = _Keep()
        T = r.T
        rho = np.zeros(r.n_full_points * T) if rho is None else rho
        grad = np.zeros(3 * r.n_max_batch_size * r.n_my_batches_work * T) if grad is None else grad
        P1 = r.first_order_density_matrix if P1 is None else P1
        bias = r.first_order_rho_bias_part2 if bias is None else bias
        gbias = r.first_order_gradient_rho_bias if gbias is None else gbias
        zi = np.zeros(1, np.int32)
        z = np.zeros(1)
        lib().frpa_clear_error()
        lib().evaluate_first_order_rho_reduce_memory_c_v3_batches_atoms_cu_host_(
            _iref(r.n_my_batches_work), _iref(r.j_atom_begin), _iref(r.j_atom_end), _iref(r.j_coord),
            _iref(r.n_full_points), _iref(r.n_basis), _iref(r.n_atoms), _iref(r.n_max_compute_ham),
            _iref(r.n_centers_basis_I), _iref(r.n_max_batch_size), k.i(zi), k.i(zi), k.i(zi), k.i(zi), k.i(zi),
            k.i(zi), k.i(zi), k.i(zi), k.d(z), k.d(z), _host_ptr(P1, k), _host_ptr(rho, k, writable=True),
            _host_ptr(bias, k), _host_ptr(grad, k, writable=True), _host_ptr(gbias, k), k.i(zi), k.d(z), k.d(z))
        check_void_call()
        return rho, grad

    def sumup(self, delta_v=None, lhmfd=None, mrs=None, opr=None, Q=None, spline=None):
        """sum_up_..._cu_host_ with the session's constants; per-call arrays
        default to the problem's.  Returns the accumulated delta_v (host)."""
        s = self.sumup_prob
        k = _Keep()
        dv = np.array(s.delta_v_hartree if delta_v is None else delta_v, dtype=np.float64).ravel(order="F").copy()
        zi = np.zeros(1, np.int32)
        z = np.zeros(1)
        lib().frpa_clear_error()
        fn = self._fn("sum_up_whole_potential_c_v3_atoms_full_points_j_atom_tile_cu_host_")
        fn(c_int(s.j_atom_begin), c_int(s.j_atom_end), c_int(s.n_full_points), c_int(s.l_max_analytic_multipole),
           c_int(s.index_cc_dim_0), c_int(s.n_valid_points), c_int(s.l_pot_max), c_int(s.n_max_radial),
           c_int(s.n_hartree_grid), c_int(s.n_centers), c_int(s.n_centers_hartree_potential), c_int(s.n_atoms),
           c_int(s.hartree_force_l_add), c_int(s.n_species), k.i(zi), k.i(zi), k.i(zi),
           k.i(s.l_hartree_max_far_distance if lhmfd is None else lhmfd), k.i(zi), k.d(z),
           k.d(s.multipole_radius_sq if mrs is None else mrs), k.d(s.outer_potential_radius if opr is None else opr),
           k.d(s.multipole_moments if Q is None else Q), k.d(s.spline if spline is None else spline), k.i(zi),
           k.i(zi), k.i(zi), k.i(zi), k.i(zi), k.i(zi), k.i(zi), k.d(z), k.d(z), k.d(z), k.d(z), k.d(z), k.d(z),
           _ptr(dv))
        check_void_call()
        return dv.reshape((s.n_full_points, s.T), order="F")

    def _fn(self, name):
        f = getattr(self._entry, name, None) if self._entry is not None else None
        return f if f is not None else getattr(lib(), name)

    def close(self):
        self._fn("free_dfpt_device_data")()
        self._fn("free_dfpt_device_info")()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _host_ptr(a, keep: _Keep, writable: bool = False):
    """Pointer to a host array without copying when it is already a
    contiguous float64 buffer (numpy, or a pinned torch CPU tensor)."""
    if hasattr(a, "data_ptr"):
        return c_void_p(a.data_ptr())
    a = np.asarray(a)
    if a.dtype == np.float64 and (a.flags.f_contiguous or a.flags.c_contiguous) and (a.ndim <= 1 or a.flags.f_contiguous):
        return c_void_p(a.ctypes.data)
    if writable:
        raise ValueError("output arrays must be contiguous float64")
    return keep.d(a)


def probe_fp64_tflops(kind: str = "mma") -> float:
    """Measured FP64 throughput of the current device: 'mma' (tensor pipe,
    m8n8k4 f64) or 'fma' (DFMA pipe)."""
    v = ctypes.c_double(0.0)
    fn = lib().frpa_probe_fp64_mma_tflops if kind == "mma" else lib().frpa_probe_fp64_fma_tflops
    check(fn(ctypes.byref(v), c_void_p(0)))
    return v.value


def capture_graph(fn, warmup: int = 1):
    """A torch.cuda.CUDAGraph of ``fn()`` (plan launches on the current stream:
    the library allocates nothing after plan creation, so its launches
    capture).  ``fn`` runs ``warmup`` times first, outside the capture, so
    that one-time kernel attribute set-up happens before it.  Replay with
    ``graph.replay()``."""
    import torch

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(warmup):
            fn()
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    return g


def dropin_bias_part2(prob, density_matrix, j_coord: int = 1, bias=None):
    """generate_first_order_rho_bias_part2_ through the reference-named entry
    point (host arrays); returns (n_max_batch_size, n_batches, 4)."""
    L = lib()
    nmb, nb = prob.n_max_batch_size, prob.n_my_batches_work
    out = np.zeros(nmb * nb * 4) if bias is None else np.array(bias, dtype=np.float64).ravel(order="F").copy()
    keep = []

    def ip(a):
        a = np.ascontiguousarray(np.asarray(a).ravel(order="F"), dtype=np.int32)
        keep.append(a)
        return a.ctypes.data_as(c_int_p)

    def dp(a):
        a = np.ascontiguousarray(np.asarray(a).ravel(order="F"), dtype=np.float64)
        keep.append(a)
        return a.ctypes.data_as(c_dbl_p)

    ints = [nb, prob.j_atom_begin, prob.j_atom_end, j_coord, prob.n_full_points, prob.n_basis, prob.n_atoms,
            prob.n_max_compute_ham, prob.n_centers_basis_I, nmb]
    refs = [ctypes.byref(c_int(int(v))) for v in ints]
    L.generate_first_order_rho_bias_part2_(
        *refs, ip(prob.batch_sizes), ip(prob.n_point_batches), ip(prob.n_compute_c_batches), ip(prob.i_basis_batches),
        ip(prob.atom_valid_n_compute_c_batches), ip(prob.i_batch_2_wave_offset), dp(prob.wave),
        dp(prob.gradient_wave), out.ctypes.data_as(c_dbl_p), dp(prob.partition_tab), dp(density_matrix))
    check_void_call()
    return out.reshape((nmb, nb, 4), order="F")
