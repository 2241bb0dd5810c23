"""Capture / replay of the reference's binary problem dumps.

The reference writes the batch metadata of evaluate_first_order_rho and the
inputs of the sum-up as little-endian binary files
(fast_rap_src_dfpt_gpu_eval/evaluate_first_order_rho_direct_test.hpp:27-70 and
sum_up_direct_test.hpp:50-140): a fixed list of int32 scalars, then each
array as a size_t (uint64) element count followed by its int32 / float64
elements, in a fixed order.  The layout is kept byte for byte so that dumps
taken from FHI-aims runs with the reference can be replayed here, and dumps
written here read back in the reference.

    meta = read_rho_meta("first_order_rho.bin")      # dict of scalars / arrays
    write_rho_meta("copy.bin", meta)                  # identical bytes
    sumup = read_sumup_data("sumup.bin")
"""

from __future__ import annotations

import struct

import numpy as np

_I32 = np.dtype("<i4")
_F64 = np.dtype("<f8")

# evaluate_first_order_rho_direct_test.hpp:8-26 (FirstOrderRhoMetaData)
RHO_SCALARS = ("n_my_batches_work", "n_full_points", "n_basis", "n_atoms", "n_max_compute_ham",
               "n_centers_basis_I", "n_max_batch_size")
RHO_ARRAYS = (("basis_atom", _I32), ("batch_sizes", _I32), ("n_point_batches", _I32),
              ("n_point_batches_prefix_sum", _I32), ("i_valid_point_2_i_full_points_map", _I32),
              ("n_compute_c_batches", _I32), ("i_basis_batches", _I32), ("atom_valid_n_compute_c_batches", _I32),
              ("i_batch_2_wave_offset", _I32))

# sum_up_direct_test.hpp:8-49 (HartreePotentialData)
SUMUP_SCALARS = ("j_atom_begin", "j_atom_end", "n_full_points", "l_max_analytic_multipole", "index_cc_dim_0",
                 "n_valid_points", "l_pot_max", "n_max_radial", "n_hartree_grid", "n_centers",
                 "n_centers_hartree_potential", "n_atoms", "hartree_force_l_add", "n_species")
SUMUP_ARRAYS = (("n_radial", _I32), ("species", _I32), ("species_center", _I32),
                ("l_hartree_max_far_distance", _I32), ("i_valid_point_2_i_full_points_map", _I32),
                ("coord_points", _F64), ("multipole_radius_sq", _F64), ("outer_potential_radius", _F64),
                ("multipole_moments", _F64), ("l_hartree", _I32), ("n_grid", _I32), ("n_cc_lm_ijk", _I32),
                ("centers_hartree_potential", _I32), ("center_to_atom", _I32), ("index_cc", _I32),
                ("index_ijk_max_cc", _I32), ("cc", _F64), ("coords_center", _F64), ("r_grid_min", _F64),
                ("log_r_grid_inc", _F64), ("scale_radial", _F64), ("partition_tab", _F64))


class CaptureError(ValueError):
    pass


def _read(path: str, scalars, arrays) -> dict:
    buf = open(path, "rb").read()
    pos = 4 * len(scalars)
    if len(buf) < pos:
        raise CaptureError(f"{path}: {len(buf)} bytes, shorter than its {len(scalars)} scalars")
    out = dict(zip(scalars, struct.unpack_from(f"<{len(scalars)}i", buf, 0)))
    for name, dt in arrays:
        if pos + 8 > len(buf):
            raise CaptureError(f"{path}: ends before the size of '{name}'")
        (n,) = struct.unpack_from("<Q", buf, pos)
        pos += 8
        if n == 0:
            raise CaptureError(f"{path}: '{name}' has size 0 (the reference writes non-empty arrays only)")
        end = pos + n * dt.itemsize
        if end > len(buf):
            raise CaptureError(f"{path}: '{name}' needs {n} elements, the file ends first")
        out[name] = np.frombuffer(buf, dtype=dt, count=n, offset=pos).copy()
        pos = end
    if pos != len(buf):
        raise CaptureError(f"{path}: {len(buf) - pos} trailing bytes")
    return out


def _write(path: str, data: dict, scalars, arrays) -> None:
    parts = [struct.pack(f"<{len(scalars)}i", *[int(data[s]) for s in scalars])]
    for name, dt in arrays:
        a = np.ascontiguousarray(np.asarray(data[name]).ravel(order="F"), dtype=dt)
        if a.size == 0:
            raise CaptureError(f"'{name}' is empty; the format stores non-empty arrays only")
        parts.append(struct.pack("<Q", a.size))
        parts.append(a.tobytes())
    with open(path, "wb") as f:
        f.write(b"".join(parts))


def read_rho_meta(path: str) -> dict:
    """rho1 batch metadata (evaluate_first_order_rho_direct_test.hpp:73-128)."""
    return _read(path, RHO_SCALARS, RHO_ARRAYS)


def write_rho_meta(path: str, data: dict) -> None:
    """Same bytes as write_first_order_rho_meta_data (…_direct_test.hpp:27-70)."""
    _write(path, data, RHO_SCALARS, RHO_ARRAYS)


def read_sumup_data(path: str) -> dict:
    """Sum-up inputs (sum_up_direct_test.hpp, HartreePotentialData)."""
    return _read(path, SUMUP_SCALARS, SUMUP_ARRAYS)


def write_sumup_data(path: str, data: dict) -> None:
    """Same bytes as write_hartree_potential_data (sum_up_direct_test.hpp:50-140)."""
    _write(path, data, SUMUP_SCALARS, SUMUP_ARRAYS)


def rho_meta_of(prob) -> dict:
    """The capture record of a rho1 problem (the metadata the reference dumps)."""
    d = {s: int(getattr(prob, s)) for s in RHO_SCALARS}
    for name, dt in RHO_ARRAYS:
        d[name] = np.asarray(getattr(prob, name)).ravel(order="F").astype(dt)
    return d


def check_rho_meta(meta: dict) -> None:
    """Consistency of a replayed rho1 record (what a plan would reject)."""
    nb = meta["n_my_batches_work"]
    pre, off = meta["n_point_batches_prefix_sum"], meta["i_batch_2_wave_offset"]
    if len(meta["n_compute_c_batches"]) != nb or len(meta["n_point_batches"]) != nb:
        raise CaptureError("per-batch arrays do not have n_my_batches_work entries")
    if len(pre) != nb + 1 or len(off) != nb + 1:
        raise CaptureError("prefix / offset arrays need n_my_batches_work + 1 entries")
    if np.any(np.diff(pre) != meta["n_point_batches"]):
        raise CaptureError("n_point_batches_prefix_sum is not the running sum of n_point_batches")
    if len(meta["i_basis_batches"]) != meta["n_centers_basis_I"] * nb:
        raise CaptureError("i_basis_batches is not (n_centers_basis_I, n_batches)")
