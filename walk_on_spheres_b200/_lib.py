"""ctypes binding of libwos_b200.so (the C ABI declared in include/wos_b200.h).

The library is the only compute path: there is no CPU or PyTorch fallback.
If the shared library is missing, importing the binding raises, and every
solver call goes through the CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("WOS_B200_LIB", PKG / "lib" / "libwos_b200.so"))

WOS_OK = 0
STATUS_NAMES = {0: "WOS_OK", 1: "WOS_ERR_INVALID", 2: "WOS_ERR_CUDA", 3: "WOS_ERR_MESH",
                4: "WOS_ERR_DEVICE", 5: "WOS_ERR_IO"}


class WosError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Grid(C.Structure):
    """wos_grid (include/wos/grid.hpp:5-10)."""
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int),
                ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
                ("ymax", C.c_double), ("zmin", C.c_double), ("zmax", C.c_double)]


class Params(C.Structure):
    """wos_params: the registry entry's scalars plus the walk method."""
    _fields_ = [("equation", C.c_int), ("source_mode", C.c_int), ("alpha", C.c_double),
                ("N_walks", C.c_int), ("epsilon", C.c_double), ("max_steps", C.c_int),
                ("max_ray_attempts", C.c_int), ("seed", C.c_uint64), ("method", C.c_int)]


class Counters(C.Structure):
    """wos_counters (include/wos/runner.hpp:240-283 plus device timings)."""
    _fields_ = [("inside_points", C.c_longlong), ("max_steps_hits", C.c_longlong),
                ("ambiguous_ray_retries", C.c_longlong), ("indeterminate_points", C.c_longlong),
                ("total_walks", C.c_longlong), ("total_steps", C.c_longlong),
                ("sum_variance", C.c_double), ("sum_standard_error", C.c_double),
                ("sum_mean_steps", C.c_double), ("effective_epsilon", C.c_double),
                ("classify_ms", C.c_float), ("walk_ms", C.c_float), ("total_ms", C.c_float),
                ("exact_queries", C.c_longlong)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class GaussianSource(C.Structure):
    """wos_gaussian_source: f(x) = Q exp(-|x - x0|^2 / sigma^2), plus the MIS mixture
    probability and proposal."""
    _fields_ = [("Q", C.c_double), ("x0", C.c_double * 3), ("sigma", C.c_double),
                ("mis_green_probability", C.c_double), ("proposal_x0", C.c_double * 3),
                ("proposal_sigma", C.c_double)]


class TransientParams(C.Structure):
    """wos_transient_params (the reference's Level2Config plus the walk method)."""
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("dt", C.c_double),
                ("total_time", C.c_double), ("heat_on_time", C.c_double),
                ("walks", C.c_int), ("max_steps", C.c_int), ("epsilon", C.c_double),
                ("seed", C.c_uint64), ("cubic", C.c_int), ("length_x", C.c_double),
                ("length_y", C.c_double), ("thickness", C.c_double),
                ("conductivity", C.c_double), ("density", C.c_double),
                ("specific_heat", C.c_double), ("electrical_power", C.c_double),
                ("efficiency", C.c_double), ("sigma_x", C.c_double), ("sigma_y", C.c_double),
                ("method", C.c_int), ("scenario", C.c_int), ("plate_x0", C.c_double),
                ("plate_y0", C.c_double), ("weld_y", C.c_double), ("source_start_x", C.c_double),
                ("weld_speed", C.c_double)]


class StationaryParams(C.Structure):
    """wos_stationary_params (the reference's Level1Config plus the case, source and method)."""
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("walks", C.c_int), ("max_steps", C.c_int),
                ("epsilon", C.c_double), ("seed", C.c_uint64), ("case_stream", C.c_uint64),
                ("length_x", C.c_double), ("length_y", C.c_double), ("thickness", C.c_double),
                ("conductivity", C.c_double), ("electrical_power", C.c_double),
                ("efficiency", C.c_double), ("sigma_x", C.c_double), ("sigma_y", C.c_double),
                ("source_x", C.c_double), ("source_y", C.c_double), ("peak_rise", C.c_double),
                ("source", C.c_int), ("source_mode", C.c_int),
                ("mis_green_probability", C.c_double), ("method", C.c_int),
                ("max_proposal_attempts", C.c_int)]


class H5Layout(C.Structure):
    """wos_h5_layout: file offsets of the five fields' values, and the file size."""
    _fields_ = [("field_offset", C.c_longlong * 5), ("file_size", C.c_longlong)]


RUN_FN = C.CFUNCTYPE(C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_char_p, C.c_int, C.c_int,
                     C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_uint64, C.c_double,
                     C.c_int)


BARRIER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p)
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_double), C.c_int, C.c_int, C.c_void_p)
DIMS_FN = C.CFUNCTYPE(C.c_int, C.c_int, C.POINTER(C.c_int), C.c_void_p)


class Collectives(C.Structure):
    """wos_collectives: the caller's barrier / all-reduce (/ dims_create) for
    registry runs with size > 1."""
    _fields_ = [("barrier", BARRIER_FN), ("allreduce", ALLREDUCE_FN),
                ("dims_create", DIMS_FN), ("user", C.c_void_p)]


class EquationEntry(C.Structure):
    """wos_equation_entry (src/equations/equations.hpp:7-17)."""
    _fields_ = [("name", C.c_char_p), ("run_2D", RUN_FN), ("run_3D", RUN_FN)]


# exported symbols of include/wos_b200.h with their signatures
VP = C.c_void_p
SIGNATURES = {
    "wos_abi_version": (C.c_int, []),
    "wos_context_create": (C.c_int, [C.c_int, C.POINTER(VP)]),
    "wos_context_destroy": (None, [VP]),
    "wos_last_error": (C.c_char_p, [VP]),
    "wos_last_global_error": (C.c_char_p, []),
    "wos_set_mesh": (C.c_int, [VP, C.c_int, VP, C.c_int, VP, C.c_int, VP, C.c_int]),
    "wos_load_obj": (C.c_int, [VP, C.c_char_p, C.c_int]),
    "wos_mesh_info": (C.c_int, [VP, C.POINTER(C.c_int), C.POINTER(C.c_int), VP]),
    "wos_grid_over_mesh": (C.c_int, [VP, C.c_int, C.c_int, C.c_int, C.POINTER(Grid)]),
    "wos_solve_grid": (C.c_int, [VP, C.POINTER(Params), C.POINTER(Grid)] + [VP] * 5 +
                       [C.POINTER(Counters)]),
    "wos_solve_grid_device": (C.c_int, [VP, C.POINTER(Params), C.POINTER(Grid)] + [VP] * 5 +
                              [C.POINTER(Counters)]),
    "wos_solve_points": (C.c_int, [VP, C.POINTER(Params), VP, VP, C.c_longlong] + [VP] * 5 +
                         [C.POINTER(Counters)]),
    "wos_prng_u64": (C.c_int, [VP, VP, C.c_longlong, C.c_int, VP]),
    "wos_closest_points": (C.c_int, [VP, C.c_int, VP, C.c_longlong, VP, VP, VP]),
    "wos_special_functions": (C.c_int, [VP, C.c_int, VP, C.c_longlong, VP, VP]),
    "wos_distance_bounds": (C.c_int, [VP, VP, C.c_longlong, VP]),
    "wos_set_tuning": (C.c_int, [VP, C.c_int, C.c_int]),
    "wos_scene_arena": (C.c_int, [VP, VP, C.c_longlong, C.POINTER(C.c_longlong)]),
    "wos_mesh_vertex_count": (C.c_int, [VP, C.POINTER(C.c_int)]),
    "wos_transient_defaults": (None, [C.POINTER(TransientParams)]),
    "wos_transient_steps": (C.c_int, [C.POINTER(TransientParams)]),
    "wos_transient_solve": (C.c_int, [VP, C.POINTER(TransientParams), VP, C.c_int, VP, VP,
                                      C.POINTER(C.c_longlong), C.POINTER(C.c_float)]),
    "wos_stationary_defaults": (None, [C.POINTER(StationaryParams), C.c_int]),
    "wos_stationary_solve": (C.c_int, [VP, C.POINTER(StationaryParams)] + [VP] * 4 +
                             [C.POINTER(C.c_longlong), C.POINTER(C.c_float)]),
    "wos_batch_create": (C.c_int, [VP, C.POINTER(VP)]),
    "wos_batch_destroy": (None, [VP]),
    "wos_batch_add_mesh": (C.c_int, [VP, C.c_int, VP, C.c_int, VP, C.c_int, VP, C.c_int,
                                     C.POINTER(C.c_int)]),
    "wos_batch_add_solve": (C.c_int, [VP, C.c_int, C.POINTER(Params), C.POINTER(Grid),
                                      C.POINTER(C.c_int)]),
    "wos_batch_set_tuning": (C.c_int, [VP, C.c_int, C.c_int]),
    "wos_batch_prepare": (C.c_int, [VP]),
    "wos_batch_run": (C.c_int, [VP, C.c_int, C.POINTER(C.c_float)]),
    "wos_batch_info": (C.c_int, [VP, C.POINTER(C.c_int)] + [C.POINTER(C.c_longlong)] * 3),
    "wos_batch_result": (C.c_int, [VP, C.c_int] + [VP] * 5 + [C.POINTER(Counters)]),
    "wos_heat_forward": (C.c_int, [VP, C.POINTER(Params), C.POINTER(GaussianSource), VP, VP, VP,
                                   C.c_longlong] + [VP] * 5 + [C.POINTER(Counters)]),
    "wos_heat_adjoint": (C.c_int, [VP, C.POINTER(Params), C.POINTER(GaussianSource), VP, VP, VP,
                                   C.c_longlong] + [VP] * 6 + [C.POINTER(Counters)]),
    "wos_build_wide_bvh": (C.c_int, [C.c_int, VP, C.c_int, VP, C.c_int] + [VP] * 5),
    "wos_equation_registry": (C.POINTER(EquationEntry), [C.POINTER(C.c_int)]),
    "wos_peek_mesh_dim": (C.c_int, [C.c_char_p]),
    "wos_set_collectives": (C.c_int, [C.POINTER(Collectives)]),
    "wos_rank_block": (C.c_int, [C.c_int] * 6 + [C.POINTER(C.c_int)] * 3 + [C.c_char_p,
                                                                         C.c_int]),
    # result files: serial writer and the parallel path (create, then blocks)
    "wos_write_hdf5": (C.c_int, [C.c_char_p, C.POINTER(Grid)] + [VP] * 5 + [
        C.c_int, C.c_double, C.c_int, C.c_longlong, C.c_int, C.c_int, C.c_longlong,
        C.c_longlong, C.c_uint64, C.c_int, C.c_double, C.c_int]),
    "wos_hdf5_layout": (C.c_int, [C.POINTER(Grid), C.c_int, C.c_int, C.POINTER(H5Layout)]),
    "wos_hdf5_create": (C.c_int, [C.c_char_p, C.POINTER(Grid), C.c_int, C.c_double, C.c_int,
                                  C.c_longlong, C.c_int, C.c_int, C.c_longlong, C.c_longlong,
                                  C.c_uint64, C.c_int, C.c_double, C.c_int,
                                  C.POINTER(H5Layout)]),
    "wos_hdf5_write_block": (C.c_int, [C.c_char_p, C.POINTER(H5Layout), C.POINTER(Grid),
                                       C.POINTER(C.c_int), C.POINTER(C.c_int)] + [VP] * 5),
    "wos_hdf5_write_range": (C.c_int, [C.c_char_p, C.POINTER(H5Layout), C.POINTER(Grid),
                                       C.c_longlong, C.c_longlong] + [VP] * 5),
}

_lib = None


def lib() -> C.CDLL:
    """Load libwos_b200.so once; raise if it is not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is not built; run `python -m walk_on_spheres_b200.build` "
                "(the CUDA library is required: there is no CPU fallback)")
        handle = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(handle, name)
            f.restype = res
            f.argtypes = args
        _lib = handle
    return _lib


def check(status: int, ctx=None) -> None:
    if status != WOS_OK:
        L = lib()
        msg = (L.wos_last_error(ctx) if ctx else L.wos_last_global_error()) or b""
        raise WosError(status, msg.decode(errors="replace"))
