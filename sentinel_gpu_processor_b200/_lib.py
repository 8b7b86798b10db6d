"""ctypes binding of ``libs1b.so`` (declared in ``include/s1b.h``).

The library is the only compute path: importing a function that needs it
raises if the shared object is missing, and every status other than
``S1B_OK`` raises :class:`S1BError`.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_size_t, c_uint64, c_void_p

PKG = os.path.dirname(os.path.abspath(__file__))
# S1B_LIBRARY selects another build of the library (it must exist: there is no fallback)
LIB_PATH = os.environ.get("S1B_LIBRARY") or os.path.join(PKG, "libs1b.so")

S1B_OK = 0
S1B_ERR_INVALID_ARGUMENT = 1
S1B_ERR_CUDA = 2
S1B_ERR_TOO_LARGE = 3
S1B_ERR_EMPTY = 4
S1B_ERR_NO_DEVICE = 5
S1B_ERR_UNSUPPORTED = 6
MAX_STATE_VECTORS = 64
S1B_INTERP_BILINEAR = 0
S1B_INTERP_SINC8 = 1
S1B_SAMPLES_C64 = 0
S1B_SAMPLES_CI16 = 1
MAX_WIN = MAX_STATE_VECTORS - 3
S1B_GOLDSTEIN_NOALLOC_MAX_PATCHES = 4096


class S1BError(RuntimeError):
    def __init__(self, status, where, detail=""):
        self.status = status
        super().__init__(f"{where}: {status_string(status)} ({status}){': ' + detail if detail else ''}")


class Orbit(ctypes.Structure):
    _fields_ = [("n", c_int32), ("t", POINTER(c_double)), ("x", POINTER(c_double)), ("v", POINTER(c_double))]


class PolyTable(ctypes.Structure):
    _fields_ = [("n", c_int32), ("time", POINTER(c_double)), ("t0", POINTER(c_double)),
                ("c0", POINTER(c_double)), ("c1", POINTER(c_double)), ("c2", POINTER(c_double))]


class Radar(ctypes.Structure):
    _fields_ = [("samples_per_burst", c_int32), ("lines_per_burst", c_int32), ("prf", c_double),
                ("wvl", c_double), ("hmin", c_double), ("hmax", c_double),
                ("range_sampling_rate", c_double), ("slant_range_time", c_double),
                ("azimuth_steering_rate", c_double), ("azimuth_time_interval", c_double),
                ("radar_frequency", c_double)]


class Burst(ctypes.Structure):
    _fields_ = [("azimuth_time", c_double), ("first_valid_line", c_int32), ("last_valid_line", c_int32),
                ("first_valid_sample", c_int32), ("last_valid_sample", c_int32)]


class Rsc(ctypes.Structure):
    _fields_ = [("nlat", c_int32), ("nlon", c_int32), ("latmax", c_double), ("lonmin", c_double),
                ("dlat", c_double), ("dlon", c_double)]


class OrbitPoly(ctypes.Structure):
    _fields_ = [("n_state", c_int32), ("n_win", c_int32), ("t0", c_double), ("inv_dt", c_double),
                ("tc", c_double * MAX_WIN), ("c", ((c_double * 8) * 3) * MAX_WIN)]


class BurstPlan(ctypes.Structure):
    _fields_ = [("orbit", OrbitPoly),
                ("lines", c_int32), ("samples", c_int32),
                ("first_valid_line", c_int32), ("last_valid_line", c_int32),
                ("first_valid_sample", c_int32), ("last_valid_sample", c_int32),
                ("win_left", c_int32), ("win_top", c_int32), ("win_right", c_int32), ("win_bottom", c_int32),
                ("rsc_nlat", c_int32), ("rsc_nlon", c_int32),
                ("tstart", c_double), ("dtaz", c_double), ("ati", c_double),
                ("rngstart", c_double), ("dmrg", c_double),
                ("slant_range_time", c_double), ("range_sampling_rate", c_double),
                ("wvl", c_double), ("k4pi_wvl", c_double),
                ("tmid", c_double), ("xmid", c_double * 3), ("vmid", c_double * 3), ("amid", c_double * 3),
                ("ks", c_double), ("etac0", c_double), ("fm", c_double * 4), ("dc", c_double * 4),
                ("lat0", c_double), ("lon0", c_double), ("dlat", c_double), ("dlon", c_double),
                ("latlon_box", c_double * 4)]

    @property
    def window(self):
        return (self.win_left, self.win_top, self.win_right, self.win_bottom)

    @property
    def nrow(self):
        return self.win_bottom - self.win_top

    @property
    def ncol(self):
        return self.win_right - self.win_left


# name -> (restype, argtypes); the table is the C ABI of include/s1b.h
class BurstGeometryIn(ctypes.Structure):
    """s1b_burst_geometry_in_t: one burst of s1b_burst_geometry."""
    _fields_ = [("orbit", c_int32), ("fm_table", c_int32), ("dc_table", c_int32), ("lines", c_int32),
                ("samples", c_int32), ("tstart", c_double), ("prf", c_double), ("azimuth_time_interval", c_double),
                ("slant_range_time", c_double), ("range_sampling_rate", c_double), ("radar_frequency", c_double),
                ("azimuth_steering_rate", c_double), ("hmin", c_double), ("hmax", c_double)]


class BurstGeometry(ctypes.Structure):
    """s1b_burst_geometry_t: footprint, DEM window and TOPS centre terms of one burst."""
    _fields_ = [("latlon_box", c_double * 4), ("ks", c_double), ("etac0", c_double), ("fm", c_double * 4),
                ("dc", c_double * 4), ("win", c_int32 * 4), ("status", c_int32)]


class StitchBurst(ctypes.Structure):
    _fields_ = [("offset", c_int64), ("left", c_int32), ("top", c_int32), ("right", c_int32), ("bottom", c_int32),
                ("subswath", c_int32), ("group", c_int32)]


class FramePair(ctypes.Structure):
    """s1b_frame_pair_t: per-pair result of a frame run."""
    _fields_ = [("ok", c_int32), ("nrow_ml", c_int32), ("ncol_ml", c_int32), ("filtered", c_int32),
                ("header", c_int32 * 6), ("box", c_int32 * 4), ("gslc_rows", c_int32 * 4)]


class FrameSizes(ctypes.Structure):
    _fields_ = [("workspace_bytes", c_size_t), ("slc_elems", c_int64), ("product_elems", c_int64),
                ("max_nrow_ml", c_int32), ("max_ncol_ml", c_int32)]


_SIGNATURES = {
    "s1b_status_string": (c_char_p, [c_int]),
    "s1b_version": (c_int, []),
    "s1b_last_error": (c_char_p, []),
    "s1b_sizeof_burst_plan": (c_size_t, []),
    "s1b_sizeof_orbit_poly": (c_size_t, []),
    "s1b_burst_plan": (c_int, [POINTER(Radar), POINTER(Orbit), POINTER(PolyTable), POINTER(PolyTable),
                               POINTER(Burst), POINTER(Rsc), POINTER(BurstPlan)]),
    "s1b_orbit_poly": (c_int, [POINTER(Orbit), POINTER(OrbitPoly)]),
    "s1b_bounds": (c_int, [POINTER(OrbitPoly), c_double, c_double, c_double, c_double, c_double, c_double,
                           POINTER(c_double)]),
    "s1b_orbit_eval_host": (c_int, [POINTER(OrbitPoly), POINTER(c_double), c_int64, POINTER(c_double),
                                    POINTER(c_double)]),
    "s1b_deramp": (c_int, [POINTER(BurstPlan), c_void_p, c_void_p, c_void_p]),
    "s1b_deramp_ci16": (c_int, [POINTER(BurstPlan), c_void_p, c_void_p, c_void_p]),
    "s1b_geo2rdr": (c_int, [POINTER(BurstPlan), c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
    "s1b_set_geocode_culling": (c_int, [c_int32]),
    "s1b_zero_doppler": (c_int, [POINTER(OrbitPoly), c_void_p, c_int64, c_double, c_void_p, c_void_p, c_void_p]),
    "s1b_llh2xyz": (c_int, [c_void_p, c_void_p, c_int64, c_void_p]),
    "s1b_crossmul_looks": (c_int, [c_void_p, c_int32, c_int32, c_int32, c_int32, c_void_p, c_int32, c_int32,
                                   c_int32, c_int32, c_int32, c_int32, c_int32, c_int32, c_int32, c_int32,
                                   c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_uint64, c_void_p]),
    "s1b_crossmul_box": (c_int, [POINTER(c_int32), POINTER(c_int32), c_int32, c_int32, c_int32,
                                 POINTER(c_int32), POINTER(c_int32)]),
    "s1b_geo2rdr_offsets": (c_int, [POINTER(BurstPlan), c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p,
                                    c_void_p, c_void_p]),
    "s1b_geo2rdr_offsets_dh": (c_int, [POINTER(BurstPlan), POINTER(BurstPlan), c_void_p, c_void_p, c_void_p,
                                       c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "s1b_resample": (c_int, [POINTER(BurstPlan), c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p,
                             c_void_p, c_void_p]),
    "s1b_box_coherence": (c_int, [c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p, c_void_p, c_void_p]),
    "s1b_goldstein_scratch_bytes": (c_size_t, [c_int32, c_int32, c_int32]),
    "s1b_goldstein": (c_int, [c_void_p, c_void_p, c_int32, c_int32, c_int32, c_float, c_void_p, c_size_t,
                              c_void_p]),
    "s1b_geo2rdr_grid_offsets": (c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p]),
    "s1b_set_staging_poll_limit": (ctypes.c_uint32, [ctypes.c_uint32]),
    "s1b_burst_geometry": (c_int, [c_void_p, c_int32, c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_int32,
                                   c_void_p, c_void_p, c_void_p]),
    "s1b_goldstein_noalloc": (c_int, [c_void_p, c_void_p, c_int32, c_int32, c_int32, c_float, c_void_p]),
    "s1b_amp_looks": (c_int, [c_void_p, c_int32, c_int32, c_int32, c_int32, c_int32, c_int32, c_int32, c_int32,
                              c_int32, c_void_p, c_void_p]),
    "s1b_coherence_cc": (c_int, [c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_uint64, c_void_p, c_void_p]),
    "s1b_xyz2llh": (c_int, [c_void_p, c_void_p, c_int64, c_void_p]),
    "s1b_los_grid": (c_int, [POINTER(OrbitPoly), c_double, c_double, c_double, c_double, c_double, c_void_p, c_int64,
                             c_int32, c_int32, c_void_p, c_void_p, c_void_p]),
    "s1b_stitch_workspace_bytes": (c_size_t, [POINTER(StitchBurst), c_int32, c_int32]),
    "s1b_stitch": (c_int, [POINTER(StitchBurst), c_int32, c_void_p, c_int32, c_int32, c_int32, c_void_p,
                           POINTER(c_double), c_void_p, c_size_t, c_void_p]),
    "s1b_frame_create": (c_int, [POINTER(BurstPlan), c_int32, POINTER(c_int32), POINTER(c_int32), c_int32, c_int32,
                                 c_int32, c_int32, c_float, c_uint64, POINTER(c_void_p)]),
    "s1b_frame_destroy": (None, [c_void_p]),
    "s1b_frame_sizes": (c_int, [c_void_p, POINTER(FrameSizes)]),
    "s1b_frame_burst_offset": (c_int, [c_void_p, c_int32, POINTER(c_int64)]),
    "s1b_frame_pair_slot": (c_int, [c_void_p, c_int32, POINTER(c_int64), POINTER(c_int32), POINTER(c_int32)]),
    "s1b_frame_run": (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
                              c_void_p, c_void_p, c_void_p, c_void_p]),
    "s1b_frame_autotune": (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
                                   c_void_p, c_void_p, c_void_p, c_int32, c_void_p]),
    "s1b_frame_profile": (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
                                  c_void_p, c_void_p, c_void_p, POINTER(c_float), c_void_p]),
    "s1b_frame_tuning": (c_int, [c_void_p, POINTER(c_int32)]),
    "s1b_adjoint_create": (c_int, [POINTER(BurstPlan), c_int32, c_int32, c_int32, c_int32, c_int32,
                                   POINTER(c_void_p)]),
    "s1b_adjoint_destroy": (None, [c_void_p]),
    "s1b_adjoint_workspace_bytes": (c_size_t, [c_void_p]),
    "s1b_adjoint_run": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "s1b_frame_set_tuning": (c_int, [c_void_p, POINTER(c_int32)]),
    "s1b_frame_set_sample_format": (c_int, [c_void_p, c_int32]),
    "s1b_frame_set_deramp_fusion": (c_int, [c_void_p, c_int32]),
    "s1b_frame_set_crossmul_fusion": (c_int, [c_void_p, c_int32]),
}

_lib = None


def load():
    """Load libs1b.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m sentinel_gpu_processor_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.s1b_sizeof_burst_plan() != ctypes.sizeof(BurstPlan) or \
            lib.s1b_sizeof_orbit_poly() != ctypes.sizeof(OrbitPoly):
        raise ImportError("libs1b.so struct layout does not match the Python binding")
    _lib = lib
    return lib


def exported_symbols():
    return list(_SIGNATURES)


def status_string(status):
    try:
        return load().s1b_status_string(status).decode()
    except ImportError:
        return "unknown"


def check(status, where):
    if status != S1B_OK:
        detail = load().s1b_last_error().decode(errors="replace")
        raise S1BError(status, where, detail)
    return status


def dptr(t):
    """Device pointer of a CUDA tensor (or None)."""
    if t is None:
        return None
    return c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return c_void_p(s.cuda_stream)
