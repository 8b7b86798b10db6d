"""Torch-facing wrappers of the s1b device entry points.

Each function takes CUDA tensors, launches on the current torch stream and
returns CUDA tensors.  They raise ``S1BError`` on any failure and
``RuntimeError`` when given CPU tensors: there is no CPU path.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

# Optional timing hook: a callable name -> context manager wrapped around the
# library call of each entry point (bench.py brackets them with CUDA events).
timer = None


def _call(name, fn, *args):
    if timer is None:
        return fn(*args)
    with timer(name):
        return fn(*args)


def _need_cuda(*ts):
    for t in ts:
        if t is not None and not t.is_cuda:
            raise RuntimeError("s1b kernels take CUDA tensors only (no CPU fallback)")


def _c64(t, name):
    if t.dtype != torch.complex64 or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous complex64 tensor")


def deramp(plan: _lib.BurstPlan, slc: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """TOPS deramp (reference deramp_burst, geo2rdr.cu:138-158).

    ``slc`` is complex64 [lines * samples] or the measurement TIFF's complex
    int16 samples as int16 [..., 2] (re, im; ``s1b_deramp_ci16``, widened on
    the device).  Returns complex64 of the input's shape (without the (re, im)
    axis for int16 input)."""
    _need_cuda(slc, out)
    ci16 = slc.dtype == torch.int16
    if ci16:
        if not slc.is_contiguous() or slc.shape[-1] != 2:
            raise ValueError("int16 slc must be a contiguous [..., 2] (re, im) tensor")
        n = slc.numel() // 2
    else:
        _c64(slc, "slc")
        n = slc.numel()
    if n != plan.lines * plan.samples:
        raise ValueError("slc size does not match the plan")
    if out is None:
        out = torch.empty(slc.shape[:-1] if ci16 else slc.shape, dtype=torch.complex64, device=slc.device)
    lib = _lib.load()
    fn, name = (lib.s1b_deramp_ci16, "s1b_deramp_ci16") if ci16 else (lib.s1b_deramp, "s1b_deramp")
    _lib.check(_call("deramp", fn, ctypes.byref(plan), _lib.dptr(slc), _lib.dptr(out), _lib.stream_ptr()), name)
    return out


def geo2rdr(plan: _lib.BurstPlan, dem: torch.Tensor, deramped: torch.Tensor, out: torch.Tensor | None = None,
            rows: torch.Tensor | None = None):
    """Geocode a deramped burst onto the plan's DEM window.

    ``dem`` is either the full RSC-grid DEM [nlat, nlon] (the window is taken
    from it without a copy) or the window itself [nrow, ncol] (int16).
    Returns (out complex64 [nrow, ncol], rows int32 [2] = first, last_excl).
    """
    _need_cuda(dem, deramped, out, rows)
    _c64(deramped, "deramped")
    if dem.dtype != torch.int16:
        raise ValueError("dem must be int16")
    nrow, ncol = plan.nrow, plan.ncol
    if nrow <= 0 or ncol <= 0:
        raise _lib.S1BError(_lib.S1B_ERR_EMPTY, "geo2rdr")
    if dem.shape == (plan.rsc_nlat, plan.rsc_nlon) and (dem.shape != (nrow, ncol) or
                                                         (plan.win_top, plan.win_left) != (0, 0)):
        win = dem[plan.win_top:plan.win_bottom, plan.win_left:plan.win_right]
    else:
        win = dem
    if tuple(win.shape) != (nrow, ncol) or win.stride(1) != 1:
        raise ValueError("dem does not cover the plan's window")
    if out is None:
        out = torch.empty((nrow, ncol), dtype=torch.complex64, device=deramped.device)
    if rows is None:
        rows = torch.empty(2, dtype=torch.int32, device=deramped.device)
    lib = _lib.load()
    _lib.check(_call("geo2rdr", lib.s1b_geo2rdr, ctypes.byref(plan), _lib.dptr(win), win.stride(0), _lib.dptr(deramped),
                               _lib.dptr(out), _lib.dptr(rows), _lib.stream_ptr()), "s1b_geo2rdr")
    return out, rows


def geo2rdr_grid_offsets(plan: _lib.BurstPlan, dem: torch.Tensor):
    """Burst line and sample (float64 [nrow, ncol] each) of every pixel of the
    plan's DEM window, solved as the geocoding solves them
    (``s1b_geo2rdr_grid_offsets``).  ``dem``: the full RSC-grid DEM or the
    window itself (int16)."""
    _need_cuda(dem)
    if dem.dtype != torch.int16:
        raise ValueError("dem must be int16")
    nrow, ncol = plan.nrow, plan.ncol
    if nrow <= 0 or ncol <= 0:
        raise _lib.S1BError(_lib.S1B_ERR_EMPTY, "geo2rdr_grid_offsets")
    win = dem[plan.win_top:plan.win_bottom, plan.win_left:plan.win_right] \
        if dem.shape == (plan.rsc_nlat, plan.rsc_nlon) else dem
    if tuple(win.shape) != (nrow, ncol) or win.stride(1) != 1:
        raise ValueError("dem does not cover the plan's window")
    az = torch.empty((nrow, ncol), dtype=torch.float64, device=dem.device)
    rg = torch.empty_like(az)
    _lib.check(_lib.load().s1b_geo2rdr_grid_offsets(ctypes.byref(plan), _lib.dptr(win), win.stride(0), _lib.dptr(az),
                                                    _lib.dptr(rg), _lib.stream_ptr()), "s1b_geo2rdr_grid_offsets")
    return az, rg


def set_geocode_culling(on: bool) -> bool:
    """Switch the geocoding's culling of blocks outside the burst's valid
    lines for later geo2rdr and frame launches of the process (on by default;
    the products are identical either way).  Returns the previous setting."""
    return bool(_lib.load().s1b_set_geocode_culling(1 if on else 0))


def crossmul_looks(ref, ref_box, sec, sec_box, box, rowlook, collook, want=("ifg", "amp1", "amp2", "coh"),
                   fill_seed=0):
    """Fused crossmul + looks + power looks + coherence.

    ref/sec: complex64 [h, w] rasters whose (top, left) global coordinates are
    ``ref_box[:2]`` = (left, top) as (left, top, right, bottom) tuples;
    ``box`` = aligned (left, top, right, bottom).  Returns a dict of outputs.
    """
    _need_cuda(ref, sec)
    _c64(ref, "ref")
    _c64(sec, "sec")
    left, top, right, bottom = box
    nrow_ml = (bottom - top) // rowlook
    ncol_ml = (right - left) // collook
    dev = ref.device
    outs = {}
    shape = (nrow_ml, ncol_ml)
    if "ifg" in want:
        outs["ifg"] = torch.empty(shape, dtype=torch.complex64, device=dev)
    for k in ("amp1", "amp2", "coh", "phase"):
        if k in want:
            outs[k] = torch.empty(shape, dtype=torch.float32, device=dev)
    lib = _lib.load()
    _lib.check(_call("crossmul_looks", lib.s1b_crossmul_looks, 
        _lib.dptr(ref), ref_box[0], ref_box[1], ref.shape[1], ref.shape[0],
        _lib.dptr(sec), sec_box[0], sec_box[1], sec.shape[1], sec.shape[0],
        left, top, nrow_ml, ncol_ml, rowlook, collook,
        _lib.dptr(outs.get("ifg")), _lib.dptr(outs.get("amp1")), _lib.dptr(outs.get("amp2")),
        _lib.dptr(outs.get("coh")), _lib.dptr(outs.get("phase")), int(fill_seed), _lib.stream_ptr()),
        "s1b_crossmul_looks")
    return outs


def goldstein_scratch_bytes(nrow, ncol, n_win=32):
    return int(_lib.load().s1b_goldstein_scratch_bytes(nrow, ncol, n_win))


def goldstein(img: torch.Tensor, alpha: float, n_win: int = 32, out: torch.Tensor | None = None,
              scratch: torch.Tensor | None = None) -> torch.Tensor:
    """Goldstein filter (reference goldstein.cu:328-408) of a complex64 image."""
    _need_cuda(img, out, scratch)
    _c64(img, "img")
    nrow, ncol = img.shape
    need = goldstein_scratch_bytes(nrow, ncol, n_win)
    if scratch is None:
        scratch = torch.empty(max(need, 1), dtype=torch.uint8, device=img.device)
    if out is None:
        out = torch.empty_like(img)
    lib = _lib.load()
    _lib.check(_call("goldstein", lib.s1b_goldstein, _lib.dptr(img), _lib.dptr(out), nrow, ncol, n_win, float(alpha),
                                 _lib.dptr(scratch), scratch.numel() * scratch.element_size(),
                                 _lib.stream_ptr()), "s1b_goldstein")
    return out


def zero_doppler(poly: _lib.OrbitPoly, xyz: torch.Tensor, tline0: float):
    """Zero-Doppler time and line-of-sight vector for ECEF points [n, 3] (float64)."""
    _need_cuda(xyz)
    xyz = xyz.contiguous().to(torch.float64)
    n = xyz.shape[0]
    t = torch.empty(n, dtype=torch.float64, device=xyz.device)
    dr = torch.empty((n, 3), dtype=torch.float64, device=xyz.device)
    _lib.check(_call("zero_doppler", _lib.load().s1b_zero_doppler, ctypes.byref(poly), _lib.dptr(xyz), n, float(tline0), _lib.dptr(t),
                                            _lib.dptr(dr), _lib.stream_ptr()), "s1b_zero_doppler")
    return t, dr


def los_grid(poly: _lib.OrbitPoly, t0: float, lat0: float, lat_step: float, lon0: float, lon_step: float,
             dem: torch.Tensor):
    """Line-of-sight unit vectors (float32 [nrow * ncol, 3]) and look angles
    (float32 [nrow, ncol], degrees) of a lat/lon grid with int16 heights
    ``dem`` [nrow, ncol] (unit column stride); ``s1b_los_grid``."""
    _need_cuda(dem)
    if dem.dtype != torch.int16 or dem.dim() != 2 or dem.stride(1) != 1:
        raise ValueError("dem must be an int16 [nrow, ncol] tensor with unit column stride")
    nrow, ncol = dem.shape
    los = torch.empty((nrow * ncol, 3), dtype=torch.float32, device=dem.device)
    theta = torch.empty((nrow, ncol), dtype=torch.float32, device=dem.device)
    _lib.check(_call("los_grid", _lib.load().s1b_los_grid, ctypes.byref(poly), float(t0), float(lat0),
                     float(lat_step), float(lon0), float(lon_step), _lib.dptr(dem), dem.stride(0), nrow, ncol,
                     _lib.dptr(los), _lib.dptr(theta), _lib.stream_ptr()), "s1b_los_grid")
    return los, theta


def llh2xyz(llh: torch.Tensor) -> torch.Tensor:
    _need_cuda(llh)
    llh = llh.contiguous().to(torch.float64)
    out = torch.empty_like(llh)
    _lib.check(_call("llh2xyz", _lib.load().s1b_llh2xyz, _lib.dptr(llh), _lib.dptr(out), llh.shape[0], _lib.stream_ptr()),
               "s1b_llh2xyz")
    return out


def xyz2llh(xyz: torch.Tensor) -> torch.Tensor:
    """ECEF [n, 3] -> (deg, deg, m) [n, 3], float64."""
    _need_cuda(xyz)
    xyz = xyz.contiguous().to(torch.float64)
    out = torch.empty_like(xyz)
    _lib.check(_call("xyz2llh", _lib.load().s1b_xyz2llh, _lib.dptr(xyz), _lib.dptr(out), xyz.shape[0],
                     _lib.stream_ptr()), "s1b_xyz2llh")
    return out


def amp_looks(slc: torch.Tensor, left: int, top: int, nrow0: int, ncol0: int, rowlook: int, collook: int,
              first: bool, amp: torch.Tensor) -> torch.Tensor:
    """Amplitude looks of a cropped geocoded SLC [h, w] (top-left (left, top))
    into the frame grid ``amp`` float32 [nrow0//rowlook, ncol0//collook]."""
    _need_cuda(slc, amp)
    _c64(slc, "slc")
    if amp.dtype != torch.float32 or tuple(amp.shape) != (nrow0 // rowlook, ncol0 // collook) or \
            not amp.is_contiguous():
        raise ValueError("amp must be contiguous float32 [nrow0//rowlook, ncol0//collook]")
    h, w = slc.shape
    _lib.check(_call("amp_looks", _lib.load().s1b_amp_looks, _lib.dptr(slc), w, h, int(left), int(top), int(nrow0),
                     int(ncol0), int(rowlook), int(collook), 1 if first else 0, _lib.dptr(amp), _lib.stream_ptr()),
               "s1b_amp_looks")
    return amp


def coherence_cc(ifg: torch.Tensor, amp1: torch.Tensor, amp2: torch.Tensor, fill_seed: int = 0,
                 out: torch.Tensor | None = None) -> torch.Tensor:
    """``.cc`` raster float32 [nrow, 2 ncol]: rows [amp1*amp2 | coherence]."""
    _need_cuda(ifg, amp1, amp2, out)
    _c64(ifg, "ifg")
    nrow, ncol = ifg.shape
    for a in (amp1, amp2):
        if a.dtype != torch.float32 or tuple(a.shape) != (nrow, ncol) or not a.is_contiguous():
            raise ValueError("amp1/amp2 must be contiguous float32 rasters of the interferogram's shape")
    if out is None:
        out = torch.empty((nrow, 2 * ncol), dtype=torch.float32, device=ifg.device)
    _lib.check(_call("coherence_cc", _lib.load().s1b_coherence_cc, _lib.dptr(ifg), _lib.dptr(amp1), _lib.dptr(amp2),
                     nrow, ncol, int(fill_seed), _lib.dptr(out), _lib.stream_ptr()), "s1b_coherence_cc")
    return out


def geo2rdr_offsets(plan: _lib.BurstPlan, lat: torch.Tensor, lon: torch.Tensor, hgt: torch.Tensor,
                    az_off: torch.Tensor | None = None, rg_off: torch.Tensor | None = None):
    """Secondary sample offsets (az_off, rg_off float32 [L, S]) of the reference
    grid pixels whose float64 lat/lon/height rasters are given."""
    _need_cuda(lat, lon, hgt, az_off, rg_off)
    for t in (lat, lon, hgt):
        if t.dtype != torch.float64 or not t.is_contiguous() or t.shape != lat.shape:
            raise ValueError("lat/lon/hgt must be contiguous float64 rasters of one shape")
    L, S = lat.shape
    if az_off is None:
        az_off = torch.empty((L, S), dtype=torch.float32, device=lat.device)
    if rg_off is None:
        rg_off = torch.empty((L, S), dtype=torch.float32, device=lat.device)
    _lib.check(_call("geo2rdr_offsets", _lib.load().s1b_geo2rdr_offsets, ctypes.byref(plan), _lib.dptr(lat), _lib.dptr(lon), _lib.dptr(hgt),
                                               L, S, _lib.dptr(az_off), _lib.dptr(rg_off), _lib.stream_ptr()),
               "s1b_geo2rdr_offsets")
    return az_off, rg_off


def geo2rdr_offsets_dh(plan: _lib.BurstPlan, ref_plan: _lib.BurstPlan, lat: torch.Tensor, lon: torch.Tensor,
                       hgt: torch.Tensor):
    """Offsets as :func:`geo2rdr_offsets` plus their sensitivities to a
    height error of the reference-grid pixels (the point moving along the
    reference's iso-range zero-Doppler circle): returns (az_off, rg_off,
    daz_dh, drg_dh), float32 [L, S] (samples per metre)."""
    _need_cuda(lat, lon, hgt)
    for t in (lat, lon, hgt):
        if t.dtype != torch.float64 or not t.is_contiguous() or t.shape != lat.shape:
            raise ValueError("lat/lon/hgt must be contiguous float64 rasters of one shape")
    L, S = lat.shape
    outs = [torch.empty((L, S), dtype=torch.float32, device=lat.device) for _ in range(4)]
    _lib.check(_call("geo2rdr_offsets", _lib.load().s1b_geo2rdr_offsets_dh, ctypes.byref(plan),
                     ctypes.byref(ref_plan), _lib.dptr(lat),
                     _lib.dptr(lon), _lib.dptr(hgt), L, S, *[_lib.dptr(o) for o in outs], _lib.stream_ptr()),
               "s1b_geo2rdr_offsets_dh")
    return tuple(outs)


def resample(plan: _lib.BurstPlan, sec: torch.Tensor, az_off: torch.Tensor, rg_off: torch.Tensor,
             interp: str = "sinc8", out: torch.Tensor | None = None,
             status: torch.Tensor | None = None) -> torch.Tensor:
    """Resample the secondary burst of ``plan`` onto the grid of the offsets.

    ``status`` (int32 device word) is set to 1 if a tile's staging did not
    complete; one is allocated when not given."""
    _need_cuda(sec, az_off, rg_off, out, status)
    _c64(sec, "sec")
    if sec.numel() != plan.lines * plan.samples:
        raise ValueError("sec size does not match the plan")
    if az_off.shape != rg_off.shape or az_off.dtype != torch.float32 or not az_off.is_contiguous() \
            or not rg_off.is_contiguous():
        raise ValueError("az_off/rg_off must be contiguous float32 rasters of one shape")
    L, S = az_off.shape
    if out is None:
        out = torch.empty((L, S), dtype=torch.complex64, device=sec.device)
    if status is None:
        status = torch.empty(1, dtype=torch.int32, device=sec.device)
    mode = {"sinc8": _lib.S1B_INTERP_SINC8, "bilinear": _lib.S1B_INTERP_BILINEAR}[interp]
    _lib.check(_call("resample", _lib.load().s1b_resample, ctypes.byref(plan), _lib.dptr(sec), _lib.dptr(az_off), _lib.dptr(rg_off),
                                        L, S, mode, _lib.dptr(out), _lib.dptr(status), _lib.stream_ptr()), "s1b_resample")
    return out


def box_coherence(ref: torch.Tensor, sec: torch.Tensor, win: int = 5, out: torch.Tensor | None = None,
                  status: torch.Tensor | None = None) -> torch.Tensor:
    """Full-resolution win x win boxcar coherence of two co-registered SLCs."""
    _need_cuda(ref, sec, out, status)
    _c64(ref, "ref")
    _c64(sec, "sec")
    if ref.shape != sec.shape:
        raise ValueError("ref and sec must have one shape")
    L, S = ref.shape
    if out is None:
        out = torch.empty((L, S), dtype=torch.float32, device=ref.device)
    if status is None:
        status = torch.empty(1, dtype=torch.int32, device=ref.device)
    _lib.check(_call("box_coherence", _lib.load().s1b_box_coherence, _lib.dptr(ref), _lib.dptr(sec), L, S, int(win), _lib.dptr(out),
                                             _lib.dptr(status), _lib.stream_ptr()), "s1b_box_coherence")
    return out
