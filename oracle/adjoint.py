"""Float64 oracle of the coregistration-refinement objective (no reference
counterpart): the model of the s1b adjoint, its objective, central finite
differences, and a float64 torch.autograd reference gradient.

Test infrastructure only (see ``oracle/__init__.py``).

Per burst (reference grid L x S, pixel (row, col)):
    az = row + az0 + p0 + p1 xa + p2 xr + daz_dh dh
    rg = col + rg0 + p3 + p4 xa + p5 xr + drg_dh dh
    xa = (row - L/2) / L,  xr = (col - S/2) / S
    s  = resample(sec, az, rg)   (8-tap windowed sinc, TOPS deramp/reramp:
                                  oracle/radargrid.py)
    over the rl x cl windows of the multilook grid:
    gamma = |sum conj(r) s| / sqrt(sum |r|^2 sum |s|^2)   (0 where a sum is 0)
    J = -(sum of gamma over every window of every burst) / (number of windows)

Height sensitivities daz/dh, drg/dh of the offsets are checked against
central differences of ``radargrid.offsets`` with the ground point of each
reference sample moved along the reference's zero-Doppler iso-range circle
(a DEM error changes the height of the point the reference sample sees).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import geometry as og
from . import radargrid as orr
from .geo2rdr import PI, SOL, BurstCoeffs, Radar


@dataclass
class AdjBurst:
    ref: np.ndarray      # complex64 [L, S]
    sec: np.ndarray      # complex64 [L, S] (secondary burst as acquired)
    radar: Radar         # secondary radar
    co: BurstCoeffs      # secondary TOPS coefficients
    az0: np.ndarray      # float32 offsets [L, S]
    rg0: np.ndarray
    daz_dh: np.ndarray   # float32 sensitivities [L, S]
    drg_dh: np.ndarray


def basis(L, S):
    rows = np.arange(L, dtype=np.float64)[:, None]
    cols = np.arange(S, dtype=np.float64)[None, :]
    return (rows - 0.5 * L) / L, (cols - 0.5 * S) / S


def coordinates(b: AdjBurst, params, dh):
    """Absolute secondary sample coordinates (az, rg), float64."""
    L, S = b.az0.shape
    xa, xr = basis(L, S)
    p = np.asarray(params, dtype=np.float64)
    rows = np.arange(L, dtype=np.float64)[:, None]
    cols = np.arange(S, dtype=np.float64)[None, :]
    dh = np.asarray(dh, dtype=np.float64)
    az = rows + b.az0.astype(np.float64) + p[0] + p[1] * xa + p[2] * xr + b.daz_dh.astype(np.float64) * dh
    rg = cols + b.rg0.astype(np.float64) + p[3] + p[4] * xa + p[5] * xr + b.drg_dh.astype(np.float64) * dh
    return az, rg


def window_gamma(ref, s, rl, cl):
    """gamma over the rl x cl multilook windows (float64)."""
    L, S = ref.shape
    nr, nc = L // rl, S // cl
    r = ref[:nr * rl, :nc * cl].astype(np.complex128)
    s = s[:nr * rl, :nc * cl]
    def box(x):
        return x.reshape(nr, rl, nc, cl).sum(axis=(1, 3))
    I = box(np.conj(r) * s)
    P1 = box(np.abs(r) ** 2)
    P2 = box(np.abs(s) ** 2)
    den = P1 * P2
    ok = (den > 0) & (np.abs(I) > 0)
    g = np.zeros(I.shape)
    g[ok] = np.abs(I[ok]) / np.sqrt(den[ok])
    return g


def objective(bursts, params, dh, rl, cl):
    """J = -mean gamma over every window of every burst (float64)."""
    tot, n = 0.0, 0
    for k, b in enumerate(bursts):
        az, rg = coordinates(b, params[k], dh[k])
        s, _ = orr.resample(b.sec, b.radar, b.co, az, rg, "sinc8", exact=True)
        g = window_gamma(b.ref, s, rl, cl)
        tot += g.sum()
        n += g.size
    return -tot / n


def support_masks(bursts, params, dh):
    """Per burst, the pixels whose 8 x 8 support lies inside the burst."""
    out = []
    for k, b in enumerate(bursts):
        az, rg = coordinates(b, params[k], dh[k])
        Ls, Ss = b.sec.shape
        na, nr = np.floor(az), np.floor(rg)
        out.append((na - 3 >= 0) & (na + 4 < Ls) & (nr - 3 >= 0) & (nr + 4 < Ss))
    return out


def fd_stable(bursts, params, dh, direction, step_p=1e-4, step_h=1e-2):
    """True when no pixel enters or leaves the support under any of the
    finite-difference perturbations (J is smooth there; a pixel crossing the
    burst edge makes J jump, and a difference quotient would measure the jump)."""
    params = np.asarray(params, dtype=np.float64)
    dh = np.asarray(dh, dtype=np.float64)
    base = support_masks(bursts, params, dh)
    cases = []
    for k in range(params.shape[0]):
        for j in range(6):
            for s in (step_p, -step_p):
                p1 = params.copy()
                p1[k, j] += s
                cases.append((p1, dh))
    for s in (step_h, -step_h):
        cases.append((params, dh + s * np.asarray(direction, dtype=np.float64)))
    for p1, h1 in cases:
        if any((m != m0).any() for m, m0 in zip(support_masks(bursts, p1, h1), base)):
            return False
    return True


def fd_params(bursts, params, dh, rl, cl, step=1e-4):
    """Central differences of J in every parameter (float64) -> [n_bursts, 6]."""
    params = np.asarray(params, dtype=np.float64)
    out = np.zeros_like(params)
    for k in range(params.shape[0]):
        for j in range(6):
            p1 = params.copy()
            p1[k, j] += step
            p2 = params.copy()
            p2[k, j] -= step
            out[k, j] = (objective(bursts, p1, dh, rl, cl) - objective(bursts, p2, dh, rl, cl)) / (2 * step)
    return out


def fd_direction(bursts, params, dh, direction, rl, cl, step=1e-2):
    """Central difference of J along a height-error direction (float64)."""
    dh = np.asarray(dh, dtype=np.float64)
    d = np.asarray(direction, dtype=np.float64)
    return (objective(bursts, params, dh + step * d, rl, cl) - objective(bursts, params, dh - step * d, rl, cl)) / (2 * step)


def on_reference_circle(lat, lon, h, ref_radar, ref_orbit, ref_burst_time, iters=8):
    """Ground points of the reference samples (row, col) at geodetic height h:
    (lat, lon) with |p - X(t)| = R and (p - X(t)).V(t) = 0, t = burst_time +
    row / prf, R = near range + col * range spacing; Newton on (lat, lon)
    from the given point with central-difference Jacobians (float64)."""
    L, S = lat.shape
    tt, xx, vv = ref_orbit
    t = ref_burst_time + np.arange(L, dtype=np.float64) / ref_radar.prf
    X, V = og.intp_orbit(tt, xx, vv, t)
    X, V = X[:, None, :], V[:, None, :]
    vhat = V / np.linalg.norm(V, axis=-1, keepdims=True)
    R = ref_radar.slant_range_time * SOL / 2.0 + np.arange(S, dtype=np.float64)[None, :] * (
        SOL / 2.0 / ref_radar.range_sampling_rate)
    la, lo = lat.astype(np.float64).copy(), lon.astype(np.float64).copy()
    h = np.broadcast_to(np.asarray(h, dtype=np.float64), la.shape)

    def resid(a, b):
        d = og.llh2xyz(np.stack([a, b, h], axis=-1)) - X
        return np.linalg.norm(d, axis=-1) - R, (d * vhat).sum(-1)

    e = 1e-7
    for _ in range(iters):
        f1, f2 = resid(la, lo)
        a1, a2 = resid(la + e, lo)
        b1, b2 = resid(la - e, lo)
        c1, c2 = resid(la, lo + e)
        d1, d2 = resid(la, lo - e)
        j11, j21 = (a1 - b1) / (2 * e), (a2 - b2) / (2 * e)
        j12, j22 = (c1 - d1) / (2 * e), (c2 - d2) / (2 * e)
        det = j11 * j22 - j12 * j21
        la = la - (j22 * f1 - j12 * f2) / det
        lo = lo - (-j21 * f1 + j11 * f2) / det
    return la, lo


def sensitivities_fd(lat, lon, hgt, sec_radar, sec_orbit, sec_burst_time, ref_radar, ref_orbit, ref_burst_time,
                     step=5.0):
    """daz/dh, drg/dh by central differences of the float64 secondary offsets,
    the ground point of each reference sample moved along the reference's
    iso-range zero-Doppler circle to height hgt +- step."""
    out = []
    for s in (step, -step):
        la, lo = on_reference_circle(lat, lon, hgt + s, ref_radar, ref_orbit, ref_burst_time)
        _, _, a, r = orr.offsets(la, lo, hgt + s, sec_radar, sec_orbit, sec_burst_time)
        out.append((a, r))
    (a1, r1), (a2, r2) = out
    return (a1 - a2) / (2 * step), (r1 - r2) / (2 * step)


def torch_gradient(bursts, params, dh, rl, cl):
    """J and its gradient by torch.autograd in float64 (same model, exact
    sinc weights): returns (J, dJ/dparams [n, 6], dJ/ddh [n, L, S])."""
    import torch
    taps = torch.arange(-3, 5, dtype=torch.float64)
    p = torch.tensor(np.asarray(params, dtype=np.float64), requires_grad=True)
    h = torch.tensor(np.asarray(dh, dtype=np.float64), requires_grad=True)
    tot = 0.0
    n = 0
    for k, b in enumerate(bursts):
        L, S = b.az0.shape
        xa, xr = (torch.from_numpy(v) for v in basis(L, S))
        rows = torch.arange(L, dtype=torch.float64)[:, None]
        cols = torch.arange(S, dtype=torch.float64)[None, :]
        az = rows + torch.from_numpy(b.az0.astype(np.float64)) + p[k, 0] + p[k, 1] * xa + p[k, 2] * xr \
            + torch.from_numpy(b.daz_dh.astype(np.float64)) * h[k]
        rg = cols + torch.from_numpy(b.rg0.astype(np.float64)) + p[k, 3] + p[k, 4] * xa + p[k, 5] * xr \
            + torch.from_numpy(b.drg_dh.astype(np.float64)) * h[k]
        Ls, Ss = b.sec.shape
        rr = np.arange(Ls, dtype=np.float64)[:, None]
        cc = np.arange(Ss, dtype=np.float64)[None, :]
        der = torch.from_numpy(b.sec.astype(np.complex128) * np.exp(1j * orr.tops_phase(b.radar, b.co, rr, cc)))
        na = torch.floor(az).detach()
        nr = torch.floor(rg).detach()
        fa, fr = az - na, rg - nr
        ok = (na - 3 >= 0) & (na + 4 < Ls) & (nr - 3 >= 0) & (nr + 4 < Ss)

        def weights(f):
            x = taps - f[..., None]
            w = torch.sinc(x) * (0.5 + 0.5 * torch.cos(PI * x / 4.0))
            return w / w.sum(-1, keepdim=True)

        wa, wr = weights(fa), weights(fr)
        nai = torch.where(ok, na, torch.full_like(na, 3)).long()
        nri = torch.where(ok, nr, torch.full_like(nr, 3)).long()
        acc = torch.zeros(az.shape, dtype=torch.complex128)
        for i, ka in enumerate(range(-3, 5)):
            row = torch.zeros(az.shape, dtype=torch.complex128)
            for j, kr in enumerate(range(-3, 5)):
                row = row + wr[..., j] * der[nai + ka, nri + kr]
            acc = acc + wa[..., i] * row
        # reramp: exp(-i tops_phase(az, rg)), tops_phase = -pi kt (eta - etaref)^2
        ati = b.radar.azimuth_time_interval
        tr = b.radar.slant_range_time + rg / b.radar.range_sampling_rate
        fm0, fm1, fm2, fm3 = b.co.fm
        dc0, dc1, dc2, dc3 = b.co.dc
        ka_ = fm1 + (tr - fm0) * (fm2 + fm3 * (tr - fm0))
        fnc = dc1 + (tr - dc0) * (dc2 + dc3 * (tr - dc0))
        kt = ka_ * b.co.ks / (ka_ - b.co.ks)
        etaref = -fnc / ka_ - b.co.etac0
        eta = -Ls * ati / 2.0 + az * ati
        ph = -PI * kt * (eta - etaref) ** 2
        s = torch.where(ok, acc * torch.exp(-1j * ph), torch.zeros_like(acc))
        nrw, ncw = L // rl, S // cl
        r = torch.from_numpy(b.ref.astype(np.complex128))[:nrw * rl, :ncw * cl]
        s = s[:nrw * rl, :ncw * cl]

        def box(x):
            return x.reshape(nrw, rl, ncw, cl).sum(dim=(1, 3))
        I = box(torch.conj(r) * s)
        P1 = box(r.abs() ** 2)
        P2 = box(s.abs() ** 2)
        g = I.abs() / torch.sqrt(P1 * P2)
        g = torch.where((P1 * P2 > 0) & (I.abs() > 0), g, torch.zeros_like(g))
        tot = tot + g.sum()
        n += g.numel()
    J = -tot / n
    J.backward()
    return float(J), p.grad.numpy(), h.grad.numpy()
