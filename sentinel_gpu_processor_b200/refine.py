"""Coherence-maximising coregistration refinement: the objective
J = -mean multilooked coherence of resample -> crossmul -> multilook ->
coherence over a stack of bursts, with its hand-written adjoint behind a
``torch.autograd.Function`` (libs1b ``s1b_adjoint_run``; no counterpart in
the reference).

Unknowns per burst: an offset polynomial (6 parameters, samples)
    d_az = p0 + p1 xa + p2 xr,   d_rg = p3 + p4 xa + p5 xr,
    xa = (row - L/2) / L,  xr = (col - S/2) / S,
and a per-pixel height-error field dh (metres) entering the offsets through
their height sensitivities (``kernels.geo2rdr_offsets_dh``).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib, kernels


class CoregProblem:
    """A stack of n bursts of one size [L, S] on one device.

    ref, sec: complex64 [n, L, S] (reference grid / secondary bursts as
    acquired); az0, rg0, daz_dh, drg_dh: float32 [n, L, S]; sec_plans: the
    secondary burst plans."""

    def __init__(self, sec_plans, ref, sec, az0, rg0, daz_dh, drg_dh, rowlook, collook):
        n, L, S = ref.shape
        for t in (ref, sec):
            if t.dtype != torch.complex64 or not t.is_contiguous() or not t.is_cuda:
                raise ValueError("ref/sec must be contiguous complex64 CUDA tensors")
        for t in (az0, rg0, daz_dh, drg_dh):
            if t.dtype != torch.float32 or tuple(t.shape) != (n, L, S) or not t.is_contiguous() or not t.is_cuda:
                raise ValueError("offsets and sensitivities must be contiguous float32 [n, L, S] CUDA tensors")
        if len(sec_plans) != n or sec.numel() != n * sec_plans[0].lines * sec_plans[0].samples:
            raise ValueError("one secondary plan per burst, sec sized by the plans")
        self.n, self.L, self.S = n, L, S
        self.ref, self.sec, self.az0, self.rg0, self.daz_dh, self.drg_dh = ref, sec, az0, rg0, daz_dh, drg_dh
        self.dev = ref.device
        lib = _lib.load()
        arr = (_lib.BurstPlan * n)(*sec_plans)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.dev):
            _lib.check(lib.s1b_adjoint_create(arr, n, L, S, int(rowlook), int(collook), ctypes.byref(h)),
                       "s1b_adjoint_create")
        self._h = h
        self.ws_bytes = int(lib.s1b_adjoint_workspace_bytes(h))
        self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device=self.dev)
        self.J = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self.windows = n * (L // rowlook) * (S // collook)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().s1b_adjoint_destroy(h)
            except Exception:
                pass
            self._h = None

    def _check(self, params, dh):
        if params.dtype != torch.float32 or tuple(params.shape) != (self.n, 6) or not params.is_contiguous():
            raise ValueError("params must be contiguous float32 [n, 6]")
        if dh.dtype != torch.float32 or tuple(dh.shape) != (self.n, self.L, self.S) or not dh.is_contiguous():
            raise ValueError("dh must be contiguous float32 [n, L, S]")

    def _run(self, params, dh, gp, gh):
        self._check(params, dh)
        _lib.check(kernels._call("adjoint", _lib.load().s1b_adjoint_run, self._h, _lib.dptr(self.ref),
                                 _lib.dptr(self.sec), _lib.dptr(self.az0), _lib.dptr(self.rg0),
                                 _lib.dptr(self.daz_dh), _lib.dptr(self.drg_dh), _lib.dptr(params), _lib.dptr(dh),
                                 _lib.dptr(self.J), _lib.dptr(gp), _lib.dptr(gh), _lib.dptr(self.ws),
                                 self.ws_bytes, _lib.stream_ptr()), "s1b_adjoint_run")

    def objective(self, params, dh):
        """J (float64 device scalar, a view of this problem's buffer)."""
        self._run(params, dh, None, None)
        return self.J[0]

    def gradient(self, params, dh, gp=None, gh=None):
        """(J, dJ/dparams [n, 6], dJ/ddh [n, L, S]) from one fused pass."""
        if gp is None:
            gp = torch.empty((self.n, 6), dtype=torch.float32, device=self.dev)
        if gh is None:
            gh = torch.empty((self.n, self.L, self.S), dtype=torch.float32, device=self.dev)
        self._run(params, dh, gp, gh)
        return self.J[0], gp, gh


class CoherenceObjective(torch.autograd.Function):
    """J(params, dh) of a :class:`CoregProblem`; the backward is the fused
    adjoint (window sums recomputed, not stored)."""

    @staticmethod
    def forward(ctx, params, dh, problem):
        ctx.problem = problem
        ctx.save_for_backward(params, dh)
        return problem.objective(params.detach().contiguous(), dh.detach().contiguous()).clone()

    @staticmethod
    def backward(ctx, grad_out):
        params, dh = ctx.saved_tensors
        _, gp, gh = ctx.problem.gradient(params.detach().contiguous(), dh.detach().contiguous())
        g = grad_out.to(torch.float32)
        return gp * g, gh * g, None


def refine(problem: CoregProblem, steps=50, lr_params=0.01, lr_dh=0.5, params=None, dh=None, history=False):
    """Adam on (params, dh) to maximise the mean multilooked coherence.
    Returns (params, dh, [J per step] if ``history``)."""
    if params is None:
        params = torch.zeros((problem.n, 6), dtype=torch.float32, device=problem.dev)
    if dh is None:
        dh = torch.zeros((problem.n, problem.L, problem.S), dtype=torch.float32, device=problem.dev)
    params = params.clone().requires_grad_(True)
    dh = dh.clone().requires_grad_(True)
    opt = torch.optim.Adam([{"params": [params], "lr": lr_params}, {"params": [dh], "lr": lr_dh}])
    hist = []
    for _ in range(steps):
        opt.zero_grad(set_to_none=False)
        J = CoherenceObjective.apply(params, dh, problem)
        J.backward()
        opt.step()
        if history:
            hist.append(J.detach())
    out = (params.detach(), dh.detach())
    if history:
        return out + ([float(j) for j in torch.stack(hist).cpu()],)
    return out
