"""The coherence objective and its hand-written adjoint (s1b_adjoint_run)
against the float64 oracle (oracle/adjoint.py): objective value, the
torch.autograd float64 reference gradient, central finite differences (step
1e-4 px for the offset polynomials, 1e-2 m along a height-error direction),
height sensitivities of the offsets, the autograd.Function and a short
refinement.  Gradient tolerance (north star): relative error <= 1e-3."""
import numpy as np
import pytest
import torch

from helpers import oracle_burst, oracle_radar
from oracle import adjoint as oa
from oracle import geo2rdr as og2
from sentinel_gpu_processor_b200 import kernels, plan as P, synth
from sentinel_gpu_processor_b200.refine import CoherenceObjective, CoregProblem, refine

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stack(cuda):
    return synth.make_refine_stack(n_bursts=2, config="tiny", seed=5, device=cuda, keep_geometry=True, margin=12)


@pytest.fixture(scope="module")
def problem(stack):
    return CoregProblem(stack.sec_plans, stack.ref, stack.sec, stack.az0, stack.rg0, stack.daz_dh, stack.drg_dh,
                        stack.rowlook, stack.collook)


def _direction(dh):
    g = torch.Generator(device=dh.device)
    g.manual_seed(17)
    d = synth.gaussian_smooth(torch.randn(dh.shape, generator=g, device=dh.device), 4.0)
    return (d / d.std()).cpu().numpy().astype(np.float64)


@pytest.fixture(scope="module")
def point(stack, cuda):
    """An evaluation point away from the truth (random parameters, a smoothed
    height error) at which no pixel crosses the burst edge under the
    finite-difference steps."""
    g = torch.Generator(device=cuda)
    g.manual_seed(9)
    dh = synth.gaussian_smooth(torch.randn(stack.dh_true.shape, generator=g, device=cuda), 6.0)
    dh = (dh * (3.0 / dh.std())).contiguous()
    bursts = _oracle_bursts(stack)
    d = _direction(dh)
    for seed in range(3, 40):
        rng = np.random.default_rng(seed)
        p = rng.normal(0, 0.03, (stack.ref.shape[0], 6))
        params = torch.tensor(p, dtype=torch.float32, device=cuda)
        if oa.fd_stable(bursts, params.cpu().numpy(), dh.cpu().numpy(), d):
            return params, dh
    pytest.fail("no evaluation point without support-edge crossings")


def _oracle_bursts(stack):
    acq = stack.sec_acq
    radar = oracle_radar(acq.radar)
    co = og2.burst_coefficients(radar, acq.orbit, acq.fm, acq.dc, oracle_burst(acq.bursts[0]))
    out = []
    for b in range(stack.ref.shape[0]):
        out.append(oa.AdjBurst(ref=stack.ref[b].cpu().numpy(), sec=stack.sec[b].cpu().numpy(), radar=radar, co=co,
                               az0=stack.az0[b].cpu().numpy(), rg0=stack.rg0[b].cpu().numpy(),
                               daz_dh=stack.daz_dh[b].cpu().numpy(), drg_dh=stack.drg_dh[b].cpu().numpy()))
    return out


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_height_sensitivities_match_finite_differences(stack):
    lat, lon, hgt = (t.cpu().numpy() for t in stack.geometry)
    sa, ra = stack.sec_acq, stack.ref_acq
    fa, fr = oa.sensitivities_fd(lat, lon, hgt, oracle_radar(sa.radar), sa.orbit, sa.bursts[0].azimuth_time,
                                 oracle_radar(ra.radar), ra.orbit, ra.bursts[0].azimuth_time)
    m = stack.margin
    fa, fr = fa[m:-m, m:-m], fr[m:-m, m:-m]
    ga, gr = stack.daz_dh[0].cpu().numpy(), stack.drg_dh[0].cpu().numpy()
    assert np.abs(gr - fr).max() < 1e-4 * np.abs(fr).max()
    assert np.abs(ga - fa).max() < 1e-4 * max(np.abs(fa).max(), 1e-3)
    # the stack's offsets are those of the plain offsets entry point (shifted by the crop)
    az, rg = kernels.geo2rdr_offsets(stack.sec_plans[0], *stack.geometry)
    assert torch.equal(az[m:-m, m:-m] + m, stack.az0[0]) and torch.equal(rg[m:-m, m:-m] + m, stack.rg0[0])


def test_objective_matches_oracle(stack, problem, point):
    params, dh = point
    J = float(problem.objective(params, dh))
    Jo = oa.objective(_oracle_bursts(stack), params.cpu().numpy(), dh.cpu().numpy(), stack.rowlook, stack.collook)
    assert -1.0 < Jo < -0.05
    assert abs(J - Jo) < 2e-6


def test_gradient_matches_torch_autograd(stack, problem, point):
    params, dh = point
    J, gp, gh = problem.gradient(params, dh)
    Jt, tp, th = oa.torch_gradient(_oracle_bursts(stack), params.cpu().numpy(), dh.cpu().numpy(),
                                   stack.rowlook, stack.collook)
    assert abs(float(J) - Jt) < 2e-6
    assert _rel(gp.cpu().numpy(), tp) < 1e-3
    assert _rel(gh.cpu().numpy(), th) < 1e-3


def test_gradient_matches_finite_differences(stack, problem, point):
    params, dh = point
    _, gp, gh = problem.gradient(params, dh)
    bursts = _oracle_bursts(stack)
    p64, h64 = params.cpu().numpy().astype(np.float64), dh.cpu().numpy().astype(np.float64)
    fd = oa.fd_params(bursts, p64, h64, stack.rowlook, stack.collook, step=1e-4)
    assert _rel(gp.cpu().numpy(), fd) < 1e-3
    d = _direction(dh)
    fdd = oa.fd_direction(bursts, p64, h64, d, stack.rowlook, stack.collook, step=1e-2)
    adj = float((gh.cpu().numpy().astype(np.float64) * d).sum())
    assert abs(adj - fdd) <= 1e-3 * abs(fdd)


def test_gradient_is_deterministic(problem, point):
    params, dh = point
    J1, gp1, gh1 = problem.gradient(params, dh)
    J1, gp1, gh1 = float(J1), gp1.clone(), gh1.clone()
    J2, gp2, gh2 = problem.gradient(params, dh)
    assert J1 == float(J2) and torch.equal(gp1, gp2) and torch.equal(gh1, gh2)


def test_autograd_function_and_refinement(stack, problem):
    n = stack.ref.shape[0]
    p0 = torch.zeros((n, 6), dtype=torch.float32, device=stack.ref.device, requires_grad=True)
    h0 = torch.zeros(stack.dh_true.shape, dtype=torch.float32, device=stack.ref.device, requires_grad=True)
    J = CoherenceObjective.apply(p0, h0, problem)
    J.backward()
    _, gp, gh = problem.gradient(p0.detach(), h0.detach())
    assert torch.equal(p0.grad, gp) and torch.equal(h0.grad, gh)
    params, dh, hist = refine(problem, steps=20, history=True)
    assert hist[-1] < hist[0] - 1e-3  # coherence went up

    def offset_error(p, h):
        # rms of the total offset field error (polynomial + height term) vs the truth
        L, S = stack.az0.shape[1:]
        xa = (torch.arange(L, device=p.device)[:, None] - 0.5 * L) / L
        xr = (torch.arange(S, device=p.device)[None, :] - 0.5 * S) / S
        dp = p - stack.params_true
        hh = h - stack.dh_true
        ea = dp[:, 0, None, None] + dp[:, 1, None, None] * xa + dp[:, 2, None, None] * xr + stack.daz_dh * hh
        er = dp[:, 3, None, None] + dp[:, 4, None, None] * xa + dp[:, 5, None, None] * xr + stack.drg_dh * hh
        return float(torch.sqrt((ea ** 2 + er ** 2).mean()))

    assert offset_error(params, dh) < 0.5 * offset_error(torch.zeros_like(params), torch.zeros_like(dh))
