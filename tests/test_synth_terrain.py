"""The DEM-as-terrain function of the synthetic scenes (``synth.dem_height_fn``):
exact at the grid's points, bilinear between them, clamped at the edges;
and the synthetic rdr2geo with ``terrain=True`` puts every pixel's ground
point on that terrain (host, small burst)."""
import torch

from sentinel_gpu_processor_b200 import formats, synth


def test_dem_height_fn_is_bilinear_and_exact_on_the_grid():
    rsc = formats.Rsc(nlat=5, nlon=7, latmax=36.0, lonmin=10.0, dlat=-0.25, dlon=0.125)
    gen = torch.Generator()
    gen.manual_seed(1)
    dem = torch.randint(-100, 3000, (5, 7), generator=gen).to(torch.int16)
    f = synth.dem_height_fn(rsc, dem)
    lat = rsc.latmax + rsc.dlat * torch.arange(5, dtype=torch.float64)[:, None].expand(5, 7)
    lon = rsc.lonmin + rsc.dlon * torch.arange(7, dtype=torch.float64)[None, :].expand(5, 7)
    assert torch.equal(f(lat, lon), dem.to(torch.float64))
    # the centre of a cell is the mean of its four corners
    la = torch.tensor([rsc.latmax + 1.5 * rsc.dlat], dtype=torch.float64)
    lo = torch.tensor([rsc.lonmin + 2.5 * rsc.dlon], dtype=torch.float64)
    want = dem[1:3, 2:4].to(torch.float64).mean()
    assert torch.allclose(f(la, lo), want.reshape(1))
    # outside the grid: the edge values
    far = f(torch.tensor([40.0, 30.0], dtype=torch.float64), torch.tensor([0.0, 20.0], dtype=torch.float64))
    assert far.tolist() == [float(dem[0, 0]), float(dem[4, 6])]


def test_rdr2geo_terrain_points_lie_on_the_terrain():
    sc = synth.make_frame(n_swaths=1, n_bursts=1, scale=0.02, slc_pairs=0)
    acq = sc.ref[0]
    f = synth.dem_height_fn(sc.rsc, sc.dem)
    lat, lon, hgt = synth.rdr2geo_grid(acq.orbit, acq.radar, acq.bursts[0], f, terrain=True)
    # the bisection ends where the ray crosses the terrain: the two differ by
    # what one step of the look angle moves the ray (well under a millimetre)
    assert (hgt - f(lat, lon)).abs().max().item() < 1e-3
