"""Complex int16 ingest on the GPU: the CInt16 deramp, the read-ahead burst
stream, geo2rdr fed from a measurement TIFF and the batched frame on CInt16
samples.  Widening int16 to float is exact, so every result must equal the
complex64 path on the widened samples bit for bit -- the path the reference
takes after GDAL widens the TIFF on the host (s1proc/sentinel_scene.py:
164-207)."""
import io
import os

import numpy as np
import pytest
import torch

from helpers import GOLD, golden_acq, golden_rsc, write_cint16_tiff
from oracle import refrun
from sentinel_gpu_processor_b200 import cli, formats, kernels, plan as _plan, synth
from sentinel_gpu_processor_b200.chain import BatchedFrameChain
from sentinel_gpu_processor_b200.ingest import BurstStream, MeasurementTiff

pytestmark = pytest.mark.gpu


def _quantise(x, scale=2000.0):
    """complex64 -> int16 [..., 2] (re, im) and the complex64 of those integers."""
    x = torch.as_tensor(x)
    q = torch.stack([x.real, x.imag], -1).mul(scale).round().clamp(-32768, 32767).to(torch.int16)
    return q.contiguous(), torch.complex(q[..., 0].float(), q[..., 1].float())


@pytest.fixture(scope="module")
def tiny():
    return synth.make_pair("tiny", seed=21)


def _plan_of(sc):
    a = sc.ref[0]
    return _plan.burst_plan(a.radar, a.orbit, a.fm, a.dc, a.bursts[0], sc.rsc)


def test_deramp_ci16_equals_widened(cuda, tiny):
    pl = _plan_of(tiny)
    q, w = _quantise(tiny.ref_slc[0])
    q, w = q.to(cuda).reshape(-1, 2), w.to(cuda).reshape(-1)
    got = kernels.deramp(pl, q)
    want = kernels.deramp(pl, w)
    assert torch.equal(torch.view_as_real(got), torch.view_as_real(want))
    # an odd start (4-byte aligned only) takes the one-sample path
    buf = torch.empty((q.shape[0] + 1, 2), dtype=torch.int16, device=cuda)
    buf[1:] = q
    got2 = kernels.deramp(pl, buf[1:])
    assert torch.equal(torch.view_as_real(got2), torch.view_as_real(want))


def test_deramp_ci16_odd_width(cuda, tiny):
    pl = _plan_of(tiny)
    pl.samples -= 1  # odd width: one-sample loads throughout
    q, w = _quantise(tiny.ref_slc[0][:, :pl.samples])
    got = kernels.deramp(pl, q.to(cuda).reshape(-1, 2))
    want = kernels.deramp(pl, w.to(cuda).reshape(-1))
    assert torch.equal(torch.view_as_real(got), torch.view_as_real(want))


def test_burst_stream_reads_ahead_in_order(cuda, tmp_path):
    L, n, w = 40, 5, 300
    a = np.random.default_rng(4).integers(-3000, 3000, size=(L * n, w, 2), dtype=np.int16)
    p = str(tmp_path / "m.tiff")
    write_cint16_tiff(p, a, rows_per_strip=1)
    acc = []
    with MeasurementTiff(p) as t:
        bs = BurstStream(t, L, n, indices=[0, 2, 3, 4])
        for k, dev in bs:
            assert dev.is_cuda and dev.shape == (L, w, 2)
            # work queued on the current stream reads the burst before the
            # next step may overwrite its buffer
            acc.append((k, dev.to(torch.int32).sum(dim=(0, 1)), dev.clone()))
        torch.cuda.synchronize()
        assert bs.bytes_read == 4 * L * w * 4
    for k, s, d in acc:
        want = a[k * L:(k + 1) * L]
        assert torch.equal(d.cpu(), torch.from_numpy(want))
        assert torch.equal(s.cpu(), torch.from_numpy(want.astype(np.int32).sum(axis=(0, 1))))


@pytest.fixture(scope="module")
def golden_files(cuda, tmp_path_factory):
    z = np.load(GOLD)
    wd = str(tmp_path_factory.mktemp("ingest"))
    rscf, demf = refrun.write_dem(wd, golden_rsc(z), z["dem"])
    out = {}
    for tag in ("ref", "sec"):
        q, w = _quantise(torch.from_numpy(np.ascontiguousarray(z[tag + "_slc"])))
        db = refrun.write_geo2rdr_inputs(wd, tag, golden_acq(z, tag + "_"), [w.numpy()], rscf, demf)
        tif = os.path.join(wd, tag + ".tiff")
        write_cint16_tiff(tif, q.numpy(), rows_per_strip=1)
        out[tag] = (db, tif, w.numpy())
    return wd, out


@pytest.mark.parametrize("zipped", [False, True])
def test_geo2rdr_from_tiff_equals_stdin(golden_files, zipped):
    import zipfile
    wd, files = golden_files
    for tag, (db, tif, w) in files.items():
        src = tif
        if zipped:
            zp = os.path.join(wd, tag + "_SAFE.zip")
            with zipfile.ZipFile(zp, "w", compression=zipfile.ZIP_STORED) as zf:
                zf.write(tif, "SAFE/measurement/s1.tiff")
            src = zp + "::SAFE/measurement/s1.tiff"
        a = os.path.join(wd, f"tiff{int(zipped)}_{tag}")
        b = os.path.join(wd, f"pipe{int(zipped)}_{tag}")
        assert cli.geo2rdr_main(["geo2rdr", db, a, "--tiff", src]) == 0
        assert cli.geo2rdr_main(["geo2rdr", db, b, "--stdin"], stdin=io.BytesIO(w.tobytes())) == 0
        ha, da = formats.read_raster(a + "_burst_0.gslc")
        hb, db_ = formats.read_raster(b + "_burst_0.gslc")
        np.testing.assert_array_equal(ha, hb)
        assert np.array_equal(da.view(np.uint64), db_.view(np.uint64))


def test_geo2rdr_tiff_errors(golden_files, capsys):
    wd, files = golden_files
    db = files["ref"][0]
    assert cli.geo2rdr_main(["geo2rdr", db, os.path.join(wd, "x"), "--tiff", os.path.join(wd, "missing.tiff")]) == 1
    assert "Error" in capsys.readouterr().err


def test_frame_ci16_equals_c64(cuda):
    f = synth.make_frame(seed=7, device=cuda, n_swaths=2, n_bursts=2, scale=0.12)
    qr = [_quantise(s) for s in f.ref_slc]
    qs = [_quantise(s) for s in f.sec_slc]
    outs = []
    for fmt in ("c64", "ci16"):
        bc = BatchedFrameChain(f.ref, f.sec, f.rsc, f.rowlook, f.collook, f.alpha, device=cuda, sample_format=fmt)
        k = 0 if fmt == "ci16" else 1
        bc.load([q[k] for q in qr], [q[k] for q in qs])
        for tuning in ((16, 0, 128, 0), (8, 148, 64, 148)):  # per-tile and persistent deramp
            bc.set_tuning(*tuning)
            bc.run(f.dem)
            res = bc.results()
            outs.append([None if r is None else (r.ifg.clone(), r.coh.clone(), r.filt.clone()) for r in res])
        assert bc.launches_per_step() >= 7
    base = outs[0]
    assert any(r is not None for r in base)
    for o in outs[1:]:
        for r, w in zip(o, base):
            assert (r is None) == (w is None)
            if r is not None:
                for x, y in zip(r, w):
                    assert torch.equal(torch.view_as_real(x) if x.is_complex() else x,
                                       torch.view_as_real(y) if y.is_complex() else y)
