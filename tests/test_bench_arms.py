"""The two arms of bench.py time the same frame: the reference arm builds its
scene without the s1b library (the oracle's footprint boxes) and must pick
the same DEM grid and report the same ``config`` as the s1b arm (the
library's planner); the reference arm's process maps none of the
repository's shared objects."""
import json
import os
import subprocess
import sys
from types import SimpleNamespace

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

CODE = r"""
import json, sys
sys.path.insert(0, {root!r})
import bench
from types import SimpleNamespace
from oracle import refrun
from sentinel_gpu_processor_b200 import synth
synth.make_dem = lambda rsc, seed, hmax, device="cpu": None  # the grid, not the terrain, is under test
sc = bench.frame_scene("frame_small", 0, "cpu", refrun.footprint_boxes, slc_pairs=1)
cfg = bench.frame_config(SimpleNamespace(config="frame_small", samples="c64"), sc, 1)
print(json.dumps({{"cfg": cfg, "mapped": bench._repo_libraries_mapped(),
                  "lib": "sentinel_gpu_processor_b200._lib" in sys.modules}}))
"""


def test_reference_arm_scene_matches_s1b_arm_and_maps_no_repo_library(monkeypatch):
    r = subprocess.run([sys.executable, "-c", CODE.format(root=ROOT)], stdout=subprocess.PIPE, text=True, check=True,
                       env={**os.environ, "CUDA_VISIBLE_DEVICES": ""})
    ref = json.loads(r.stdout.strip().splitlines()[-1])
    assert ref["lib"] is False
    assert ref["mapped"] == []
    sys.path.insert(0, ROOT)
    import bench
    from sentinel_gpu_processor_b200 import plan, synth
    monkeypatch.setattr(synth, "make_dem", lambda rsc, seed, hmax, device="cpu": None)
    sc = bench.frame_scene("frame_small", 0, "cpu", plan.footprint_boxes, slc_pairs=1)
    cfg = bench.frame_config(SimpleNamespace(config="frame_small", samples="c64"), sc, 1)
    assert json.loads(json.dumps(cfg)) == ref["cfg"]
