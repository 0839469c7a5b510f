"""The drop-in, end to end: the reference's own program (AmrManager set-up, SetupMesh, its
TimeMarching loop) with the GridInfoLbmB200 plugin (zllbm_b200/plugin) in place of the
reference's GridInfoLbmInteface, against the same program without it.

``oracle/_ref/zl_ref_run_b200`` is the oracle harness built with the plugin
(``make -C oracle plugin``): each level's AdvancingAtCurrentTime runs on the GPU through the C
ABI and the populations come back into the reference's nodes before the dump.  FP64 storage:
every level's populations bit for bit, immersed-boundary runs to 1e-12 (node forces summed over
vertices in another order than the reference's unordered_map walk); FP32 storage within 1e-5.
"""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "zl_ref_run")
PLUGIN = os.path.join(ROOT, "oracle", "_ref", "zl_ref_run_b200")

CASES = {
    "cavity2d_srt": ["dims=2", "n=15,15", "coll=srt", "nu=0.016", "bc=xmin:bb", "bc=xmax:bb", "bc=ymin:bb",
                     "bc=ymax:bb:0.1,0", "steps=200"],
    "tgv3d_mrt": ["dims=3", "n=10,10,10", "coll=mrt", "nu=0.016666666666666666", "init=tgv", "u0=0.05", "steps=30"]
                 + [f"bc={f}:per" for f in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")],
    "box3d_mixed": ["dims=3", "n=9,7,8", "coll=mrt", "nu=0.05", "bc=xmin:neq:0.05,0,0", "bc=xmax:neq:0.05,0,0",
                    "bc=ymin:bb", "bc=ymax:bb:0.03,0,0.01", "bc=zmin:per", "bc=zmax:per", "steps=30"],
    "force2d_mrt": ["dims=2", "n=12,10", "coll=mrt", "nu=0.05", "cforce=1e-4,2e-5", "forces=1", "bc=xmin:per",
                    "bc=xmax:per", "bc=ymin:bb", "bc=ymax:bb", "steps=40"],
    "amr2d_l2": ["dims=2", "n=48,40", "levels=2", "geo=circle:24,20,2", "ext=3", "inner=2", "coll=mrt", "nu=0.01",
                 "bc=xmin:neq:0.04,0", "bc=xmax:neq:0.04,0", "bc=ymin:bb", "bc=ymax:bb:0.02,0", "steps=4"],
    "amr3d_l1": ["dims=3", "n=20,16,16", "levels=1", "geo=cube:10,8,8,2", "ext=2", "inner=1", "coll=mrt", "nu=0.02",
                 "bc=xmin:neq:0.05,0,0", "bc=xmax:neq:0.05,0,0", "bc=ymin:bb", "bc=ymax:bb", "bc=zmin:bb",
                 "bc=zmax:bb", "steps=3"],
    "ib2d_l1": ["dims=2", "n=48,40", "levels=1", "ib=circle:24.3,20.1,2.5", "ext=3", "inner=2", "coll=mrt",
                "nu=0.01", "vel=0.04,0", "bc=xmin:neq:0.04,0", "bc=xmax:neq:0.04,0", "bc=ymin:bb", "bc=ymax:bb",
                "steps=6"],
}


def run(exe, args, tmp, tag):
    from oracle.port import load_levels
    out = os.path.join(tmp, f"{tag}.bin")
    subprocess.run([exe] + args + [f"lout={out}"], check=True, cwd=tmp, stdout=subprocess.DEVNULL)
    return load_levels(out)[2]


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_time_loop_with_the_plugin(name, tmp_path):
    if not os.path.exists(PLUGIN):
        pytest.fail("oracle/_ref/zl_ref_run_b200 is missing: make -C oracle plugin")
    args = CASES[name]
    cpu = run(REF, args, str(tmp_path), "cpu")
    gpu = run(PLUGIN, args + ["b200=f64"], str(tmp_path), "gpu")
    f32 = run(PLUGIN, args + ["b200=f32"], str(tmp_path), "f32")
    assert len(cpu) == len(gpu) == len(f32)
    for lv, (a, b, c) in enumerate(zip(cpu, gpu, f32)):
        assert np.array_equal(a["nodes"]["code"], b["nodes"]["code"])
        fa, fb, fc = a["nodes"]["f"], b["nodes"]["f"], c["nodes"]["f"]
        if "ib=" in " ".join(args):
            np.testing.assert_allclose(fb, fa, rtol=1e-12, atol=1e-15, err_msg=f"level {lv}")
        else:
            assert np.array_equal(fb, fa), (lv, float(np.abs(fb - fa).max()))
        assert (np.abs(fc - fa) / np.abs(fa)).max() <= 1e-5, lv
