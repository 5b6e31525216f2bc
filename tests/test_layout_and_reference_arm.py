"""Host-side pieces that need no GPU: the detector-layout detection the _C
drop-in uses to pick the column walk for bare ray lists, and the isolation of
bench.py's reference arm (it must map the oracle's library, not ours)."""
import json
import os
import subprocess
import sys

import torch

from conftest import ROOT


def _cone_rays(n_view=3, det_nx=40, det_ny=64):
    from ct_laboratory_b200.ray_geometry import build_conebeam_3d_geometry
    return build_conebeam_3d_geometry(n_view, det_nx, det_ny, 100.0, 150.0, 0.8)


def test_layout_of_a_cone_beam_scan_is_view_row_column():
    from ct_laboratory_b200._layout import _layout, detect_tiling, clear_cache
    src, dst = _cone_rays()
    assert _layout(src, dst) == (3, 64, 40, 64 * 40, 40, 1)
    clear_cache()
    t = detect_tiling(src, dst)
    assert (t.n_view, t.n_row, t.n_col, t.view_stride, t.row_stride, t.col_stride, t.tile_rows, t.voxel_rule) == \
        (3, 64, 40, 2560, 40, 1, 32, 0)
    assert detect_tiling(src, dst) is t  # cached per storage and version


def test_layout_of_staticct_modules_is_rows_fastest():
    from ct_laboratory_b200._layout import _layout, detect_tiling
    from ct_laboratory_b200.workloads import StaticRingWorkload
    w = StaticRingWorkload(n=(32, 32, 8), n_source=4, n_module=12, det_nx=6, modules_per_source=4,
                           rotations_deg=(0.0,))
    src, dst, _, _ = w.geometry()
    per_view = 4 * 6 * 16
    assert _layout(src, dst) == (4, 16, per_view // 16, per_view, 1, 16)
    assert detect_tiling(src, dst).tile_rows == 16


def test_layout_rejects_unstructured_ray_lists():
    from ct_laboratory_b200._layout import detect_tiling
    src, dst = _cone_rays()
    perm = torch.randperm(src.shape[0], generator=torch.Generator().manual_seed(0))
    assert detect_tiling(src[perm].contiguous(), dst[perm].contiguous()) is None
    assert detect_tiling(src[:20].contiguous(), dst[:20].contiguous()) is None


def test_reference_arm_maps_only_the_oracle():
    code = f"""
import sys
sys.path.insert(0, {ROOT!r})
import bench
class A: pass
a = A(); a.workload = 'fan256'; a.warmup = 0; a.steps = 1; a.ref_step_s = 0.5
bench.run_reference(a, 1, 0)
libs = sorted({{l.split()[-1] for l in open('/proc/self/maps') if l.rstrip().endswith('.so')}})
print('LIBS', [l for l in libs if {ROOT!r} in l])
"""
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = [l for l in out.stdout.splitlines() if l.startswith("{")][0]
    rec = json.loads(line)
    assert rec["impl"] == "reference" and rec["value"] > 0 and rec["cpu_baseline"]["kind"] == "port"
    libs = eval(out.stdout.split("LIBS", 1)[1].strip())
    assert libs and all(os.sep + "oracle" + os.sep in p for p in libs), libs
