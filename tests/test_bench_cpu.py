"""CPU checks of bench.py: the reference arm's JSON line (it times the oracle
on the host cores, so it runs here) and the per-kernel byte model."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def run_bench(args, env_extra=None, timeout=600):
    env = dict(os.environ)
    env.update(env_extra or {})
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, capture_output=True, text=True,
                       timeout=timeout, env=env, cwd=ROOT)
    return p


SMALL = ["--frames", "4", "--width", "2048", "--height", "1536"]


def test_reference_arm_prints_the_contract_line():
    p = run_bench(["--impl", "reference", "--steps", "1", "--warmup", "0"] + SMALL)
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["higher_is_better"] is True and line["value"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    # the same workload description as the GPU arm: the ROI is the oracle's
    # restatement of the reference's computeCommonOverlapRoi
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    poses = [oracle.synth_pose(1, oracle.SCENE_PRODUCTION, 2048, 1536, k, 4) for k in range(4)]
    roi = oracle.compute_roi(poses, [2048] * 4, [1536] * 4)
    cfg = line["config"]
    assert cfg["roi"] == list(roi) and cfg["frames"] == 4 and cfg["src"] == [2048, 1536]
    assert cfg["levels"] == len(bench.level_sizes(roi[2] - roi[0], roi[3] - roi[1]))


def test_reference_arm_loads_only_the_oracle():
    """The CPU arm maps no part of the CUDA library: frames, poses and the ROI
    come from the oracle."""
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', "
            + ", ".join(repr(a) for a in SMALL) + "]; runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('LIBS', sorted({l.split()[-1] for l in maps.splitlines() if '.so' in l and 'repo' in l}))")
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    libs = [ln for ln in p.stdout.splitlines() if ln.startswith("LIBS")][0]
    assert "libfocuscuda" not in libs and "liboracle" in libs, libs


def test_reference_arm_runs_on_rank_zero_only():
    p = run_bench(["--impl", "reference", "--steps", "1", "--warmup", "0"] + SMALL,
                  {"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""


def test_level_sizes_halve_with_ceil_down_to_one():
    sizes = bench.level_sizes(7872, 5243)
    assert len(sizes) == 14 and sizes[0] == (7872, 5243) and sizes[1] == (3936, 2622) and sizes[-1] == (1, 1)
    assert bench.level_sizes(1, 1) == [(1, 1)]


@pytest.mark.parametrize("mode", ["laps", "fused", "cache", "recompute"])
def test_algorithmic_bytes_model(mode):
    w, h, f, k = 7872, 5243, 30, 8
    per_kernel, total = bench.algorithmic_bytes(w, h, f, k, mode, 4)
    assert set(per_kernel) == {"pass1", "image", "remap_weights", "blend0", "level0", "level", "collapse",
                               "mask_support"}
    assert all(v >= 0 for v in per_kernel.values()) and total == sum(per_kernel.values())
    per_px = total / (f * w * h)
    # pass 1 reads the 3 B frame; laps and cache also keep 8 B of planes,
    # fused writes the 4 B weight
    assert per_kernel["pass1"] / (f * w * h) > {"laps": 11, "cache": 11, "fused": 7}.get(mode, 3)
    assert 25 < per_px < 100
    if mode in ("laps", "fused"):
        assert per_kernel["image"] > 0 and per_kernel["blend0"] > 0 and per_kernel["remap_weights"] == 0
    if mode == "fused":
        # no level-0 Laplacian or remapped frame through HBM
        assert total < bench.algorithmic_bytes(w, h, f, k, "laps", 4)[1] - 20 * f * w * h
    if mode == "recompute":
        assert per_kernel["remap_weights"] > 0
    # FP16 storage moves fewer level bytes
    assert bench.algorithmic_bytes(w, h, f, k, mode, 2)[1] < total


def test_split_pyramid_byte_model_follows_the_fused_kernels():
    """laps: the level-0 blend reads each frame's Laplacian (12 B) and weight
    (4 B) once and writes its level-1 mask, with no level-0 mask through
    HBM; levels of at least 1184 64x32 tiles (1 and 2 of the bench stack)
    read each frame's mask once for the blend and the REDUCE together."""
    w, h, f, k = 7872, 5243, 30, 8
    per_kernel, _ = bench.algorithmic_bytes(w, h, f, k, "laps", 4)
    sizes = bench.level_sizes(w, h)
    a0, a1, a2 = (sizes[0][0] * sizes[0][1], sizes[1][0] * sizes[1][1], sizes[2][0] * sizes[2][1])
    assert per_kernel["level0"] == 0
    assert per_kernel["blend0"] == f * (16 * a0 + 4 * a1) + 17 * a0
    # the unfused model of the same levels reads every mask of levels 1 and 2 once more
    tiles = [-(-x // 64) * -(-y // 32) for x, y in sizes]
    assert tiles[1] >= 1184 and tiles[2] >= 1184 and tiles[3] < 1184
    L = len(sizes)
    unfused = 0
    for l in range(1, L):  # FP32 storage: 4 B per mask sample, 12 + 4 B per Laplacian + mask
        al = sizes[l][0] * sizes[l][1]
        if l + 1 < L:
            unfused += f * (4 * al + 4 * sizes[l + 1][0] * sizes[l + 1][1]) + al
        unfused += f * 16 * al + 12 * al
    assert unfused - per_kernel["level"] == f * 4 * (a1 + a2)
