"""Host-side logic of bench.py (no GPU): the committed DRAM-traffic data covers every kernel
of the step and is used only for the workload it was captured on, the field-error summary,
and the clock summary reports throttle reasons from any sample."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_traffic_data_covers_every_kernel():
    import json
    d = json.load(open(bench.TRAFFIC_DATA))
    kb = bench.kernel_bytes(*bench.GRID, bench.NPART)
    assert set(d["kernels"]) == set(kb)
    assert tuple(d["workload"]["grid"]) == bench.GRID and d["workload"]["particles"] == bench.NPART
    # x-pair gather: coordinates in, E out, the x-pair grid once
    n = bench.GRID[0] * bench.GRID[1] * bench.GRID[2]
    assert kb["interp_f32"] == 48 * bench.NPART + 32 * n


def test_profiled_traffic_of_the_dominant_kernel():
    t = bench.profiled_traffic("interp_f32", bench.GRID, bench.NPART, "random")
    a = bench.kernel_bytes(*bench.GRID, bench.NPART)["interp_f32"]
    # the measured DRAM traffic is the algorithmic bytes to within 3% (no re-reads)
    assert t is not None and abs(t - a) <= 0.03 * a
    assert bench.profiled_traffic("no_such_kernel", bench.GRID, bench.NPART, "random") is None
    # a capture of another workload is not used
    assert bench.profiled_traffic("interp_f32", (64, 64, 64), bench.NPART, "random") is None
    assert bench.profiled_traffic("interp_f32", bench.GRID, bench.NPART, "sorted") is None


def test_field_errors():
    import numpy as np
    ref = np.random.default_rng(0).standard_normal((100, 3))
    e = bench.field_errors(ref * (1 + 1e-7), ref)
    assert e["max"] <= 1.1e-7 and e["rms"] <= 1.1e-7 and len(e["max_per_component"]) == 3


def test_clock_summary_reasons():
    c = bench.ClockSampler(0)
    c.samples = [(1965.0, 1965.0, set()), (1950.0, 1965.0, {"sw_power_cap"}), (1965.0, 1965.0, set())]
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] == 3
    c.samples = []
    assert c.summary()["samples"] == 0


@pytest.mark.parametrize("np_", [1, 1000, 10 ** 7])
def test_kernel_bytes_scale_with_particles(np_):
    kb0 = bench.kernel_bytes(64, 64, 128, 0)
    kb1 = bench.kernel_bytes(64, 64, 128, np_)
    assert kb1["deposit_f32"] - kb0["deposit_f32"] == 24 * np_
    assert kb1["interp_f32"] - kb0["interp_f32"] == 48 * np_
    assert kb1["fft_z_conv"] == kb0["fft_z_conv"]


def test_plan_launch_never_times_one_gpu_for_several():
    assert bench.plan_launch(1, {}) == ("run", "")
    assert bench.plan_launch(2, {})[0] == "spawn"
    assert bench.plan_launch(4, {"WORLD_SIZE": "4"})[0] == "run"
    assert bench.plan_launch(2, {"WORLD_SIZE": "1"})[0] == "error"
    assert bench.plan_launch(8, {"WORLD_SIZE": "2"})[0] == "error"
    assert bench.plan_launch(0, {})[0] == "error"


def test_gpus_2_without_a_launcher_spawns_two_ranks():
    """`bench.py --gpus 2` started bare runs two ranks itself (gloo on 127.0.0.1); the
    reference arm needs no GPU, so the whole launch path runs here on a tiny workload."""
    import json
    import subprocess
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR",
                                                            "MASTER_PORT")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--np", "20000", "--grid", "16,16,16", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2


def test_gpus_mismatching_the_launcher_is_an_error():
    import subprocess
    env = dict(os.environ, WORLD_SIZE="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 2 and "WORLD_SIZE" in r.stderr
