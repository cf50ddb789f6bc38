"""The bench's JSON contract on CPU: the reference arm's line (its keys, the same workload
config as ours, a CPU-baseline block, an e2e block without copies) and the pieces of our
line that need no GPU."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1", "--ref-n", "20000"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT, env={**os.environ, "RANK": "0", "WORLD_SIZE": "1"})
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "dtype",
                "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    # the config names the N actually timed (the headline's own N by default)
    assert line["config"] == bench.headline_config(20000, 1) and line["config"]["n_points"] == 20000
    assert line["ms_per_step"] > 0 and abs(20000 / (line["ms_per_step"] * 1e-3) / 1e6 - line["value"]) < 1e-3 * line["value"] + 1e-3
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and "N=20000" in cb["sample"] and cb["value"] == line["value"]
    e = line["e2e"]
    assert e["value"] == line["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_passes_hbm_figures():
    info = {"nboxes": 1000, "nleaves": 800, "nsources": 50000, "ntargets": 50000, "w_pairs": 2000}
    kinds = {"p2m": 0.5, "m2m": 0.25, "l2l": 0.25, "l2p_m2p": 1.0}
    out = bench.passes_hbm(info, kinds, {"hbm_gbs": 6000.0})
    nc = (bench.P + 1) ** 2
    assert out["m2m"]["bytes"] == 2 * 1000 * nc * 4
    assert abs(out["m2m"]["gbs"] - out["m2m"]["bytes"] / 0.25e-3 / 1e9) < 0.1
    assert out["peak_gbs"] == 6000.0 and 0 < out["l2p_m2p"]["frac"] < 1


def test_cpu_baseline_is_a_median_of_five():
    class A:
        cpu_n = 20000

    b = bench.cpu_baseline(A())
    assert len(b["evaluations_s"]) == bench.CPU_REPEATS >= 5 and b["n_points"] == 20000
    import numpy as np

    assert abs(b["value"] - 20000 / float(np.median(b["evaluations_s"])) / 1e6) < 0.02 * b["value"]
