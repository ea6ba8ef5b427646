"""bench.py's output contract, checked on the CPU: the reference arm (the
reference's own step compiled from its sources where it covers the
workload, else the oracle, timed on the host cores) prints one JSON line
with the keys the driver reads; the GPU arm, on a machine without a GPU, exits with an error
instead of falling back to the CPU."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _run(args, timeout=600):
    env = dict(os.environ)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=timeout)


def _line(out):
    lines = [l for l in out.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out[-2000:]
    return json.loads(lines[0])


@pytest.mark.parametrize("scene", ["c1", "c2", "c4"])
def test_reference_arm_line(scene):
    # c2 at its full size, advanced on the host cores by one settle step
    # (the default settle count takes minutes on a small host); the batch's
    # sample bounded to a few seconds
    extra = {"c2": ["--settle", "1"], "c4": ["--cpu-seconds", "4"]}.get(scene, [])
    r = _run(["--impl", "reference", "--scene", scene, "--steps", "2", "--warmup", "1"] + extra)
    assert r.returncode == 0, r.stderr[-2000:]
    d = _line(r.stdout)
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    assert d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["config"]["workload"]
    from oracle import refstep
    if refstep.available():  # the reference's own step is compiled here
        assert d["cpu_baseline"]["kind"] == "reference"
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"] and cb["value"] == d["value"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert cb["cpu_model"]
    if scene == "c1":
        assert d["config"]["dt"] == 5e-4 and "dt_note" in d["config"]
    if scene == "c2":
        # the full configuration, not a sample, after the settle steps
        assert d["config"]["same_config"] is True and d["config"]["fluid_particles"] == 1048576
        assert d["config"]["settle_steps"] == 1


def test_gpu_arm_fails_loudly_without_a_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    r = _run(["--scene", "c1", "--steps", "1", "--warmup", "1"], timeout=300)
    assert r.returncode != 0
    assert not [l for l in r.stdout.splitlines() if l.startswith("{") and '"impl": "reference"' not in l]
