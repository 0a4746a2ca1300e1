"""The CPU reference arm of bench.py (`--impl reference`): the oracle's FP64 stage on the
host cores, printed as one JSON line with the GPU arm's metric and unit.  Runs on the CPU
on a small box; rank 0 alone measures under torchrun, the other ranks exit 0 silently."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CMD = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--nex", "2", "--p", "3",
       "--steps", "2", "--warmup", "3"]


def _run(env_extra):
    env = dict(os.environ)
    env.update(env_extra)
    return subprocess.run(CMD, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)


def test_reference_arm_line():
    r = _run({"RANK": "0"})
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "DOF-RK-stages/s FP64 at p=8" and d["unit"] == "DOF-RK-stages/s"
    assert d["higher_is_better"] is True and d["steps"] == 2 and d["warmup"] == 3
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["config"]["unknowns"] == 5 * 8 * 4 ** 3
    assert d["config"]["workload"] == "taylor-green 2^3 hex p=3, Re=1600, Mach 0.1, 5-stage LSRK"


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"RANK": "1"})
    assert r.returncode == 0, r.stderr
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
