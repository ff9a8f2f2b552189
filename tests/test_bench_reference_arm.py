"""The reference arm of bench.py (`--impl reference`): the CPU restatement of
the reference's step on the host cores, printed as one JSON line with the
same metric, unit and config as the GPU arm.  Runs on CPU only, on a small
box so that it takes seconds."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.timeout(300)
def test_reference_arm_line():
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--box", "16", "--steps", "2",
                        "--warmup", "4"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=280)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["steps"] == 2 and d["warmup"] == 4
    assert d["unit"] == "MLUPS" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["box"] == [16, 16, 16] and d["config"]["storage"] == "f32"


@pytest.mark.timeout(300)
def test_reference_arm_does_not_load_the_product_library():
    """The reference arm sets its box up with the oracle's own helpers: the
    process never maps liblbfast_b200.so."""
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    code = ("import sys; sys.argv = ['bench.py', '--impl', 'reference', '--box', '16', '--steps', '1', "
            "'--warmup', '3']; import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); print('MAPPED' if 'liblbfast_b200' in maps else 'CLEAN')")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=280)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "CLEAN"
