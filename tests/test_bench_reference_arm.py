"""bench.py --impl reference prints one contract line (CPU only): the reference's own Numba path when
bempp_cl is installed under baseline/_ref, else the oracle port, on the host cores."""

import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_one_json_line():
    env = dict(os.environ, OMP_NUM_THREADS="2", NUMBA_NUM_THREADS="2")
    proc = subprocess.run(
        [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--level", "3", "--steps", "1",
         "--warmup", "1", "--cpu-seconds", "0.2"],
        capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert proc.returncode == 0, proc.stderr[-2000:]
    lines = [l for l in proc.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    from oracle import reference

    expect = "reference" if reference.load() is not None else "port"
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == expect
    sys.path.insert(0, ROOT)
    import bench

    assert line["config"] == json.loads(json.dumps(bench.bench_config(bench.parse(["--level", "3"]))))
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
