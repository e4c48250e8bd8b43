"""CPU checks of bench.py's host logic: the reference arm's rotating sample
(including a sample as large as the workload) and its JSON line."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_next_offset_stays_inside_the_workload():
    from bench import next_offset
    for n in (1, 7, 300, 1 << 20):
        for m in (1, 3, n - 1, n, n + 5):
            if m <= 0:
                continue
            off = 0
            for _ in range(50):
                off = next_offset(off, m, n)
                assert 0 <= off and off + min(m, n) <= n, (n, m, off)


def test_reference_arm_with_a_sample_of_the_whole_workload():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref (the compiled reference) is not built here")
    # 300 points: the sample is clamped to the whole workload (m == n)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--points", "300", "--steps", "2", "--warmup", "1"],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"]["points_per_step"] == 300
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["cores"] >= 1
