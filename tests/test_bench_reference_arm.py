"""The benchmark's CPU reference arm on the host: the sampled estimate of one plain-arm POLFED
solve by the CPU restatement (oracle/), on the C2 workload with a shortened recurrence so the
test takes seconds.  Checks that every part of the estimate is measured (positive, finite),
that the parts add up, that the sampled operands are made once and reused by later samples,
and that `--impl reference` prints one JSON line with the contract's keys."""
import json
import math
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    sys.path.insert(0, ROOT)
    import bench

    return bench


def test_cpu_estimate_parts_and_reuse():
    bench = _bench()
    wl = bench.Workload("c2")
    wl.cpu_steps = 8
    bench._CPU_INPUTS.pop("c2", None)
    est = bench.cpu_plain_estimate(wl, 2)
    for k in ("seconds", "filter_s", "block_dense_s", "extract_s"):
        assert math.isfinite(est[k]) and est[k] > 0, (k, est)
    assert est["seconds"] == pytest.approx(est["filter_s"] + est["block_dense_s"] + est["extract_s"])
    inp = bench._CPU_INPUTS["c2"]
    assert inp["D"] == 8 and inp["Q"].shape == (wl.A.shape[0], wl.s)
    assert inp["V"].shape == (wl.A.shape[0], wl.s * wl.mmax // 2)
    bench.cpu_plain_estimate(wl, 2)
    assert bench._CPU_INPUTS["c2"] is inp  # made once, reused


@pytest.mark.timeout(600)
def test_reference_arm_prints_one_line():
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--workload", "c2", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, cwd=ROOT, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "eigenpairs/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["higher_is_better"] is True and d["steps"] == 1
