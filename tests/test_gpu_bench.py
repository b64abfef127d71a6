"""bench.py on a small plain search, end to end on the GPU: one JSON line with
the contract's keys, every hit rechecked, the B = 64 sections of both walks,
the roofline's ALU and IMAD-class fractions, and the end-to-end rate through
the C ABI."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_line_on_a_small_search():
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--total-keys", "2e9",
                        "--steps", "2", "--warmup", "3", "--no-cpu-baseline", "--no-cpu-search", "--no-ref-cuda",
                        "--no-batched", "--served-seconds", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "dtype", "config", "e2e", "roofline", "clocks", "gpu_launches", "ranks"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == 2 and d["gpu_launches"] == 2 and d["value"] > 1e9
    assert d["hits"]["rechecked"] == d["hits"]["found"] and d["hits"]["rechecked_bad"] == 0
    assert d["e2e"]["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] > 0
    r = d["roofline"]
    assert r["bound"] == "alu" and 0 < r["frac"] < 1.2 and 0 < r["imad_ncu"]["frac"] < 1.2
    for key, walk in (("at_batch_64", "group"), ("xadd_b64", "xadd")):
        s = d[key]
        assert s["config"]["walk"] == walk and s["config"]["batch"] == 64 and s["value"] > 1e9
        assert s["hits"]["rechecked_bad"] == 0 and "imad_ncu" in s["roofline"]
