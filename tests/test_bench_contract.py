"""The benchmark's reference arm (CPU restatement) prints one JSON line with the contract's keys (small case)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "6", "--p",
                          "2", "--steps", "1", "--warmup", "1"], capture_output=True, text=True, timeout=300,
                         cwd=ROOT, env={**os.environ, "WORLD_SIZE": "1", "RANK": "0"})
    assert out.returncode == 0, out.stderr
    d = json.loads(out.stdout.strip().splitlines()[-1])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is False
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and "workload" in d["config"]


def test_other_workloads_reference_arm_is_explicit():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "xdg48"], capture_output=True, text=True, timeout=120, cwd=ROOT)
    assert out.returncode == 0
    d = json.loads(out.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference" and "unavailable" in d


def test_learned_training_solve_count():
    """The learned variant collects 200 training residuals: enough seeded solves of the fast form's iteration
    count, at least 2 and at most 25."""
    sys.path.insert(0, ROOT)
    import bench
    assert bench.learned_rhs_count(9) == 24 and bench.learned_rhs_count(41) == 6
    assert bench.learned_rhs_count(1) == 25 and bench.learned_rhs_count(500) == 2
    for it in (1, 5, 9, 17, 41, 120):
        n = bench.learned_rhs_count(it)
        assert n * it >= 200 or n == 25
