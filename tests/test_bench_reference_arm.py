"""bench.py's reference arm on CPU: one whole oracle step of the bubble
column on a 16^3 grid prints one JSON line with the contract's keys, and the
process never loads the product library (the arm runs the oracle only, with
scene inputs from the oracle's own build)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--n", "16", "--steps", "1", "--warmup", "0"]
import bench
bench.run_reference(bench.parse(), 0)
libs = sorted({l.split()[-1] for l in open("/proc/self/maps") if l.rstrip().endswith(".so")})
print(json.dumps({"libs": libs}))
"""


def test_reference_arm_line_and_libraries():
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    line, libs = json.loads(lines[0]), json.loads(lines[-1])["libs"]
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["config"]["grid"] == 16 and line["config"]["particles"] > 0
    assert not [l for l in libs if os.path.basename(l) == "libmp.so"], libs
    assert [l for l in libs if "oracle" in l], libs


def test_cpu_baseline_reports_all_threads_and_one_thread():
    """The GPU arm's cpu_baseline: a whole oracle step on all host threads and
    one on a single thread at the smaller of the two grids."""
    import sys
    sys.path.insert(0, ROOT)
    import bench
    cb = bench.cpu_baseline(5, 16, 2017005, single_n=12)
    assert cb["value"] > 0 and cb["cores"] >= 1 and cb["kind"] == "port" and "16^3" in cb["sample"]
    st = cb["single_thread"]
    assert st["value"] > 0 and st["cores"] == 1 and "12^3" in st["sample"]
