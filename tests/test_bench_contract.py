"""The benchmark's output contract, checked on the CPU: the reference arm
(the reference's algorithm, restated by the oracle, on the host cores) prints
one JSON line with the metric, its unit, the CPU-baseline description and an
end-to-end block; the serving workload has no reference arm and says so."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


def test_reference_arm_line():
    """One line with the all-core, single-thread and reference-Jacobian
    samples; the arm builds its meshes with the oracle alone, so neither the
    library's Python package nor its shared object is ever loaded."""
    probe = ("import json, runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', "
             "'--warmup', '0']; runpy.run_path('bench.py', run_name='__main__'); "
             "maps = open('/proc/self/maps').read(); "
             "print(json.dumps({'package': 'cpolyg_b200' in sys.modules, 'so': 'libcpolyg_b200' in maps}))")
    r = subprocess.run([sys.executable, "-c", probe], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 2 and lines[1] == {"package": False, "so": False}, r.stdout
    d = lines[0]
    assert d["impl"] == "reference" and d["unit"] == "steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["n_gpus"] == 1 and d["steps"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert cb["value_1thread"] > 0 and "1 thread" in cb["sample_1thread"]
    assert cb["value_reference_jacobian"] > 0
    assert d["e2e"] == {"value": d["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["cells"] == 100000 and d["config"]["block"] == 40 and d["config"]["tableau"] == "sdirk3"


def test_serving_workload_has_no_reference_arm():
    d = run_bench("--impl", "reference", "--workload", "serve")
    assert d["impl"] == "reference" and "unavailable" in d
