"""bench.py --impl reference on CPU, on a small grid: it prints one JSON line
with the same configuration as this build's arm, times the host restatement
fed by the host build of the generator, and never maps the CUDA library."""
import json
import os
import subprocess
import sys

from conftest import REPO

PROBE = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--grid", "120", "80", "30", "--steps", "2", "--warmup", "1",
            "--band-rows", "20"]
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
print("MAPPED " + " ".join(sorted({ln.split()[-1] for ln in maps.splitlines() if ln.endswith(".so")})))
"""


def test_reference_arm_runs_without_the_product_library():
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=REPO, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    line = json.loads(lines[0])
    mapped = lines[-1].split()[1:]
    assert not any("liblicom_tracer" in m for m in mapped), mapped
    assert any(m.endswith("oracle/liblicom_oracle.so") for m in mapped)
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 1
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["one_thread"]["value"] > 0
    assert cb["full_grid"]["steps"] == 2 and cb["full_grid"]["value"] > 0
    # the configuration is the one this build's arm reports
    sys.path.insert(0, REPO)
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_cfg", os.path.join(REPO, "bench.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)

    class A:
        grid = [120, 80, 30]
        hypsometry = 0
    assert line["config"] == b.config_of(A, 1)
    assert line["ms_per_step"] * line["steps"] < 60e3
