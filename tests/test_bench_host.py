"""The benchmark's reference arm, on the host: it must run the reference's
own CPU path without the product library (its inputs come from the oracle's
restated generators), and print the same workload config as the library's
arm, so the two lines compare like for like."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_PROBE = r"""
import io, json, sys, contextlib
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"]
sys.path.insert(0, %r)
import bench
out = io.StringIO()
with contextlib.redirect_stdout(out):
    bench.main()
maps = open("/proc/self/maps").read()
print(json.dumps({"line": out.getvalue().strip().splitlines()[-1],
                  "daspmm": "libdaspmm.so" in maps,
                  "oracle": "liboracle.so" in maps,
                  "torch": "torch" in sys.modules,
                  "config": bench.bench_config(bench.NR, 1242101, 1)}))
"""


def test_reference_arm_loads_no_product_library():
    r = subprocess.run([sys.executable, "-c", _PROBE % ROOT], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    line = json.loads(res["line"])
    assert not res["daspmm"], "the reference arm mapped libdaspmm.so"
    assert res["oracle"] and not res["torch"]
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"] == res["config"], "the arms' configs differ"
    assert line["config"]["nnz"] == 1242101
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["cores"] >= 1
