"""bench.py's reference arm on the host cores (no GPU needed).

The arm times the oracle port of the reference's kernels on one 800x800 view
per step and prints the contract line; it must never map the product library
(libdiffsoup_b200.so), and under torchrun only rank 0 runs it.
"""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RUN = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '1']; "
       "runpy.run_path('bench.py', run_name='__main__'); "
       "print('PRODUCT_LIBRARY_MAPPED', 'libdiffsoup_b200' in open('/proc/self/maps').read())")


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, "-c", RUN], cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=900)


def test_reference_arm_prints_the_contract_line_without_the_product_library():
    out = _run({"RANK": "0"})
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference"
    assert line["unit"] == "views/s" and line["higher_is_better"] is True
    assert line["steps"] == 1 and line["warmup"] == 1
    assert line["value"] > 0 and line["n_gpus"] == 1
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "views/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["views_per_step"] == 8 and line["config"]["triangles"] == 15000
    assert "PRODUCT_LIBRARY_MAPPED False" in out.stdout


def test_reference_arm_other_ranks_exit_without_work():
    out = _run({"RANK": "1"})
    assert out.returncode == 0, out.stderr[-2000:]
    assert not [x for x in out.stdout.splitlines() if x.startswith("{")]
