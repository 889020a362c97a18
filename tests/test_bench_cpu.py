"""bench.py's reference arm on the CPU: it times the reference's own CPU entry
(oracle/_ref, compiled from the reference sources) on a whole burst built on
the host, maps no library of the product (only oracle/ ones), prints one JSON
line whose config equals the one the GPU arm prints, and counts the burst's
terms with the oracle."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WRAP = r"""
import runpy, sys, atexit
root = sys.argv[1]
def maps():
    libs = sorted({l.split()[-1] for l in open('/proc/self/maps') if '.so' in l and root in l})
    print('MAPPED ' + ' '.join(libs), file=sys.stderr)
atexit.register(maps)
sys.argv = [root + '/bench.py'] + sys.argv[2:]
runpy.run_path(root + '/bench.py', run_name='__main__')
"""


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_cpu.so")),
                    reason="the reference CPU code is not compiled here")
def test_reference_arm_runs_whole_bursts_without_the_product_library():
    p = subprocess.run([sys.executable, "-c", WRAP, ROOT, "--impl", "reference", "--workload", "c1",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                       timeout=900, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench
    assert d["impl"] == "reference" and d["config"] == bench.workload_config("c1", 1)
    assert d["value"] > 0 and d["ms_per_step"] > 0 and d["cpu_baseline"]["kind"] == "reference"
    assert "552389028 terms" in d["cpu_baseline"]["sample"]      # the burst's exact term count
    mapped = [ln for ln in p.stderr.splitlines() if ln.startswith("MAPPED")][-1].split()[1:]
    assert mapped and all("/oracle/" in m for m in mapped), mapped
    assert not any("srg_b200" in m for m in mapped)
