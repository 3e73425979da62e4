"""The bench's reference arm on the CPU: `bench.py --impl reference` runs the reference's own CPU pair loop
(oracle/_ref, built from the reference's sources) and prints one JSON line with the keys the bench contract
asks for -- the same metric, unit and workload description as the GPU arm, its CPU baseline and an e2e block
with no host-device copies.  A small workload keeps the run to seconds."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libkiwi_ref.so")):
        pytest.skip("oracle/_ref is not built (it needs the reference checkout)")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1",
                        "--n", "20000", "--res", "64"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference"
    assert line["metric"] == "particle-cell integrals/s (support pairs), sph-to-grid"
    assert line["unit"] == "pair-integrals/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert "workload" in line["config"]


def test_reference_arm_loads_nothing_of_the_engine():
    """The reference arm runs the reference's own code only: after `bench.py --impl reference` the process
    has not imported kiwi_b200 and has not mapped libkiwi_b200.so."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libkiwi_ref.so")):
        pytest.skip("oracle/_ref is not built (it needs the reference checkout)")
    code = (
        "import runpy, sys\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '1', '--n', '20000', "
        "'--res', '64']\n"
        "try:\n"
        "    runpy.run_path('bench.py', run_name='__main__')\n"
        "except SystemExit:\n"
        "    pass\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('ENGINE_IMPORTED' if any(m.startswith('kiwi_b200') for m in sys.modules) else 'NO_ENGINE_IMPORT')\n"
        "print('ENGINE_MAPPED' if 'libkiwi_b200' in maps else 'NO_ENGINE_MAPPED')\n"
        "print('REF_MAPPED' if 'libkiwi_ref' in maps else 'NO_REF_MAPPED')\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    tail = r.stdout.strip().splitlines()[-3:]
    assert tail == ["NO_ENGINE_IMPORT", "NO_ENGINE_MAPPED", "REF_MAPPED"], tail
