"""The kernel coefficient tables (derived here in exact arithmetic) against the reference's values."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GEN = os.path.join(ROOT, "kiwi_b200", "tables", "gen_kernel_tables.py")


def test_header_up_to_date():
    r = subprocess.run([sys.executable, GEN, "--check"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


def test_tables_equal_reference_values():
    ref = json.load(open(os.path.join(ROOT, "tests", "golden", "kernel_spec_ref.json")))
    mine = json.loads(subprocess.check_output([sys.executable, GEN, "--json"]))
    assert [k["key"] for k in mine] == ["M4", "M5", "M6", "WC2", "WC4", "WC6"]
    for r, m in zip(ref, mine):
        for field in ("key", "name", "nreg", "c", "A2_pi", "A3_pi", "radkern", "hfact", "a", "B"):
            assert r[field] == m[field], (r["key"], field)
