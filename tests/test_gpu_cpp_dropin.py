"""The C++ drop-in on the GPU.

* The reference's own kernel-integral regression test (tools/test_generic_kernel.cpp of the reference:
  normalisation, the generic series against the hand-written cubic form and against brute-force quadrature,
  continuity across kernel regions, box masses from the face walk, partitions of boxes), compiled unchanged
  against kiwi_b200's headers (include/kiwi/) and linked with libkiwi_b200.so by oracle/Makefile into
  oracle/_ref/test_generic_kernel_b200: every integral it checks is evaluated by the GPU.
* The sph-to-grid stage as a KIWI maintainer replaces its particle loop (tests/cpp/sph_to_grid_stage.cpp,
  INTEGRATION.md's code): its cartesian_grid.dat has the reference's header byte for byte and the reference's
  values (tests/golden/grid_cubic_cube.npz, from the reference library) within the reference's own error
  envelope.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

from gpu_checks import assert_within_envelope, velocity_errors

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "test_generic_kernel_b200")


@pytest.mark.parametrize("npts", [40, 400])
def test_reference_kernel_regression_test_on_gpu(npts):
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/test_generic_kernel_b200 not built (make -C oracle REF=<KIWI checkout>)")
    r = subprocess.run([BIN, str(npts)], capture_output=True, text=True, timeout=900)
    print(r.stdout[-4000:])
    assert r.returncode == 0 and "FAIL" not in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]


def _read_grid(path):
    with open(path, "rb") as f:
        raw = f.read()
    nx, ny, nz = struct.unpack("<3i", raw[8:20])
    n = nx * ny * nz
    arr = np.frombuffer(raw[68:], dtype="<f8")
    assert arr.size == 4 * n
    return raw[:68], arr.reshape(4, n)


def test_stage_harness_writes_the_reference_file(tmp_path, reflib):
    exe = tmp_path / "sph_to_grid_stage"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-o", str(exe),
                    os.path.join(ROOT, "tests", "cpp", "sph_to_grid_stage.cpp"), "-L", os.path.join(ROOT, "kiwi_b200"),
                    "-lkiwi_b200", "-Wl,-rpath," + os.path.join(ROOT, "kiwi_b200")], check=True)
    d = np.load(os.path.join(ROOT, "tests", "golden", "grid_cubic_cube.npz"))
    snap = tmp_path / "snap.txt"
    cols = [d[k] for k in ("x", "y", "z", "vx", "vy", "vz", "m", "h")]
    np.savetxt(snap, np.column_stack(cols + [np.ones_like(cols[0])]), fmt="%.17g")
    b, s = d["bounds"], d["shape"]
    ours = tmp_path / "cartesian_grid.dat"
    subprocess.run([str(exe), str(snap), str(ours), *[repr(float(v)) for v in b], *[str(int(v)) for v in s]], check=True)
    theirs = tmp_path / "reference_grid.dat"
    reflib.save_cartesian_grid(str(theirs), s, b, d["out_density"], d["out_vx"], d["out_vy"], d["out_vz"])
    h_ours, a_ours = _read_grid(ours)
    h_ref, a_ref = _read_grid(theirs)
    assert h_ours == h_ref
    # against the exact integral, within 4x the reference's own error per band (as the fixture tests judge)
    tr = d["truth_raw"]
    vol = np.prod([(b[2 * i + 1] - b[2 * i]) / s[i] for i in range(3)])
    assert_within_envelope(a_ours[0], a_ref[0], tr[0] / vol, label="cartesian_grid.dat")
    with np.errstate(invalid="ignore", divide="ignore"):
        for i in range(3):
            tv = np.where(tr[0] > 0, tr[i + 1] / np.where(tr[0] > 0, tr[0], 1.0), 0.0)
            assert velocity_errors(a_ours[i + 1], tv, tr[0]) <= 4.0 * velocity_errors(a_ref[i + 1], tv, tr[0]) + 1e-13
