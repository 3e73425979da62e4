#!/usr/bin/env python3
"""Extract the reference's kernel coefficient tables into ``kernel_spec_ref.json`` (a test fixture).

Reads ``src/kernel_spec_data.cpp`` of a KIWI checkout (first argument, or KIWI_REF) as text and collects
the numbers of each KernelSpec initializer in declaration order: key, name, nreg, c[4], A2_pi, A3_pi,
radkern, hfact, a[4][15], B[4][4][16].  Run once where the reference is present; the JSON it writes
is committed so that the tests never need the reference itself.
"""
import json
import os
import re
import sys

ROOT = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("KIWI_REF")
if not ROOT:
    sys.exit("usage: make_kernel_spec_fixture.py <KIWI checkout>  (or set KIWI_REF)")
src = open(os.path.join(ROOT, "src", "kernel_spec_data.cpp")).read()
body = src[src.index("kKernels[] = {"):src.index("} // namespace")]
body = re.sub(r"//[^\n]*", "", body)
out = []
for block in re.findall(r"\{\s*\"(\w+)\",\s*\"([^\"]+)\",(.*?)\n    \}", body, re.S):
    key, name, rest = block
    nums = [float(x) for x in re.findall(r"-?\d+(?:\.\d*)?(?:e-?\d+)?", rest)]
    nreg = int(nums[0])
    c = nums[1:5]
    A2_pi, A3_pi, radkern, hfact = nums[5:9]
    a = [nums[9 + 15 * k: 9 + 15 * (k + 1)] for k in range(4)]
    b0 = 9 + 60
    B = [[nums[b0 + 64 * j + 16 * k: b0 + 64 * j + 16 * (k + 1)] for k in range(4)] for j in range(4)]
    assert len(nums) == b0 + 256, (key, len(nums))
    out.append({"key": key, "name": name, "nreg": nreg, "c": c, "A2_pi": A2_pi, "A3_pi": A3_pi,
                "radkern": radkern, "hfact": hfact, "a": a, "B": B})
here = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(here, "kernel_spec_ref.json"), "w") as f:
    json.dump(out, f)
print("wrote", len(out), "kernels")
