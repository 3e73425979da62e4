"""CPU-side checks of the C ABI: libkiwi_b200.so loads, exports every entry point include/kiwi_b200.h
declares, and without a GPU every compute entry fails loudly (KIWI_ERR_NODEV) -- there is no CPU fallback."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "kiwi_b200.h")
LIB = os.path.join(ROOT, "kiwi_b200", "libkiwi_b200.so")


def declared_functions():
    text = open(HDR).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(kiwi_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("kiwi_ctx_create", "kiwi_sph_to_grid", "kiwi_face_integral_batch", "kiwi_full_integral_batch",
              "kiwi_map_voronoi", "kiwi_sph_to_grid_device"):
        assert n in names


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build it with python -m kiwi_b200.build"
    lib = C.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_kernel_lookup_without_gpu():
    lib = C.CDLL(LIB)
    lib.kiwi_kernel_index.argtypes = [C.c_char_p]
    assert lib.kiwi_kernel_index(b"cubic_spline") == 0
    assert lib.kiwi_kernel_index(b"Wendland-C4") == 4
    assert lib.kiwi_kernel_index(b"quintic") == 2
    assert lib.kiwi_kernel_index(b"gaussian") == -1


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU failure path")
def test_no_cpu_fallback_without_gpu():
    import kiwi_b200
    with pytest.raises(kiwi_b200.KiwiError) as e:
        kiwi_b200.Context(0)
    assert e.value.code == -3
