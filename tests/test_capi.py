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


# The C++ drop-in of the reference's kernel-integral layer (include/kiwi/*.hpp): its functions, by the
# reference's names and signatures (include/kiwi/kernel_integral.hpp:42-193, kernel_integral_generic.hpp:27-56,
# kernel_spec.hpp:41-44 of the reference).
CPP_SYMBOLS = (
    "kiwi::get_kernel(std::__cxx11::basic_string<char, std::char_traits<char>, std::allocator<char> > const&)",
    "kiwi::all_kernels()",
    "kiwi::full_integral_new(double, double, double, double)",
    "kiwi::compute_wall_constants(double, double)",
    "kiwi::compute_edge_constants(kiwi::WallIntegralConstants const&, double)",
    "kiwi::vertex_integral(kiwi::WallIntegralConstants const&, kiwi::EdgeIntegralConstants const&, double)",
    "kiwi::compute_face_integral(double, double, double, double, bool, kiwi::DensityLookupTable const*, "
    "std::vector<double, std::allocator<double> > const&, int*)",
    "kiwi::compute_face_integral_generic(double, double, double, kiwi::KernelSpec const&, double, "
    "std::vector<double, std::allocator<double> > const&, int*)",
    "kiwi::generic_wall_constants(kiwi::KernelSpec const&, double, double)",
    "kiwi::generic_edge_constants(kiwi::GenericWallConstants const&, double)",
    "kiwi::generic_vertex_integral(kiwi::GenericWallConstants const&, kiwi::GenericEdgeConstants const&, double)",
    "kiwi::generic_full_integral(kiwi::KernelSpec const&, double, double, double, double)",
    "kiwi::gridded_integral(kiwi::DensityLookupTable const&, double, double, double, double)",
    "kiwi::load_density_table(std::__cxx11::basic_string<char, std::char_traits<char>, std::allocator<char> > const&)",
    "kiwi::generate_density_table()",
    "kiwi::DensityLookupTable::at(int, int, int) const",
)


def test_library_exports_cpp_dropin():
    import subprocess

    out = subprocess.run(["nm", "-D", "--defined-only", "-C", LIB], capture_output=True, text=True, check=True).stdout
    have = {ln.split(" ", 2)[2] for ln in out.splitlines() if ln.count(" ") >= 2}
    missing = [s for s in CPP_SYMBOLS if s not in have]
    assert not missing, missing


def test_cpp_dropin_headers_compile(tmp_path):
    """A translation unit written against the reference's API (every header, the integrator template with a
    configuration type that has the reference's Config accessors) compiles and links against the library."""
    import subprocess

    src = tmp_path / "use.cpp"
    src.write_text('''
#include "kiwi/kernel_integrator.hpp"
struct Cfg {
    double kernel_support_in_h() const { return 3.0; }
    bool use_generic_kernel_path() const { return true; }
    const kiwi::KernelSpec& kernel_spec() const { return kiwi::get_kernel("quintic_spline"); }
};
int main() {
    kiwi::KernelIntegrator ki = kiwi::make_kernel_integrator(Cfg{}, false, nullptr);
    std::vector<double> f{1, 0, 1, 1, 1, 1, 1, 1, 0, 1, 0, 0};
    return ki.support(2.0) == 6.0 && ki.generic == &kiwi::get_kernel("M6") ? 0 : (int)ki.face(0, 0, 0, 1, f);
}
''')
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-o", str(tmp_path / "use"), str(src),
                    "-L", os.path.join(ROOT, "kiwi_b200"), "-lkiwi_b200"], check=True)


def test_header_is_plain_c_and_links(tmp_path):
    """include/kiwi_b200.h compiles as strict C99 and a plain C program links against the library and calls
    its host-only entry points (kernel lookup, the split of one grid over parts) without a GPU."""
    import subprocess

    src = tmp_path / "use.c"
    src.write_text(r'''
#include <stdio.h>
#include "kiwi_b200.h"
int main(void) {
    double x[2] = {0.5, 1.5}, y[2] = {0.5, 1.5}, z[2] = {0.5, 1.5}, v[2] = {0, 0}, m[2] = {1, 1}, h[2] = {0.2, 0.2};
    KiwiParticles p = {2, x, y, z, v, v, v, m, h};
    KiwiCartGrid g = {{0.0, 2.0, 0.0, 2.0, 0.0, 2.0}, 32, 16, 16};
    KiwiKernelSel k = {0, 0.0, 0, 0};
    int a0 = -1, a1 = -1, b0 = -1, b1 = -1;
    if (kiwi_kernel_index("cubic_spline") != 0) return 1;
    if (kiwi_part_rows(NULL, &p, &g, &k, 0, 2, &a0, &a1) != 0) return 2;
    if (kiwi_part_rows(NULL, &p, &g, &k, 1, 2, &b0, &b1) != 0) return 3;
    printf("%d %d %d %d\n", a0, a1, b0, b1);
    return 0;
}
''')
    exe = tmp_path / "use"
    libdir = os.path.dirname(LIB)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"), str(src),
                    "-o", str(exe), "-L", libdir, "-lkiwi_b200", "-Wl,-rpath," + libdir], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out
    a0, a1, b0, b1 = (int(t) for t in out.stdout.split())
    # two particles touching tiles 0, 4 and 11, 15 of the 4 x 2 x 2 tiles: part 0 owns tiles 0-4 (x rows
    # 0-15), part 1 tiles 5-15 (x rows 8-31)
    assert (a0, a1) == (0, 16) and (b0, b1) == (8, 32)
