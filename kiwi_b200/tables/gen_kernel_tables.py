#!/usr/bin/env python3
"""Exact-rational derivation of the vertex-pyramid coefficient tables for the six SPH kernels.

Writes ``kiwi_b200/csrc/kernel_tables.h`` (shared by the CUDA kernels and by the CPU oracle).

Kernel convention (Petkova 2018 thesis, appendix A; restated by the reference in
``tools/kernel_tables/kernels.py:1-101``): W(r) = A3 / H^3 * w(q), q = r / H, support radius H,
w = 0 for q >= 1.  The q axis is split at breakpoints c_1 < ... < c_n = 1 into n pieces, numbered
1..n, and q > 1 is region n + 1.

Derivation (the method of ``tools/kernel_tables/derive.py:19-63``, written out here from the maths):

* enclosed-mass shape  m_k(rho) = int_0^rho w(s) s^2 ds  on piece k (continuous across pieces);
* F_k(rho) = int m_k(rho) / rho^2 drho   (a Laurent polynomial without constant term);
* the kernel mass of the vertex pyramid has dI_P/dphi = A3 * r0 * [F_k(r) - F_j(r0) + C_jk],
  r = vertex radius (region k), r0 = wall distance (region j <= k), C_jk the continuity constant
  that joins the pieces crossed between r0 and r.  With mu = r0 / r and q0 = r0 (H = 1) a term
  f_p rho^p of F_k becomes f_p q0^(1-i) mu^i with i = -p, so
    a[k][1 - i] = f_{-i}  (i <= 1, i != 0),
    B[j][k](q0) = -q0 F_j(q0) + q0 * C_jk,
    C_jk = F_j(c_j) + sum_{l=j+1}^{k-1} (F_l(c_l) - F_l(c_{l-1})) - F_k(c_{k-1})   (k > j), 0 if k == j.

Usage:  python gen_kernel_tables.py            (write the header)
        python gen_kernel_tables.py --check    (exit 1 if the committed header is stale)
        python gen_kernel_tables.py --json     (print the tables as JSON, for tests)
"""
from __future__ import annotations

import json
import os
import sys
from fractions import Fraction as Q

MAX_REGIONS = 4   # pieces + 1 (quartic and quintic splines have 3 pieces)
NI = 15           # basis integrals I_i for i = 1, 0, -1, ..., -13, stored at index 1 - i
NB = 16           # powers q0^0 .. q0^15 in the B polynomials

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.normpath(os.path.join(HERE, "..", "csrc", "kernel_tables.h"))


class Laurent:
    """Sparse Laurent polynomial with exact rational coefficients: {power: Fraction}."""

    __slots__ = ("c",)

    def __init__(self, c=None):
        self.c = {p: Q(v) for p, v in (c or {}).items() if v != 0}

    def __add__(self, o):
        r = dict(self.c)
        for p, v in o.c.items():
            r[p] = r.get(p, Q(0)) + v
        return Laurent(r)

    def __neg__(self):
        return Laurent({p: -v for p, v in self.c.items()})

    def __sub__(self, o):
        return self + (-o)

    def __mul__(self, o):
        if not isinstance(o, Laurent):
            return Laurent({p: v * o for p, v in self.c.items()})
        r = {}
        for p, v in self.c.items():
            for q, w in o.c.items():
                r[p + q] = r.get(p + q, Q(0)) + v * w
        return Laurent(r)

    __rmul__ = __mul__

    def __pow__(self, n):
        r = Laurent({0: 1})
        for _ in range(n):
            r = r * self
        return r

    def antiderivative(self):
        r = {}
        for p, v in self.c.items():
            if p == -1:
                raise ValueError("1/x term: the antiderivative would need a logarithm")
            r[p + 1] = v / (p + 1)
        return Laurent(r)

    def at(self, x):
        x = Q(x)
        return sum((v * x ** p for p, v in self.c.items()), Q(0))


X = Laurent({1: 1})
ONE = Laurent({0: 1})


class KernelDef:
    """A kernel given either as a truncated-power B-spline sum  sum coef * (shift - q)_+^deg  or as a
    Wendland function (1 - q)_+^deg * poly(q)."""

    def __init__(self, key, name, radkern, hfact, spline=None, wendland=None):
        self.key, self.name, self.radkern, self.hfact = key, name, radkern, hfact
        self.spline, self.wendland = spline, wendland
        if spline:
            self.breaks = sorted({Q(s) for _, s, _ in spline})
        else:
            self.breaks = [Q(1)]

    def piece_polys(self):
        """Polynomial of w on each piece (c_{k-1}, c_k], k = 1..n."""
        out = []
        for hi in self.breaks:
            if self.spline:
                w = Laurent()
                for coef, shift, deg in self.spline:
                    if Q(shift) >= hi:          # (shift - q)_+ is active on this whole piece
                        w = w + Q(coef) * (Laurent({0: Q(shift)}) - X) ** deg
            else:
                deg, poly = self.wendland
                w = (ONE - X) ** deg * Laurent(poly)
            out.append(w)
        return out

    def a3_times_pi(self):
        """A3 * pi, with A3 chosen so that 4 pi int_0^1 A3 w q^2 dq = 1."""
        tot = Q(0)
        lo = Q(0)
        for hi, w in zip(self.breaks, self.piece_polys()):
            P = (w * X ** 2).antiderivative()
            tot += P.at(hi) - P.at(lo)
            lo = hi
        return 1 / (4 * tot)

    def a2_times_pi(self):
        """A2 * pi, with A2 chosen so that 2 pi int_0^1 A2 w q dq = 1 (the 2D normalisation)."""
        tot = Q(0)
        lo = Q(0)
        for hi, w in zip(self.breaks, self.piece_polys()):
            P = (w * X).antiderivative()
            tot += P.at(hi) - P.at(lo)
            lo = hi
        return 1 / (2 * tot)

    def enclosed_mass_polys(self):
        """m_k(rho) = int_0^rho w s^2 ds on each region k = 1..n+1 (region n+1: the constant total)."""
        out = []
        lo, carried = Q(0), Q(0)
        for hi, w in zip(self.breaks, self.piece_polys()):
            P = (w * X ** 2).antiderivative()
            m = P + Laurent({0: carried - P.at(lo)})
            out.append(m)
            carried = m.at(hi)
            lo = hi
        out.append(Laurent({0: carried}))
        return out

    def pyramid_tables(self):
        """(a, B): a[k] = {i: coef} for k = 1..n+1, B[(j, k)] = {power: coef} for j <= k."""
        ms = self.enclosed_mass_polys()
        nreg = len(ms)
        cs = [Q(0)] + list(self.breaks)
        F = [(m * Laurent({-2: 1})).antiderivative() for m in ms]
        a = {k: {-p: v for p, v in F[k - 1].c.items()} for k in range(1, nreg + 1)}
        B = {}
        for j in range(1, nreg + 1):
            for k in range(j, nreg + 1):
                poly = -(X * F[j - 1])
                if k > j:
                    C = F[j - 1].at(cs[j]) if j < nreg else Q(0)
                    for l in range(j + 1, k):
                        C += F[l - 1].at(cs[l]) - F[l - 1].at(cs[l - 1])
                    C -= F[k - 1].at(cs[k - 1])
                    poly = poly + Laurent({1: C})
                B[(j, k)] = dict(poly.c)
        return a, B


KERNELS = [
    KernelDef("M4", "Cubic spline", 2.0, 1.2, spline=[(1, 1, 3), (-4, Q(1, 2), 3)]),
    KernelDef("M5", "Quartic spline", 2.5, 1.1, spline=[(1, 1, 4), (-5, Q(3, 5), 4), (10, Q(1, 5), 4)]),
    KernelDef("M6", "Quintic spline", 3.0, 1.0, spline=[(1, 1, 5), (-6, Q(2, 3), 5), (15, Q(1, 3), 5)]),
    KernelDef("WC2", "Wendland C2", 2.0, 1.3, wendland=(4, {0: 1, 1: 4})),
    KernelDef("WC4", "Wendland C4", 2.0, 1.5, wendland=(6, {0: 1, 1: 6, 2: Q(35, 3)})),
    KernelDef("WC6", "Wendland C6", 2.0, 1.6, wendland=(8, {0: 1, 1: 8, 2: 25, 3: 32})),
]


def tables():
    """Float tables, laid out exactly as the C header stores them."""
    out = []
    for K in KERNELS:
        a, B = K.pyramid_tables()
        nreg = len(K.breaks) + 1
        assert nreg <= MAX_REGIONS
        arow = [[0.0] * NI for _ in range(MAX_REGIONS)]
        for k, coefs in a.items():
            for i, v in coefs.items():
                assert i != 0 and 0 <= 1 - i < NI, (K.key, i)
                arow[k - 1][1 - i] = float(v)
        Brow = [[[0.0] * NB for _ in range(MAX_REGIONS)] for _ in range(MAX_REGIONS)]
        for (j, k), poly in B.items():
            for p, v in poly.items():
                assert 0 <= p < NB, (K.key, j, k, p)
                Brow[j - 1][k - 1][p] = float(v)
        out.append({
            "key": K.key, "name": K.name, "nreg": nreg,
            "c": [float(c) for c in K.breaks] + [0.0] * (MAX_REGIONS - len(K.breaks)),
            "A2_pi": float(K.a2_times_pi()), "A3_pi": float(K.a3_times_pi()),
            "radkern": K.radkern, "hfact": K.hfact, "a": arow, "B": Brow,
        })
    return out


def _num(x):
    r = repr(float(x))
    return r if ("." in r or "e" in r or "inf" in r or "nan" in r) else r + ".0"


def header_text():
    T = tables()
    L = [
        "// GENERATED by kiwi_b200/tables/gen_kernel_tables.py -- do not edit by hand.",
        "// Vertex-pyramid coefficient tables of the six SPH kernels (M4, M5, M6, WC2, WC4, WC6),",
        "// derived in exact rational arithmetic from the kernel definitions and rounded once to double.",
        "// Layout: a[k][1 - i] multiplies mu^i q0^(1-i) for a vertex in region k (0-based);",
        "//         B[j][k][p] is the coefficient of q0^p for a wall in region j and a vertex in region k.",
        "#pragma once",
        "",
        f"#define KIWI_MAX_REGIONS {MAX_REGIONS}",
        f"#define KIWI_NI {NI}",
        f"#define KIWI_NB {NB}",
        f"#define KIWI_NUM_KERNELS {len(T)}",
        "",
        "typedef struct KiwiKernelTable {",
        "    const char* key;",
        "    const char* name;",
        "    int nreg;                               /* pieces + 1 */",
        "    double c[KIWI_MAX_REGIONS];             /* breakpoints in units of H, c[nreg-2] == 1 */",
        "    double A2_pi, A3_pi;                    /* normalisation constants times pi */",
        "    double radkern;                         /* support radius in units of h */",
        "    double hfact;                           /* default h = hfact * (m/rho)^(1/3) */",
        "    double a[KIWI_MAX_REGIONS][KIWI_NI];",
        "    double B[KIWI_MAX_REGIONS][KIWI_MAX_REGIONS][KIWI_NB];",
        "} KiwiKernelTable;",
        "",
        "#ifndef KIWI_TABLE_QUALIFIER",
        "#define KIWI_TABLE_QUALIFIER static const",
        "#endif",
        "",
        "KIWI_TABLE_QUALIFIER KiwiKernelTable kiwi_kernel_tables[KIWI_NUM_KERNELS] = {",
    ]
    for t in T:
        L.append(f"    {{ /* {t['name']} */")
        L.append(f"        \"{t['key']}\", \"{t['name']}\", {t['nreg']},")
        L.append("        {" + ", ".join(_num(c) for c in t["c"]) + "},")
        L.append(f"        {_num(t['A2_pi'])}, {_num(t['A3_pi'])}, {_num(t['radkern'])}, {_num(t['hfact'])},")
        L.append("        {" + ",\n         ".join("{" + ", ".join(_num(v) for v in row) + "}" for row in t["a"]) + "},")
        jrows = []
        for j in range(MAX_REGIONS):
            jrows.append("{" + ",\n          ".join("{" + ", ".join(_num(v) for v in t["B"][j][k]) + "}"
                                                   for k in range(MAX_REGIONS)) + "}")
        L.append("        {" + ",\n         ".join(jrows) + "}")
        L.append("    },")
    L.append("};")
    L.append("")
    return "\n".join(L)


def main(argv):
    if "--json" in argv:
        print(json.dumps(tables()))
        return 0
    text = header_text()
    if "--check" in argv:
        cur = open(OUT).read() if os.path.exists(OUT) else ""
        if cur != text:
            print(f"{OUT} is stale: rerun gen_kernel_tables.py")
            return 1
        print(f"{OUT} is up to date")
        return 0
    with open(OUT, "w") as f:
        f.write(text)
    print("wrote", OUT)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
