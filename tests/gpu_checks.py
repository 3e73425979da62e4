"""Comparison helpers shared by the GPU parity tests.

Parity of a floating-point FP64 implementation with the reference is judged against the exact
integral: the __float128 oracle (oracle/kiwi_oracle_q.c) evaluates the same algorithm with ~34
significant digits.  The reference's closed forms cancel heavily (terms ~ (h/r0)^3, phi - atan(u/a) at
small R_0/r0, and the signed sum of up to 48 vertex-pyramid terms per cell), so two correct FP64
implementations that differ only in the last bit of a libm call (glibc vs CUDA) can differ by far more
than 1e-12 in a cell; the reference itself is that far from the exact value.  The bar is therefore:
in every density band, the GPU's largest error against the truth is no more than ENVELOPE_FACTOR times
the reference's own largest error there (plus a few ulp).
"""
import numpy as np

ENVELOPE_FACTOR = 4.0
ULP_FLOOR = 4e-15
# density bands, as fractions of the peak of the exact density
BANDS = ((1e-2, np.inf), (1e-4, 1e-2), (1e-6, 1e-4))


def band_max_rel(x, truth, bands=BANDS):
    x, truth = np.asarray(x), np.asarray(truth)
    peak = float(np.max(np.abs(truth)))
    out = []
    for lo, hi in bands:
        m = (np.abs(truth) > lo * peak) & (np.abs(truth) <= hi * peak)
        out.append(float(np.max(np.abs(x[m] - truth[m]) / np.abs(truth[m]))) if m.any() else 0.0)
    low = np.abs(truth) <= bands[-1][0] * peak
    out.append(float(np.max(np.abs(x[low] - truth[low])) / peak) if low.any() and peak > 0 else 0.0)
    return out


def assert_within_envelope(gpu, ref, truth, label="", factor=ENVELOPE_FACTOR, floor=ULP_FLOOR):
    g = band_max_rel(gpu, truth)
    r = band_max_rel(ref, truth)
    for i, (ge, re_) in enumerate(zip(g, r)):
        assert ge <= factor * re_ + floor, f"{label}: band {i}: GPU err {ge:.3e} vs reference err {re_:.3e}"
    return g, r


def velocity_errors(v, truth_v, truth_m, floor=1e-6):
    truth_m = np.asarray(truth_m)
    m = truth_m > floor * truth_m.max()
    if not m.any():
        return 0.0
    return float(np.max(np.abs(np.asarray(v)[m] - np.asarray(truth_v)[m])))


def assert_band_tolerance(gpu, ref, tols, label=""):
    """GPU vs the FP64 reference/oracle with per-band relative tolerances (used where no exact
    truth is at hand; the tolerances are the reference's own error envelope on similar input)."""
    errs = band_max_rel(gpu, ref)
    for i, (e, t) in enumerate(zip(errs, tols)):
        assert e <= t, f"{label}: band {i}: |gpu - ref| {e:.3e} > {t:.1e}"
    return errs
