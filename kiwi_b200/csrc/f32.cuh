// A float that stays a float: the real type with which the lattice tiers (lattice_math.cuh, written over T
// with double literals such as 1. / 6. or 0.5 * kPi) are instantiated for the FP32-mixed form.  Arithmetic
// with a double constant converts the constant to float first, so every operation of the instantiated tier
// is an FP32 operation and every libm call the FP32 one (atanf, log1pf, sqrtf, atan2f).
#pragma once

#include <math.h>

namespace kiwi_b200 {
namespace f32 {

#ifdef __CUDACC__
#define KIWI_FF __host__ __device__ __forceinline__
#else
#define KIWI_FF inline
#endif

struct F32 {
    float v;
    KIWI_FF F32() : v(0.0f) {}
    KIWI_FF F32(double x) : v((float)x) {}
    KIWI_FF explicit operator double() const { return (double)v; }
};

KIWI_FF F32 mk(float x) {
    F32 r;
    r.v = x;
    return r;
}

KIWI_FF F32 operator+(F32 a, F32 b) { return mk(a.v + b.v); }
KIWI_FF F32 operator-(F32 a, F32 b) { return mk(a.v - b.v); }
KIWI_FF F32 operator*(F32 a, F32 b) { return mk(a.v * b.v); }
KIWI_FF F32 operator/(F32 a, F32 b) { return mk(a.v / b.v); }
KIWI_FF F32 operator-(F32 a) { return mk(-a.v); }
KIWI_FF F32 operator+(F32 a, double b) { return mk(a.v + (float)b); }
KIWI_FF F32 operator+(double a, F32 b) { return mk((float)a + b.v); }
KIWI_FF F32 operator-(F32 a, double b) { return mk(a.v - (float)b); }
KIWI_FF F32 operator-(double a, F32 b) { return mk((float)a - b.v); }
KIWI_FF F32 operator*(F32 a, double b) { return mk(a.v * (float)b); }
KIWI_FF F32 operator*(double a, F32 b) { return mk((float)a * b.v); }
KIWI_FF F32 operator/(F32 a, double b) { return mk(a.v / (float)b); }
KIWI_FF F32 operator/(double a, F32 b) { return mk((float)a / b.v); }
KIWI_FF F32& operator+=(F32& a, F32 b) { return a = a + b; }
KIWI_FF F32& operator-=(F32& a, F32 b) { return a = a - b; }
KIWI_FF F32& operator*=(F32& a, F32 b) { return a = a * b; }

#define KIWI_F32_CMP(op)                                                           \
    KIWI_FF bool operator op(F32 a, F32 b) { return a.v op b.v; }                  \
    KIWI_FF bool operator op(F32 a, double b) { return a.v op (float)b; }          \
    KIWI_FF bool operator op(double a, F32 b) { return (float)a op b.v; }
KIWI_F32_CMP(<)
KIWI_F32_CMP(>)
KIWI_F32_CMP(<=)
KIWI_F32_CMP(>=)
KIWI_F32_CMP(==)
KIWI_F32_CMP(!=)
#undef KIWI_F32_CMP

KIWI_FF F32 sqrt(F32 x) { return mk(sqrtf(x.v)); }
KIWI_FF F32 fabs(F32 x) { return mk(fabsf(x.v)); }
KIWI_FF F32 atan(F32 x) { return mk(atanf(x.v)); }
KIWI_FF F32 atan2(F32 y, F32 x) { return mk(atan2f(y.v, x.v)); }
KIWI_FF F32 log1p(F32 x) { return mk(log1pf(x.v)); }
KIWI_FF F32 fmax(F32 x, double c) { return mk(fmaxf(x.v, (float)c)); }
KIWI_FF F32 fmin(double c, F32 x) { return mk(fminf((float)c, x.v)); }
KIWI_FF F32 acos(F32 x) { return mk(acosf(x.v)); }
KIWI_FF F32 sin(F32 x) { return mk(sinf(x.v)); }
KIWI_FF F32 cos(F32 x) { return mk(cosf(x.v)); }
KIWI_FF F32 atanh(F32 x) { return mk(atanhf(x.v)); }
KIWI_FF F32 fma(F32 a, F32 b, F32 c) { return mk(fmaf(a.v, b.v, c.v)); }

#undef KIWI_FF

}  // namespace f32
using f32::F32;
}  // namespace kiwi_b200
