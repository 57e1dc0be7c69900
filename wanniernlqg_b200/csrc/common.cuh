// common.cuh - complex arithmetic on double2/float2 and small device utilities.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define WNLQG_HD __host__ __device__ __forceinline__
#define WNLQG_D __device__ __forceinline__

// ---- complex helpers (re = .x, im = .y) -------------------------------------------------
WNLQG_HD double2 cmk(double r, double i) { return make_double2(r, i); }
WNLQG_HD double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
WNLQG_HD double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
WNLQG_HD double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
WNLQG_HD double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
WNLQG_HD double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
WNLQG_HD double2 cmuli(double2 a) { return make_double2(-a.y, a.x); }          // i*a
WNLQG_HD double2 cmulmi(double2 a) { return make_double2(a.y, -a.x); }         // -i*a
// acc + a*b
WNLQG_HD double2 cfma(double2 a, double2 b, double2 acc) {
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, acc.x)), fma(a.x, b.y, fma(a.y, b.x, acc.y)));
}
// acc + conj(a)*b
WNLQG_HD double2 cfmaconj(double2 a, double2 b, double2 acc) {
    return make_double2(fma(a.x, b.x, fma(a.y, b.y, acc.x)), fma(a.x, b.y, fma(-a.y, b.x, acc.y)));
}

WNLQG_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
WNLQG_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
WNLQG_HD float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
WNLQG_HD float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
WNLQG_HD float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
WNLQG_HD float2 cmuli(float2 a) { return make_float2(-a.y, a.x); }
WNLQG_HD float2 cmulmi(float2 a) { return make_float2(a.y, -a.x); }
WNLQG_HD float2 cfma(float2 a, float2 b, float2 acc) {
    return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y)));
}
WNLQG_HD float2 cfmaconj(float2 a, float2 b, float2 acc) {
    return make_float2(fmaf(a.x, b.x, fmaf(a.y, b.y, acc.x)), fmaf(a.x, b.y, fmaf(-a.y, b.x, acc.y)));
}

WNLQG_HD double2 make_neg(double2 a) { return make_double2(-a.x, -a.y); }
WNLQG_HD float2 make_neg(float2 a) { return make_float2(-a.x, -a.y); }

// Complex type traits for templated kernels: real type R, complex type C.
template <typename A, typename B> struct same_type { static constexpr bool value = false; };
template <typename A> struct same_type<A, A> { static constexpr bool value = true; };

template <typename R> struct cplx_of;
template <> struct cplx_of<double> { typedef double2 type; };
template <> struct cplx_of<float> { typedef float2 type; };

WNLQG_HD double2 to_c64(double2 a) { return a; }
WNLQG_HD double2 to_c64(float2 a) { return make_double2((double)a.x, (double)a.y); }
template <typename C> WNLQG_HD C from_c64(double2 a);
template <> WNLQG_HD double2 from_c64<double2>(double2 a) { return a; }
template <> WNLQG_HD float2 from_c64<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <typename C> WNLQG_HD C czero();
template <> WNLQG_HD double2 czero<double2>() { return make_double2(0.0, 0.0); }
template <> WNLQG_HD float2 czero<float2>() { return make_float2(0.0f, 0.0f); }

// Neumaier compensated addition of one double into (sum, comp).
WNLQG_HD void neumaier_add(double &sum, double &comp, double v) {
    double t = sum + v;
    if (fabs(sum) >= fabs(v)) comp += (sum - t) + v;
    else comp += (v - t) + sum;
    sum = t;
}

// Physical constants (src/Core/Constants.jl:1-4 of the reference).
#define WNLQG_ELEMENTARY_CHARGE_C 1.602176634e-19
#define WNLQG_HBAR_J_S 1.054571817e-34
#define WNLQG_HBAR_EV_S 6.582119569e-16
#define WNLQG_KB_EV_K 8.617333262e-5
#define WNLQG_PI 3.14159265358979323846
