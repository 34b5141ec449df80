// hb_math.cuh -- per-particle predictor and per-pair interaction arithmetic.
//
// The algebra is the reference's (it has to be: these are the Hermite
// derivatives of the softened Newtonian force); the arrangement is ours.
//   predictor:   SRC/hermite4-titan.cu:20-61, SRC/hermite6-titan.cu:20-94,
//                SRC/hermite8-titan.cu:20-134 (spec: generic GPredictor in
//                SRC/hermite{4,6,8}.h)
//   interaction: SRC/hermite4-titan.cu:122-154, SRC/hermite6-titan.cu:156-208,
//                SRC/hermite8-titan.cu:195-265 (spec: SRC/hermite4.h:342-357,
//                SRC/hermite6.h:332-360, SRC/hermite8.h:385-425)
#pragma once
#include <cuda_runtime.h>
#include "hb_common.cuh"

namespace hb {

// ---------------------------------------------------------------------------
// Reciprocal square root in FP64.
// Seed y0: the double-precision approximate reciprocal square root
// instruction (PTX rsqrt.approx.ftz.f64; no float conversions), then one
// third-order correction from the binomial series
//   (1 - h)^(-1/2) = 1 + h/2 + 3h^2/8 + O(h^3),   h = 1 - x*y0^2,
// so y = y0*(1 + h/2 + 3h^2/8) has relative error ~ (5/16) h^3: below FP64
// rounding for any seed error under 2^-18 (tests/test_fp64_rsqrt.py measures
// the seed's error on the device).  HB_FP64_SEED=0 selects the
// single-precision seed (double)rsqrtf((float)x) instead (two conversions).
#ifndef HB_FP64_SEED
#define HB_FP64_SEED 1
#endif
__device__ __forceinline__ double rsqrt_seed_fp64(double x)
{
#if HB_FP64_SEED == 1
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    return y;
#else
    return (double)rsqrtf((float)x);
#endif
}

__device__ __forceinline__ double rsqrt_fp64(double x)
{
    const double y0 = rsqrt_seed_fp64(x);
    const double h = fma(-x * y0, y0, 1.0);
    return fma(y0 * h, fma(h, 0.375, 0.5), y0);
}

// ---------------------------------------------------------------------------
// Predictor: slot record -> position, velocity [, acceleration [, jerk]] at
// tsys, Horner form with c_k = dt/k.  ORDER 9 (double-double positions, the
// reference's GPredictor of SRC/hermite8dd.h:284-314): x is the unchanged
// high part posH, xl the low part posL advanced by the 8th-order Taylor
// series.
template <int ORDER>
__device__ __forceinline__ void predict_slot(const double *r, double tsys,
                                             double x[3], double v[3],
                                             double a[3], double jk[3], double *xl = nullptr)
{
    const double dt = tsys - r[7];
    const double c2 = dt * (1.0 / 2.0), c3 = dt * (1.0 / 3.0);
    const double c4 = dt * (1.0 / 4.0), c5 = dt * (1.0 / 5.0);
    const double c6 = dt * (1.0 / 6.0), c7 = dt * (1.0 / 7.0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double p0 = r[k], v0 = r[4 + k], a0 = r[8 + k], j0 = r[11 + k];
        if constexpr (ORDER == 4) {
            x[k] = p0 + dt * (v0 + c2 * (a0 + c3 * j0));
            v[k] = v0 + dt * (a0 + c2 * j0);
        } else if constexpr (ORDER == 6) {
            const double s0 = r[14 + k], k0 = r[17 + k];
            x[k] = p0 + dt * (v0 + c2 * (a0 + c3 * (j0 + c4 * (s0 + c5 * k0))));
            v[k] = v0 + dt * (a0 + c2 * (j0 + c3 * (s0 + c4 * k0)));
            a[k] = a0 + dt * (j0 + c2 * (s0 + c3 * k0));
        } else {
            const double s0 = r[14 + k], k0 = r[17 + k];
            const double d4 = r[20 + k], d5 = r[23 + k];
            if constexpr (ORDER == 9) {
                x[k] = p0;
                xl[k] = r[kRecPosL + k] + dt * (v0 + c2 * (a0 + c3 * (j0 + c4 * (s0 + c5 * (k0 + c6 * (d4 + c7 * d5))))));
            } else {
                x[k] = p0 + dt * (v0 + c2 * (a0 + c3 * (j0 + c4 * (s0 + c5 * (k0 + c6 * (d4 + c7 * d5))))));
            }
            v[k] = v0 + dt * (a0 + c2 * (j0 + c3 * (s0 + c4 * (k0 + c5 * (d4 + c6 * d5)))));
            a[k] = a0 + dt * (j0 + c2 * (s0 + c3 * (k0 + c4 * (d4 + c5 * d5))));
            jk[k] = j0 + dt * (s0 + c2 * (k0 + c3 * (d4 + c4 * d5)));
        }
    }
}

// ---------------------------------------------------------------------------
// FP64 pair interaction.  `I` holds the i-particle, `J` the j-particle
// (x[3], m, v[3], a[3], jk[3]); f accumulates acc, jrk [, snp [, crk]].
struct Body64 {
    double x[3], m, v[3], a[3], jk[3], xl[3];   // xl: ORDER 9 only
};

template <int ORDER>
__device__ __forceinline__ void interact64(const Body64 &I, const Body64 &J,
                                           double eps2, double *f)
{
    double dr[3], dv[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if constexpr (ORDER == 9)   // (posHj - posHi) + (posLj - posLi), SRC/hermite8dd.h:358
            dr[k] = (J.x[k] - I.x[k]) + (J.xl[k] - I.xl[k]);
        else
            dr[k] = J.x[k] - I.x[k];
        dv[k] = J.v[k] - I.v[k];
    }
    const double r2 = fma(dr[2], dr[2], fma(dr[1], dr[1], fma(dr[0], dr[0], eps2)));
    const double rv = fma(dr[2], dv[2], fma(dr[1], dv[1], dr[0] * dv[0]));
    double ri;
    if constexpr (ORDER == 9)       // pairs at zero separation are skipped (SRC/hermite8dd.h:362)
        ri = r2 == eps2 ? 0.0 : rsqrt_fp64(r2);
    else
        ri = rsqrt_fp64(r2);
    const double ri2 = ri * ri;
    const double mr3 = J.m * ri * ri2;
    const double al = rv * ri2;              // alpha = (r.v)/r^2
    double t[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        f[k] = fma(mr3, dr[k], f[k]);
        t[k] = fma(-3.0 * al, dr[k], dv[k]);   // v - 3 alpha r
        f[3 + k] = fma(mr3, t[k], f[3 + k]);
    }
    if constexpr (ORDER >= 6) {
        double da[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) da[k] = J.a[k] - I.a[k];
        // v.v + r.a as one chain of fused multiply-adds (one add fewer than
        // two dot products and their sum)
        const double vvra = fma(dr[2], da[2], fma(dr[1], da[1], fma(dr[0], da[0],
                            fma(dv[2], dv[2], fma(dv[1], dv[1], dv[0] * dv[0])))));
        const double be = fma(al, al, vvra * ri2);       // beta
        double u[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            u[k] = fma(-3.0 * be, dr[k], fma(-6.0 * al, t[k], da[k]));
            f[6 + k] = fma(mr3, u[k], f[6 + k]);
        }
        if constexpr (ORDER >= 8) {
            double dj[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) dj[k] = J.jk[k] - I.jk[k];
            const double va = fma(dv[2], da[2], fma(dv[1], da[1], dv[0] * da[0]));
            const double rj = fma(dr[2], dj[2], fma(dr[1], dj[1], dr[0] * dj[0]));
            // gamma = (3 v.a + r.j)/r^2 + alpha (3 beta - 4 alpha^2)
            const double ga = fma(al, fma(-4.0 * al, al, 3.0 * be), fma(3.0, va, rj) * ri2);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double w = fma(-3.0 * ga, dr[k],
                                 fma(-9.0 * be, t[k], fma(-9.0 * al, u[k], dj[k])));
                f[9 + k] = fma(mr3, w, f[9 + k]);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Mixed precision, two j-particles at a time in packed FP32 (sm_100 f32x2).
// The i-particle is held negated and duplicated into both halves, so every
// difference is one packed add; positions carry a hi/lo split so the relative
// position is ((xj_hi - xi_hi) + (xj_lo - xi_lo)), exact to FP32 rounding of
// the result even when |x| >> |xj - xi|.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

struct NegI32 {                 // -(i-particle), duplicated
    float2 xh[3], xl[3], v[3], a[3], jk[3];
};
struct JPair32 {                // two j-particles
    float2 xh[3], xl[3], m, v[3], a[3], jk[3];
};

// Reciprocal square root of both halves: hardware rsqrt (documented maximum
// error 2 ulp), then, if REFINE, one Newton step y <- y*(3/2 - x y^2/2).
template <bool REFINE>
__device__ __forceinline__ float2 rsqrt2(float2 x)
{
    float2 y = make_float2(rsqrtf(x.x), rsqrtf(x.y));
    if constexpr (REFINE) {
        const float2 xyy = mul2(mul2(x, y), y);
        y = mul2(y, fma2(xyy, f2(-0.5f), f2(1.5f)));
    }
    return y;
}

// Accumulates into s[] (FP32, packed over the two j) for acc, jrk [, snp
// [, crk]]; the caller flushes these partial sums into FP64 accumulators.
template <int ORDER, bool REFINE>
__device__ __forceinline__ void interact_mixed(const NegI32 &I, const JPair32 &J,
                                               float2 eps2, float2 *s)
{
    float2 dr[3], dv[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        dr[k] = add2(add2(J.xh[k], I.xh[k]), add2(J.xl[k], I.xl[k]));
        dv[k] = add2(J.v[k], I.v[k]);
    }
    const float2 r2 = fma2(dr[2], dr[2], fma2(dr[1], dr[1], fma2(dr[0], dr[0], eps2)));
    const float2 rv = fma2(dr[2], dv[2], fma2(dr[1], dv[1], mul2(dr[0], dv[0])));
    const float2 ri = rsqrt2<REFINE>(r2);
    const float2 ri2 = mul2(ri, ri);
    const float2 mr3 = mul2(mul2(J.m, ri), ri2);
    const float2 al = mul2(rv, ri2);
    const float2 al3 = mul2(al, f2(-3.0f));
    float2 t[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        s[k] = fma2(mr3, dr[k], s[k]);
        t[k] = fma2(al3, dr[k], dv[k]);
        s[3 + k] = fma2(mr3, t[k], s[3 + k]);
    }
    if constexpr (ORDER >= 6) {
        float2 da[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) da[k] = add2(J.a[k], I.a[k]);
        const float2 vvra = fma2(dr[2], da[2], fma2(dr[1], da[1], fma2(dr[0], da[0],
                            fma2(dv[2], dv[2], fma2(dv[1], dv[1], mul2(dv[0], dv[0]))))));
        const float2 be = fma2(al, al, mul2(vvra, ri2));
        const float2 al6 = add2(al3, al3);
        const float2 be3 = mul2(be, f2(-3.0f));
        float2 u[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            u[k] = fma2(be3, dr[k], fma2(al6, t[k], da[k]));
            s[6 + k] = fma2(mr3, u[k], s[6 + k]);
        }
        if constexpr (ORDER == 8) {
            float2 dj[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) dj[k] = add2(J.jk[k], I.jk[k]);
            const float2 va = fma2(dv[2], da[2], fma2(dv[1], da[1], mul2(dv[0], da[0])));
            const float2 rj = fma2(dr[2], dj[2], fma2(dr[1], dj[1], mul2(dr[0], dj[0])));
            // gamma = (3 v.a + r.j)/r^2 + alpha (3 beta - 4 alpha^2)
            const float2 g0 = mul2(fma2(f2(3.0f), va, rj), ri2);
            const float2 g1 = fma2(mul2(al, f2(-4.0f)), al, mul2(be, f2(3.0f)));
            const float2 ga3 = mul2(fma2(al, g1, g0), f2(-3.0f));
            const float2 al9 = mul2(al, f2(-9.0f));
            const float2 be9 = mul2(be, f2(-9.0f));
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float2 w = fma2(ga3, dr[k], fma2(be9, t[k], fma2(al9, u[k], dj[k])));
                s[9 + k] = fma2(mr3, w, s[9 + k]);
            }
        }
    }
}

}  // namespace hb
