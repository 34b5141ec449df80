/*
 * fp32pair.h -- TEST INFRASTRUCTURE ONLY: the mixed-precision force kernel's
 * pair arithmetic (hermite_b200/csrc/hb_math.cuh interact_mixed and the
 * chunk flush of hb_force.cuh chunk_mixed) restated in C float, for the
 * noise-tolerance runs (noise_gravity.inl) and the per-evaluation error
 * comparisons of tests/test_noise_tolerance.py.
 *
 * Predicted states as the oracle's (oracle/hermite_oracle.c):
 *   pos[3] mass vel[3] [acc[3]] [jrk[3]]   (7 / 10 / 13 doubles)
 * Relative positions from hi/lo FP32 parts, ((xj_hi - xi_hi) + (xj_lo -
 * xi_lo)); velocities [, accelerations [, jerks]] as single FP32 values, or
 * with split != 0 as hi/lo pairs like the positions; FP32 interaction;
 * partial sums over the 16 pairs of each half of a 32-slot chunk flushed
 * into FP64; rsqrt correctly rounded (the kernel's hardware rsqrt is within
 * 2 ulp).
 */
#ifndef FP32PAIR_H
#define FP32PAIR_H
#include <math.h>
#include <stddef.h>

static inline void fp32_split(double x, float *h, float *l)
{
    *h = (float)x;
    *l = (float)(x - (double)*h);
}

/* difference b - a of two FP64 values as the kernel forms it */
static inline float fp32_diff(double b, double a, int split)
{
    if (!split) return (float)b + -(float)a;
    float bh, bl, ah, al;
    fp32_split(b, &bh, &bl);
    fp32_split(a, &ah, &al);
    return (bh + -ah) + (bl + -al);
}

static inline void fp32pair_force_one(int order, int n, const double *pred, int i, float eps2,
                                      int split, double *f)
{
    const int P = 7 + 3 * (order / 2 - 2), F = 3 * (order / 2);
    const double *pi = pred + (size_t)i * P;
    for (int c = 0; c < F; ++c) f[c] = 0.0;
    for (int c0 = 0; c0 < n; c0 += 32) {
        float s[2][12] = {{0}};
        for (int jl = 0; jl < 32 && c0 + jl < n; ++jl) {
            const double *pj = pred + (size_t)(c0 + jl) * P;
            float dr[3], dv[3], da[3] = {0, 0, 0}, dj[3] = {0, 0, 0};
            for (int k = 0; k < 3; ++k) {
                dr[k] = fp32_diff(pj[k], pi[k], 1);
                dv[k] = fp32_diff(pj[4 + k], pi[4 + k], split);
                if (order >= 6) da[k] = fp32_diff(pj[7 + k], pi[7 + k], split);
                if (order >= 8) dj[k] = fp32_diff(pj[10 + k], pi[10 + k], split);
            }
            const float m = (float)pj[3];
            float *a = s[jl & 1];
            const float r2 = fmaf(dr[2], dr[2], fmaf(dr[1], dr[1], fmaf(dr[0], dr[0], eps2)));
            const float rv = fmaf(dr[2], dv[2], fmaf(dr[1], dv[1], dr[0] * dv[0]));
            const float ri = (float)(1.0 / sqrt((double)r2));
            const float ri2 = ri * ri, mr3 = (m * ri) * ri2, al = rv * ri2, al3 = al * -3.0f;
            float t[3], u[3];
            for (int k = 0; k < 3; ++k) {
                a[k] = fmaf(mr3, dr[k], a[k]);
                t[k] = fmaf(al3, dr[k], dv[k]);
                a[3 + k] = fmaf(mr3, t[k], a[3 + k]);
            }
            if (order >= 6) {
                const float vvra = fmaf(dr[2], da[2], fmaf(dr[1], da[1], fmaf(dr[0], da[0],
                                   fmaf(dv[2], dv[2], fmaf(dv[1], dv[1], dv[0] * dv[0])))));
                const float be = fmaf(al, al, vvra * ri2);
                const float al6 = al3 + al3, be3 = be * -3.0f;
                for (int k = 0; k < 3; ++k) {
                    u[k] = fmaf(be3, dr[k], fmaf(al6, t[k], da[k]));
                    a[6 + k] = fmaf(mr3, u[k], a[6 + k]);
                }
                if (order >= 8) {
                    const float va = fmaf(dv[2], da[2], fmaf(dv[1], da[1], dv[0] * da[0]));
                    const float rj = fmaf(dr[2], dj[2], fmaf(dr[1], dj[1], dr[0] * dj[0]));
                    const float g0 = fmaf(3.0f, va, rj) * ri2;
                    const float g1 = fmaf(al * -4.0f, al, be * 3.0f);
                    const float ga3 = fmaf(al, g1, g0) * -3.0f;
                    for (int k = 0; k < 3; ++k) {
                        const float w = fmaf(ga3, dr[k], fmaf(be * -9.0f, t[k],
                                             fmaf(al * -9.0f, u[k], dj[k])));
                        a[9 + k] = fmaf(mr3, w, a[9 + k]);
                    }
                }
            }
        }
        for (int c = 0; c < F; ++c) f[c] += (double)s[0][c] + (double)s[1][c];
    }
}

#endif
