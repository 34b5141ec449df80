// hb_corrector.cuh -- Hermite corrector and Aarseth timestep on the device.
//
// Restates, per particle, Particle::correct / aarseth_step_quant / init_dt of
// the reference (SRC/hermite4.h:72-153, SRC/hermite6.h:77-184,
// SRC/hermite8.h:92-222) and the bit-level helpers of SRC/pownth.h:3-33
// (power-of-two quantised n-th root; exact h = dt/2 and 2/dt for power-of-two
// dt).  The arithmetic order follows the reference's vector expressions.
#pragma once
#include <cstdint>
#include "hb_common.cuh"

namespace hb {

// x^(1/N) rounded down to a power of two, by integer arithmetic on the
// biased exponent: e' = (e - (1023 % N)) / N + (1023 - 1023 / N).
template <int N>
__device__ __forceinline__ double quantised_root(double x)
{
    uint64_t e = (uint64_t)__double_as_longlong(x) >> 52;
    e = (e - (uint64_t)(1023 % N)) / N + (uint64_t)(1023 - 1023 / N);
    return __longlong_as_double((long long)(e << 52));
}

// dt a power of two: h = dt/2 and 1/h = 2/dt exactly, from the exponent bits.
// (A vector divided by a scalar is a multiplication by its reciprocal, as the
// reference's vector3 does it, SRC/vector3.h:127-130.)
__device__ __forceinline__ void half_step(double dt, double &h, double &hinv)
{
    const long long b = __double_as_longlong(dt) - (1LL << 52);
    h = __longlong_as_double(b);
    hinv = __longlong_as_double((2046LL << 52) - b);
}

struct V3 {
    double x, y, z;
};
__device__ __forceinline__ V3 v3(const double *p) { return V3{p[0], p[1], p[2]}; }
__device__ __forceinline__ void st3(double *p, V3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return V3{__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y), __dadd_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return V3{__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 operator*(double s, V3 a) { return V3{__dmul_rn(s, a.x), __dmul_rn(s, a.y), __dmul_rn(s, a.z)}; }
__device__ __forceinline__ V3 operator*(V3 a, double s) { return s * a; }
__device__ __forceinline__ double norm2(V3 a)
{
    return __dadd_rn(__dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y)), __dmul_rn(a.z, a.z));
}

// Particle state in a j-particle record r (pos mass vel tlast acc jrk [snp
// crk] [d4a d5a] [posL]); f = the new force (acc jrk [snp] [crk]).  ORDER 9
// is the 8th-order corrector with double-double positions
// (Particle::correct, SRC/hermite8dd.h:187-239).  Returns the new
// dt; writes the corrected state into r.  If aux is not null it receives the
// two higher derivatives the reference's Particle also keeps and dumps (snp
// crk at 4th order, d4a d5a at 6th, d6a d7a at 8th: 6 doubles).
template <int ORDER>
__device__ double correct_particle(double *r, const double *f, double dt, double etapow,
                                   double dtlim, double *aux = nullptr)
{
    double h, hinv;
    half_step(dt, h, hinv);
    const V3 pos = v3(r + 0), vel = v3(r + 4), acc = v3(r + 8), jrk = v3(r + 11);
    const V3 fa = v3(f + 0), fj = v3(f + 3);
    const V3 Ap = fa + acc, Am = fa - acc;
    const V3 Jp = (fj + jrk) * h, Jm = (fj - jrk) * h;
    double dtq;
    if constexpr (ORDER == 4) {
        const V3 vel1 = vel + h * (Ap - (1. / 3.) * Jm);
        const V3 pos1 = pos + h * ((vel + vel1) + h * ((-(1. / 3.)) * Am));
        V3 snp = (__dmul_rn(__dmul_rn(0.5, hinv), hinv)) * Jm;
        const V3 crk = (__dmul_rn(__dmul_rn(__dmul_rn(1.5, hinv), hinv), hinv)) * (Jp - Am);
        snp = snp + h * crk;
        st3(r + 0, pos1);
        st3(r + 4, vel1);
        st3(r + 8, fa);
        st3(r + 11, fj);
        if (aux) {
            st3(aux + 0, snp);
            st3(aux + 3, crk);
        }
        const double s0 = norm2(fa), s1 = norm2(fj), s2 = norm2(snp), s3 = norm2(crk);
        const double u = __dadd_rn(sqrt(__dmul_rn(s0, s2)), s1);
        const double l = __dadd_rn(sqrt(__dmul_rn(s1, s3)), s2);
        dtq = quantised_root<2>(__dmul_rn(etapow, __ddiv_rn(u, l)));
    } else if constexpr (ORDER == 6) {
        const V3 snp = v3(r + 14);
        const V3 fs = v3(f + 6);
        const double hh = __dmul_rn(h, h);
        const V3 Sp = (fs + snp) * hh, Sm = (fs - snp) * hh;
        const V3 vel1 = vel + h * ((Ap - 0.4 * Jm) + (1. / 15) * Sp);
        const V3 pos1 = pos + h * ((vel + vel1) + h * ((-0.4) * Am + (1. / 15) * Jp));
        const double hinv2 = __dmul_rn(hinv, hinv), hinv3 = __dmul_rn(hinv2, hinv);
        const double hinv4 = __dmul_rn(hinv2, hinv2), hinv5 = __dmul_rn(hinv2, hinv3);
        V3 crk = (__dmul_rn(0.75, hinv3)) * (((-5.) * Am + 5. * Jp) - Sm);
        V3 d4a = (__dmul_rn(1.5, hinv4)) * ((-1.) * Jm + Sp);
        const V3 d5a = (__dmul_rn(7.5, hinv5)) * ((3. * Am - 3. * Jp) + Sm);
        crk = crk + h * (d4a + __dmul_rn(0.5, h) * d5a);
        d4a = d4a + h * d5a;
        st3(r + 0, pos1);
        st3(r + 4, vel1);
        st3(r + 8, fa);
        st3(r + 11, fj);
        st3(r + 14, fs);
        st3(r + 17, crk);
        if (aux) {
            st3(aux + 0, d4a);
            st3(aux + 3, d5a);
        }
        const double s0 = norm2(fa), s1 = norm2(fj), s2 = norm2(fs);
        const double s3 = norm2(crk), s4 = norm2(d4a), s5 = norm2(d5a);
        const double u = __dadd_rn(sqrt(__dmul_rn(s0, s2)), s1);
        const double l = __dadd_rn(sqrt(__dmul_rn(s3, s5)), s4);
        dtq = quantised_root<6>(__dmul_rn(etapow, __ddiv_rn(u, l)));
    } else {
        const V3 snp = v3(r + 14), crk0 = v3(r + 17);
        const V3 fs = v3(f + 6), fc = v3(f + 9);
        const double hh = __dmul_rn(h, h), hhh = __dmul_rn(hh, h);
        const V3 Sp = (fs + snp) * hh, Sm = (fs - snp) * hh;
        const V3 Cp = (fc + crk0) * hhh, Cm = (fc - crk0) * hhh;
        const V3 vel1 = vel + h * (((Ap + (-3. / 7.) * Jm) + (2. / 21) * Sp) - (1. / 105.) * Cm);
        const V3 dpos = h * ((vel + vel1) + h * (((-3. / 7.) * Am + (2. / 21) * Jp) - (1. / 105.) * Sm));
        const double hinv2 = __dmul_rn(hinv, hinv), hinv3 = __dmul_rn(hinv2, hinv);
        const double hinv4 = __dmul_rn(hinv2, hinv2), hinv5 = __dmul_rn(hinv2, hinv3);
        const double hinv6 = __dmul_rn(hinv3, hinv3), hinv7 = __dmul_rn(hinv3, hinv4);
        V3 d4a = (__ddiv_rn(__dmul_rn(hinv4, 24.), 32.)) * (((-5.) * Jm + 5. * Sp) - Cm);
        V3 d5a = (__ddiv_rn(__dmul_rn(hinv5, 120.), 32.)) * (((21. * Am - 21. * Jp) + 8. * Sm) - Cp);
        V3 d6a = (__ddiv_rn(__dmul_rn(hinv6, 720.), 32.)) * ((Jm - Sp) + Cm * __ddiv_rn(1., 3.));
        const V3 d7a = (__ddiv_rn(__dmul_rn(hinv7, 5040.), 32.)) *
                       ((((-5.) * Am + 5. * Jp) - 2. * Sm) + Cp * __ddiv_rn(1., 3.));
        const double h2 = __dmul_rn(0.5, h), h3 = __dmul_rn(1. / 3., h);
        d4a = d4a + h * (d5a + h2 * (d6a + h3 * d7a));
        d5a = d5a + h * (d6a + h2 * d7a);
        d6a = d6a + h * d7a;
        if constexpr (ORDER == 9) {
            // double-double position: dd_accumulate(posH, posL, dpos)
            // (SRC/hermite8dd.h:4-23,203)
            double *xh = r, *xl = r + kRecPosL;
            const double dp[3] = {dpos.x, dpos.y, dpos.z};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double yh = __dadd_rn(xh[k], dp[k]);
                const double res = __dsub_rn(dp[k], __dsub_rn(yh, xh[k]));
                const double yl = __dadd_rn(xl[k], res);
                const double zh = __dadd_rn(yh, yl);
                const double zl = __dsub_rn(yl, __dsub_rn(zh, yh));
                xh[k] = zh;
                xl[k] = zl;
            }
        } else {
            st3(r + 0, pos + dpos);
        }
        st3(r + 4, vel1);
        st3(r + 8, fa);
        st3(r + 11, fj);
        st3(r + 14, fs);
        st3(r + 17, fc);
        st3(r + 20, d4a);
        st3(r + 23, d5a);
        if (aux) {
            st3(aux + 0, d6a);
            st3(aux + 3, d7a);
        }
        const double s0 = norm2(fa), s1 = norm2(fj), s2 = norm2(fs);
        const double s5 = norm2(d5a), s6 = norm2(d6a), s7 = norm2(d7a);
        const double u = __dadd_rn(sqrt(__dmul_rn(s0, s2)), s1);
        const double l = __dadd_rn(sqrt(__dmul_rn(s5, s7)), s6);
        dtq = quantised_root<10>(__dmul_rn(etapow, __ddiv_rn(u, l)));
    }
    r[7] = __dadd_rn(r[7], dt);   // tlast += dt
    return dtq < dtlim ? dtq : dtlim;
}

// Initial timestep from the first force evaluation, halving 0.25*dtmax until
// it is below the natural step (the reference's init_dt); at most 64 halvings.
template <int ORDER>
__device__ double initial_dt(const double *f, double eta_s, double dtmax)
{
    const double s0 = norm2(v3(f + 0)), s1 = norm2(v3(f + 3));
    double dtnat;
    if constexpr (ORDER == 4) {
        dtnat = __dmul_rn(eta_s, sqrt(__ddiv_rn(s0, s1)));
    } else if constexpr (ORDER == 6) {
        const double s2 = norm2(v3(f + 6));
        dtnat = __dmul_rn(eta_s, sqrt(sqrt(__ddiv_rn(s0, s2))));
    } else {
        const double s2 = norm2(v3(f + 6)), s3 = norm2(v3(f + 9));
        const double u = __dadd_rn(sqrt(__dmul_rn(s0, s2)), s1);
        const double l = __dadd_rn(sqrt(__dmul_rn(s1, s3)), s2);
        dtnat = __dmul_rn(eta_s, sqrt(__ddiv_rn(u, l)));
    }
    double dt = __dmul_rn(0.25, dtmax);
    for (int k = 0; k < 64 && dt > dtnat; ++k) dt = __dmul_rn(dt, 0.5);
    return dt;
}

}  // namespace hb
