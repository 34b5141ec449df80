// ref_gravity.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A thin extern "C" wrapper that compiles the reference's OWN force
// calculator (its `struct Gravity` from SRC/hermite{4,6,8}.h, generic or
// AVX backend) from the reference sources where they lie, so that the oracle
// restatement and the CUDA path can be compared with the reference itself,
// and so that the benchmark's CPU arm times the reference's AVX path.
// Built by oracle/Makefile into oracle/_ref/ (git-ignored); never shipped as
// part of the product.
//
// Compile with -I<reference>/SRC and exactly one of -DREF_ORDER=4|6|8|9 (9: the
// 8th order with double-double positions, SRC/hermite8dd.h), and
// optionally -DAVX_GRAVITY (the reference's AVX backend, SRC/hermite*-avx.h).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cassert>
#include "vector3.h"

#ifdef __AVX__
typedef double v2df __attribute__((vector_size(16)));
typedef double v4df __attribute__((vector_size(32)));
#endif
#include "allocate.h"

#if REF_ORDER == 4
#include "hermite4.h"
#elif REF_ORDER == 6
#include "hermite6.h"
#elif REF_ORDER == 8
#include "hermite8.h"
#elif REF_ORDER == 9
#include "hermite8dd.h"   // 8th order, double-double positions
#else
#error "REF_ORDER must be 4, 6, 8 or 9"
#endif

namespace {
constexpr int kOrder = REF_ORDER;
constexpr int kRecWords = 8 + 3 * (kOrder - 2);
constexpr int kForceWords = 3 * (kOrder / 2);

struct RefCtx {
    int n;
    Gravity *g;
    Force *fbuf;   // padded to a multiple of 4 for the AVX backend
};

Particle make_particle(const double *r)
{
    // record: pos[3] mass vel[3] tlast derivs[3*(order-2)]; order 9: the
    // 8th-order record, then posL[3]
    Particle p(0, r[3], dvec3(r[0], r[1], r[2]), dvec3(r[4], r[5], r[6]));
    p.tlast = r[7];
    dvec3 *d = &p.acc;   // acc, jrk, snp, crk, d4a, d5a are contiguous
    const int nd = kOrder == 9 ? 6 : kOrder - 2;
    for (int k = 0; k < nd; k++)
        d[k] = dvec3(r[8 + 3 * k], r[9 + 3 * k], r[10 + 3 * k]);
#if REF_ORDER == 9
    p.posL = dvec3(r[26], r[27], r[28]);
#endif
    return p;
}
}  // namespace

extern "C" {

int ref_order(void) { return kOrder; }

void *ref_create(int n)
{
    RefCtx *c = new RefCtx;
    c->n = n;
    c->g = new Gravity(n);
    c->fbuf = allocate<Force, 64>((size_t)n + 4);
    return c;
}

void ref_destroy(void *vc)
{
    RefCtx *c = static_cast<RefCtx *>(vc);
    delete c->g;
    deallocate<Force, 64>(c->fbuf);
    delete c;
}

void ref_set_jp(void *vc, int addr, const double *rec)
{
    RefCtx *c = static_cast<RefCtx *>(vc);
    c->g->set_jp(addr, make_particle(rec));
}

void ref_set_jp_all(void *vc, int n, const double *recs)
{
    RefCtx *c = static_cast<RefCtx *>(vc);
    for (int i = 0; i < n; i++)
        c->g->set_jp(i, make_particle(recs + (size_t)i * kRecWords));
}

void ref_predict_all(void *vc, double tsys)
{
    static_cast<RefCtx *>(vc)->g->predict_all(tsys);
}

void ref_force(void *vc, int nact, double eps2, double *out)
{
    RefCtx *c = static_cast<RefCtx *>(vc);
    c->g->calc_force_on_first_nact(nact, eps2, c->fbuf);
    for (int i = 0; i < nact; i++)
        std::memcpy(out + (size_t)i * kForceWords, &c->fbuf[i],
                    sizeof(double) * kForceWords);
}

void ref_potential(void *vc, double eps2, double *pot)
{
    RefCtx *c = static_cast<RefCtx *>(vc);
    double *buf = allocate<double, 64>((size_t)c->n + 4);
    c->g->calc_potential(eps2, buf);
    std::memcpy(pot, buf, sizeof(double) * c->n);
    deallocate<double, 64>(buf);
}

}  // extern "C"
