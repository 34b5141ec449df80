// hb_gravity.inl -- the drop-in `struct Gravity` over the hermite_b200 C ABI.
//
// Included by hermite{4,6,8}-titan.h with HB_GRAVITY_ORDER set, after the
// including header (the reference's SRC/hermite{4,6,8}.h) has defined
// `Particle` and `Force`.  Mirrors the members of the reference's CUDA
// Gravity that SRC/nbodysystem.h uses (SRC/nbodysystem.h:152-153,308,326,
// 565-765): the constructor/destructor, set_jp, predict_all,
// calc_force_on_first_nact, calc_potential, and the GParticle / GPredictor
// types (only their sizes are used, for the "prediction bandwidth" report).
//
// Precision: HB_FP64 unless built with -DHB_GRAVITY_PRECISION=HB_MIXED or
// run with HERMITE_B200_PRECISION=mixed|fp64 in the environment.
// Errors print the library's message and abort, as the reference's
// checkCudaErrors does (SRC/cuda_pointer.h:6-10).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "hermite_b200.h"

#ifndef HB_GRAVITY_ORDER
#error "HB_GRAVITY_ORDER must be 4, 6 or 8"
#endif
#ifndef HB_GRAVITY_PRECISION
#define HB_GRAVITY_PRECISION HB_FP64
#endif

struct Gravity {
    enum {
        ORDER = HB_GRAVITY_ORDER,
        NRECORD = 8 + 3 * (HB_GRAVITY_ORDER - 2),
        NPREDICT = 7 + 3 * (HB_GRAVITY_ORDER / 2 - 2),
        NFORCE = 3 * (HB_GRAVITY_ORDER / 2),
    };
    // FP64 sizes of the j-particle record and of the predicted state, so that
    // Profile::show's bandwidth line counts the bytes the FP64 path moves.
    struct GParticle { double w[NRECORD]; };
    struct GPredictor { double w[NPREDICT]; };

    const int nbody;
    hb_ctx *ctx;

    static void check(hb_ctx *c, int status, const char *what)
    {
        if (status != HB_OK) {
            std::fprintf(stderr, "hermite_b200: %s failed: %s%s%s\n", what,
                         hb_status_string(status), c ? ": " : "", c ? hb_last_error(c) : "");
            std::abort();
        }
    }

    static int precision_from_env()
    {
        const char *s = std::getenv("HERMITE_B200_PRECISION");
        if (!s || !*s) return HB_GRAVITY_PRECISION;
        if (!std::strcmp(s, "mixed")) return HB_MIXED;
        if (!std::strcmp(s, "fp64")) return HB_FP64;
        std::fprintf(stderr, "hermite_b200: HERMITE_B200_PRECISION=%s (want fp64|mixed)\n", s);
        std::abort();
    }

    explicit Gravity(const int _nbody) : nbody(_nbody), ctx(nullptr)
    {
        static_assert(sizeof(Force) == sizeof(double) * NFORCE, "Force layout");
        check(nullptr, hb_create(ORDER, nbody, precision_from_env(), &ctx), "hb_create");
    }
    ~Gravity() { hb_destroy(ctx); }
    Gravity(const Gravity &) = delete;
    Gravity &operator=(const Gravity &) = delete;

    // Safe from several OpenMP threads on distinct addr.
    void set_jp(const int addr, const Particle &p)
    {
        // acc, jrk [, snp, crk [, d4a, d5a]] are consecutive dvec3 members
        check(ctx, hb_set_jp(ctx, addr, &p.pos.x, p.mass, &p.vel.x, p.tlast, &p.acc.x),
              "set_jp");
    }

    void predict_all(const double tsys) { check(ctx, hb_predict_all(ctx, tsys), "predict_all"); }

    void calc_force_on_first_nact(const int nact, const double eps2, Force force[])
    {
        check(ctx, hb_force_first_nact(ctx, nact, eps2, reinterpret_cast<double *>(force)),
              "calc_force_on_first_nact");
    }

    void calc_potential(const double eps2, double potbuf[])
    {
        check(ctx, hb_potential(ctx, eps2, potbuf), "calc_potential");
    }

    // -DFAST_OMP_SYNC builds of the integrator call these from every thread of
    // one OpenMP parallel region (SRC/nbodysystem.h:767-838), as the CPU
    // backends provide them (SRC/hermite4-avx.h:9,155,404).  One thread drives
    // the GPU; the integrator's barrier after the prediction, and the barrier
    // here after the force, keep the others in step.  Above
    // NACT_PARALLEL_THRESH active particles the integrator spreads set_jp over
    // the threads, which set_jp allows for distinct slots; the thresholds are
    // the reference's AVX backends' (8 at 4th order, 12 at 6th and 8th:
    // SRC/hermite4-avx.h:9, SRC/hermite6-avx.h:9, SRC/hermite8-avx.h:10).
    enum { NACT_PARALLEL_THRESH = HB_GRAVITY_ORDER == 4 ? 8 : 12 };

    void predict_all_fast_omp(const double tsys)
    {
#pragma omp master
        predict_all(tsys);
    }

    void calc_force_on_first_nact_fast_omp(const int nact, const double eps2, Force force[])
    {
#pragma omp master
        calc_force_on_first_nact(nact, eps2, force);
#pragma omp barrier
    }
};
