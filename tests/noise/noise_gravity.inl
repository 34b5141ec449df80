// noise_gravity.inl -- TEST INFRASTRUCTURE ONLY: a CPU `struct Gravity` for
// the reference's own integrator (SRC/nbodysystem.h), used to measure how much
// force error its Hermite corrector and Aarseth step criterion tolerate.
//
// Forces come from the oracle (oracle/hermite_oracle.c: the FP64
// restatement of the reference's generic Gravity), then, by environment:
//   HB_NOISE_MODE=fp64      the oracle's FP64 force (default)
//   HB_NOISE_MODE=fp32pair  the mixed-precision kernel's pair arithmetic,
//                           restated in C float (fp32pair.h)
//   HB_NOISE_MODE=dr32      FP64 pair arithmetic except that the relative
//                           position is the mixed kernel's hi/lo FP32
//                           difference (one FP32 rounding per component)
//   HB_NOISE_REL=s          adds to each derivative vector of each force a
//                           seeded perturbation of relative size ~s
//                           (uniform sums, standard deviation s*|f_k| per
//                           component)
//   HB_NOISE_MAX_CALLS=n    exit(3) after n force calls: a run whose block
//                           steps blow up ends early
// Included by this directory's hermite{4,6,8}-titan.h, which SRC/hermite*.h
// include under -DCUDA_TITAN; the product path never uses it.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fp32pair.h"

extern "C" {
void oracle_predict(int order, int n, const double *rec, double tsys, double *pred);
void oracle_force(int order, int n, const double *pred, int nact, double eps2, double *force);
void oracle_potential(int order, int n, const double *rec, double eps2, double *pot);
}

struct Gravity {
    enum {
        ORDER = NOISE_GRAVITY_ORDER,
        NREC = 8 + 3 * (NOISE_GRAVITY_ORDER - 2),
        NPRED = 7 + 3 * (NOISE_GRAVITY_ORDER / 2 - 2),
        NFORCE = 3 * (NOISE_GRAVITY_ORDER / 2),
    };
    struct GParticle { double w[NREC]; };
    struct GPredictor { double w[NPRED]; };

    const int nbody;
    std::vector<double> rec, pred;
    bool fp32pair = false, dr32 = false;
    double rel = 0.0;
    long max_calls = 0, calls = 0;

    static double env_num(const char *k, double d)
    {
        const char *s = std::getenv(k);
        return s && *s ? std::atof(s) : d;
    }

    explicit Gravity(int n) : nbody(n), rec((size_t)n * NREC), pred((size_t)n * NPRED)
    {
        const char *m = std::getenv("HB_NOISE_MODE");
        fp32pair = m && !std::strcmp(m, "fp32pair");
        dr32 = m && !std::strcmp(m, "dr32");
        rel = env_num("HB_NOISE_REL", 0.0);
        max_calls = (long)env_num("HB_NOISE_MAX_CALLS", 0);
    }

    void set_jp(int addr, const Particle &p)
    {
        double *r = &rec[(size_t)addr * NREC];
        r[0] = p.pos.x; r[1] = p.pos.y; r[2] = p.pos.z; r[3] = p.mass;
        r[4] = p.vel.x; r[5] = p.vel.y; r[6] = p.vel.z; r[7] = p.tlast;
        std::memcpy(r + 8, &p.acc.x, sizeof(double) * 3 * (ORDER - 2));
    }

    void predict_all(double tsys) { oracle_predict(ORDER, nbody, rec.data(), tsys, pred.data()); }

    // FP64 pair arithmetic (the oracle's algebra, SRC/hermite4.h:342-357,
    // SRC/hermite6.h:332-360, SRC/hermite8.h:385-425) on a relative position
    // formed as the mixed kernel forms it: ((xj_hi - xi_hi) + (xj_lo - xi_lo))
    // in FP32.
    void force_dr32(int i, double eps2, double *f) const
    {
        const double *pi = &pred[(size_t)i * NPRED];
        for (int c = 0; c < NFORCE; ++c) f[c] = 0.0;
        for (int j = 0; j < nbody; ++j) {
            const double *pj = &pred[(size_t)j * NPRED];
            double dr[3], dv[3], da[3] = {0, 0, 0}, dj[3] = {0, 0, 0};
            for (int k = 0; k < 3; ++k) {
                const float hj = (float)pj[k], hi = (float)pi[k];
                const float lj = (float)(pj[k] - (double)hj), li = (float)(pi[k] - (double)hi);
                dr[k] = (double)((hj - hi) + (lj - li));
                dv[k] = pj[4 + k] - pi[4 + k];
                if (ORDER >= 6) da[k] = pj[7 + k] - pi[7 + k];
                if (ORDER >= 8) dj[k] = pj[10 + k] - pi[10 + k];
            }
            const double r2 = eps2 + dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
            const double rv = dr[0] * dv[0] + dr[1] * dv[1] + dr[2] * dv[2];
            const double ri2 = 1.0 / r2, mr3 = pj[3] * ri2 * std::sqrt(ri2), al = rv * ri2;
            double t[3], u[3];
            for (int k = 0; k < 3; ++k) {
                t[k] = dv[k] - 3.0 * al * dr[k];
                f[k] += mr3 * dr[k];
                f[3 + k] += mr3 * t[k];
            }
            if (ORDER >= 6) {
                const double vv = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
                const double ra = dr[0] * da[0] + dr[1] * da[1] + dr[2] * da[2];
                const double be = (vv + ra) * ri2 + al * al;
                for (int k = 0; k < 3; ++k) {
                    u[k] = da[k] - 6.0 * al * t[k] - 3.0 * be * dr[k];
                    f[6 + k] += mr3 * u[k];
                }
                if (ORDER >= 8) {
                    const double va = dv[0] * da[0] + dv[1] * da[1] + dv[2] * da[2];
                    const double rj = dr[0] * dj[0] + dr[1] * dj[1] + dr[2] * dj[2];
                    const double ga = (3.0 * va + rj) * ri2 + al * (3.0 * be - 4.0 * al * al);
                    for (int k = 0; k < 3; ++k)
                        f[9 + k] += mr3 * (dj[k] - 9.0 * al * u[k] - 9.0 * be * t[k] - 3.0 * ga * dr[k]);
                }
            }
        }
    }

    // Uniform sums (4 terms) scaled to standard deviation rel*|f_k| per
    // component; xorshift64 seeded by the call count and the slot.
    void perturb(int i, double *f) const
    {
        unsigned long long st = 0x9E3779B97F4A7C15ull ^ ((unsigned long long)calls << 20) ^ (unsigned long long)i;
        for (int q = 0; q < NFORCE / 3; ++q) {
            const double *v = f + 3 * q;
            const double nrm = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
            for (int k = 0; k < 3; ++k) {
                double u = 0.0;
                for (int r = 0; r < 4; ++r) {
                    st ^= st << 13; st ^= st >> 7; st ^= st << 17;
                    u += (double)(st >> 11) * (1.0 / 9007199254740992.0) - 0.5;
                }
                f[3 * q + k] += rel * nrm * u * std::sqrt(3.0);
            }
        }
    }

    void calc_force_on_first_nact(int nact, double eps2, Force force[])
    {
        if (max_calls > 0 && calls >= max_calls) {
            std::fprintf(stderr, "noise_gravity: %ld force calls, stopping\n", calls);
            std::fflush(stdout);
            std::exit(3);
        }
        double *out = reinterpret_cast<double *>(force);
        if (fp32pair) {
#pragma omp parallel for schedule(dynamic, 8)
            for (int i = 0; i < nact; ++i)
                fp32pair_force_one(ORDER, nbody, pred.data(), i, (float)eps2, 0, out + (size_t)i * NFORCE);
        } else if (dr32) {
#pragma omp parallel for schedule(dynamic, 8)
            for (int i = 0; i < nact; ++i) force_dr32(i, eps2, out + (size_t)i * NFORCE);
        } else {
            oracle_force(ORDER, nbody, pred.data(), nact, eps2, out);
        }
        if (rel > 0.0) {
#pragma omp parallel for schedule(static)
            for (int i = 0; i < nact; ++i) perturb(i, out + (size_t)i * NFORCE);
        }
        ++calls;
    }

    void calc_potential(double eps2, double potbuf[])
    {
        oracle_potential(ORDER, nbody, rec.data(), eps2, potbuf);
    }
};
