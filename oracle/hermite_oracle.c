/*
 * hermite_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Scalar FP64 CPU restatement of the reference's generic (backend-free)
 * force calculator, used as the parity checker for the CUDA path.  Only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark may load
 * this; the product path never calls it.
 *
 * Pinned against: (1) the reference's own generic and AVX `Gravity`, compiled
 * from its sources into oracle/_ref/ by oracle/Makefile and compared on the
 * same inputs (tests/test_oracle.py); (2) golden vectors made by that build
 * (tests/golden/, script tests/golden/make_golden.py).
 *
 * Data formats (shared with the C-ABI, include/hermite_b200.h):
 *   j-particle record, R = 8 + 3*(order-2) doubles:
 *     pos[3] mass vel[3] tlast acc[3] jrk[3] (snp[3] crk[3]) (d4a[3] d5a[3])
 *     -- the field order of the reference's CUDA GParticle
 *        (SRC/hermite4-titan.h:20-27, SRC/hermite6-titan.h:20-29,
 *         SRC/hermite8-titan.h:20-31).
 *   predicted record, P = 7 / 10 / 13 doubles:
 *     pos[3] mass vel[3] (acc[3]) (jrk[3])
 *   force record, F = 6 / 9 / 12 doubles:
 *     acc[3] jrk[3] (snp[3]) (crk[3])  -- the reference's `struct Force`
 *        (SRC/hermite4.h:4-14, SRC/hermite6.h:4-17, SRC/hermite8.h:8-24).
 */
#include <math.h>
#include <stddef.h>

/*
 * Order code 9 is the 8th order with double-double positions, the
 * reference's SRC/hermite8dd.h: the record is the 8th-order record followed
 * by posL[3] (29 doubles), the predicted record the 8th-order one (posH as
 * the position) followed by the predicted posL[3] (16 doubles).
 */
static int rec_words(int order)  { return 8 + 3 * (order - 2); }
static int pred_words(int order) { return 7 + 3 * (order / 2 - 2) + (order == 9 ? 3 : 0); }
static int force_words(int order){ return 3 * (order / 2); }

int oracle_record_words(int order)    { return rec_words(order); }
int oracle_predicted_words(int order) { return pred_words(order); }
int oracle_force_words(int order)     { return force_words(order); }

/*
 * Taylor predictor of every slot to tsys from its own tlast, nested (Horner)
 * as in the reference's generic GPredictor constructors:
 *   4th: SRC/hermite4.h:296-307   6th: SRC/hermite6.h:276-293
 *   8th: SRC/hermite8.h:323-346
 * c_k = dt / k; x(t) = x0 + dt*(v + c2*(a + c3*(j + c4*(s + ...)))).
 */
void oracle_predict(int order, int n, const double *rec, double tsys,
                    double *pred)
{
    const int R = rec_words(order), P = pred_words(order);
    for (int i = 0; i < n; i++) {
        const double *p = rec + (size_t)i * R;
        double *q = pred + (size_t)i * P;
        const double dt = tsys - p[7];
        const double c2 = (1. / 2.) * dt, c3 = (1. / 3.) * dt;
        const double c4 = (1. / 4.) * dt, c5 = (1. / 5.) * dt;
        const double c6 = (1. / 6.) * dt, c7 = (1. / 7.) * dt;
        /* derivative vectors: d[0]=vel, d[1]=acc, d[2]=jrk, ... */
        const double *pos = p + 0, *vel = p + 4, *acc = p + 8, *jrk = p + 11;
        for (int k = 0; k < 3; k++) {
            double x, v, a = 0, jj = 0;
            if (order == 4) {
                x = pos[k] + dt * (vel[k] + c2 * (acc[k] + c3 * jrk[k]));
                v = vel[k] + dt * (acc[k] + c2 * jrk[k]);
            } else if (order == 6) {
                const double s = p[14 + k], c = p[17 + k];
                x = pos[k] + dt * (vel[k] + c2 * (acc[k] + c3 * (jrk[k] + c4 * (s + c5 * c))));
                v = vel[k] + dt * (acc[k] + c2 * (jrk[k] + c3 * (s + c4 * c)));
                a = acc[k] + dt * (jrk[k] + c2 * (s + c3 * c));
            } else {
                const double s = p[14 + k], c = p[17 + k];
                const double d4 = p[20 + k], d5 = p[23 + k];
                /* order 9: posH unchanged, posL advanced (SRC/hermite8dd.h:304-306) */
                const double x0 = order == 9 ? p[26 + k] : pos[k];
                x = x0 + dt * (vel[k] + c2 * (acc[k] + c3 * (jrk[k] + c4 * (s + c5 * (c + c6 * (d4 + c7 * d5))))));
                v = vel[k] + dt * (acc[k] + c2 * (jrk[k] + c3 * (s + c4 * (c + c5 * (d4 + c6 * d5)))));
                a = acc[k] + dt * (jrk[k] + c2 * (s + c3 * (c + c4 * (d4 + c5 * d5))));
                jj = jrk[k] + dt * (s + c2 * (c + c3 * (d4 + c4 * d5)));
            }
            if (order == 9) {
                q[k] = pos[k];
                q[13 + k] = x;
            } else {
                q[k] = x;
            }
            q[4 + k] = v;
            if (order >= 6) q[7 + k] = a;
            if (order >= 8) q[10 + k] = jj;
        }
        q[3] = p[3];
    }
}

static inline double dot3(const double *a, const double *b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/*
 * Direct-summation force on slots [0,nact) from all slots [0,n), self pair
 * included (it is exactly zero because eps2 > 0 makes every difference 0).
 * Per-pair algebra as in the reference's generic kernels:
 *   4th: SRC/hermite4.h:342-357  (acc, jerk)
 *   6th: SRC/hermite6.h:332-360  (+ snap; alpha, beta)
 *   8th: SRC/hermite8.h:385-425  (+ crackle; gamma)
 * j is summed in ascending order in FP64.  The i-particles are shared out
 * over OpenMP threads (when built with -fopenmp); each i's sum stays a
 * single ascending loop, so the result does not depend on the thread count.
 */
void oracle_force(int order, int n, const double *pred, int nact, double eps2,
                  double *force)
{
    const int P = pred_words(order), F = force_words(order);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < nact; i++) {
        const double *pi = pred + (size_t)i * P;
        double f[12] = {0};
        for (int j = 0; j < n; j++) {
            const double *pj = pred + (size_t)j * P;
            double dr[3], dv[3], da[3] = {0, 0, 0}, dj[3] = {0, 0, 0};
            for (int k = 0; k < 3; k++) {
                /* order 9: (posHj - posHi) + (posLj - posLi), SRC/hermite8dd.h:358 */
                dr[k] = order == 9 ? (pj[k] - pi[k]) + (pj[13 + k] - pi[13 + k]) : pj[k] - pi[k];
                dv[k] = pj[4 + k] - pi[4 + k];
                if (order >= 6) da[k] = pj[7 + k] - pi[7 + k];
                if (order >= 8) dj[k] = pj[10 + k] - pi[10 + k];
            }
            const double r2 = eps2 + dot3(dr, dr);
            if (order == 9 && r2 == eps2) continue;   /* SRC/hermite8dd.h:362 */
            const double drdv = dot3(dr, dv);
            const double ri2 = 1.0 / r2;
            const double mri3 = pj[3] * ri2 * sqrt(ri2);
            if (order == 4) {
                const double alpha = -3.0 * drdv * ri2;
                for (int k = 0; k < 3; k++) {
                    f[k] += mri3 * dr[k];
                    f[3 + k] += mri3 * dv[k] + alpha * (mri3 * dr[k]);
                }
            } else {
                const double dvdv = dot3(dv, dv), drda = dot3(dr, da);
                const double alpha = drdv * ri2;
                const double beta = (dvdv + drda) * ri2 + alpha * alpha;
                double gamma = 0.0;
                if (order >= 8) {
                    const double dvda = dot3(dv, da), drdj = dot3(dr, dj);
                    gamma = (3.0 * dvda + drdj) * ri2
                          + alpha * (3.0 * beta - 4.0 * alpha * alpha);
                }
                for (int k = 0; k < 3; k++) {
                    f[k] += mri3 * dr[k];
                    const double t1 = dv[k] + (-3.0 * alpha) * dr[k];
                    f[3 + k] += mri3 * t1;
                    const double t2 = da[k] + (-6.0 * alpha) * t1 + (-3.0 * beta) * dr[k];
                    f[6 + k] += mri3 * t2;
                    if (order >= 8) {
                        const double t3 = dj[k] + (-9.0 * alpha) * t2
                                        + (-9.0 * beta) * t1 + (-3.0 * gamma) * dr[k];
                        f[9 + k] += mri3 * t3;
                    }
                }
            }
        }
        for (int k = 0; k < F; k++) force[(size_t)i * F + k] = f[k];
    }
}

/*
 * Softened potential phi_i = -sum_{j != i} m_j / sqrt(r^2 + eps2) on the
 * un-predicted positions (the j-particle records), self pair skipped by slot
 * index as the reference's CUDA kernel does (SRC/pot-titan.hu:1-18,80-129;
 * generic form SRC/hermite6.h:367-387).
 */
void oracle_potential(int order, int n, const double *rec, double eps2,
                      double *pot)
{
    const int R = rec_words(order);
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < n; i++) {
        const double *pi = rec + (size_t)i * R;
        double s = 0.0;
        for (int j = 0; j < n; j++) {
            if (j == i) continue;
            const double *pj = rec + (size_t)j * R;
            double dr[3] = {pj[0] - pi[0], pj[1] - pi[1], pj[2] - pi[2]};
            if (order == 9)   /* SRC/hermite8dd.h:405-407 */
                for (int k = 0; k < 3; k++) dr[k] = dr[k] + (pj[26 + k] - pi[26 + k]);
            const double r2 = eps2 + dot3(dr, dr);
            s -= pj[3] / sqrt(r2);
        }
        pot[i] = s;
    }
}
