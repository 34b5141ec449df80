// hb_dump.cu -- checkpoints in the reference's dump format (host only).
//
// File layout (NbodySystem::dump / restore, SRC/nbodysystem.h:405-446):
//   "%d %d\n%ld\n%20.16f\n"   order, dumpid, nbody, tsys
//   "%A %A\n"                 initial and previous total energy
//   "%ld %ld\n"               particle steps and block steps so far
//   one line per particle (Particle::dump, SRC/hermite4.h:45-54,
//   SRC/hermite6.h:49-60, SRC/hermite8.h:61-74):
//   "%8ld %A" id, mass, then "   %A %A %A" for pos vel acc jrk snp crk
//   [d4a d5a [d6a d7a]] -- order + 2 vectors.
// tlast is not stored: a dump is taken when every particle is at tsys, and
// the restore sets tlast = tsys.  Our j-particle records hold pos mass vel
// tlast acc jrk [snp crk [d4a d5a]]; the two higher vectors the corrector
// derives on top of them (snp crk at 4th order, d4a d5a at 6th, d6a d7a at
// 8th) travel in a separate 6-double "aux" row per particle.
#include <cmath>
#include <cstdio>

#include "hermite_b200.h"
#include "hb_internal.h"

namespace hb {

namespace {
double norm2h(const double *a) { return a[0] * a[0] + a[1] * a[1] + a[2] * a[2]; }
}  // namespace

// Particle::recalc_dt (SRC/hermite4.h:95-116, SRC/hermite6.h:109-134,
// SRC/hermite8.h:136-164): the unquantised Aarseth step from the stored
// derivatives, then dtmax halved while it exceeds it.  Host arithmetic in the
// reference's order ((x*x + y*y) + z*z; sqrt and pow of the C library).
double recalc_dt(int order, const double *rec, const double *aux, double eta, double dtmax)
{
    const double *acc = rec + 8, *jrk = rec + 11;
    double dta;
    if (order == 4) {
        const double s0 = norm2h(acc), s1 = norm2h(jrk), s2 = norm2h(aux), s3 = norm2h(aux + 3);
        const double u = std::sqrt(s0 * s2) + s1;
        const double l = std::sqrt(s1 * s3) + s2;
        dta = eta * std::sqrt(u / l);
    } else if (order == 6) {
        const double *snp = rec + 14, *crk = rec + 17;
        const double s0 = norm2h(acc), s1 = norm2h(jrk), s2 = norm2h(snp);
        const double s3 = norm2h(crk), s4 = norm2h(aux), s5 = norm2h(aux + 3);
        const double u = std::sqrt(s0 * s2) + s1;
        const double l = std::sqrt(s3 * s5) + s4;
        dta = eta * std::pow(u / l, 1. / 6.);
    } else {
        const double *snp = rec + 14, *d5a = rec + 23;
        const double s0 = norm2h(acc), s1 = norm2h(jrk), s2 = norm2h(snp);
        const double s5 = norm2h(d5a), s6 = norm2h(aux), s7 = norm2h(aux + 3);
        const double u = std::sqrt(s0 * s2) + s1;
        const double l = std::sqrt(s5 * s7) + s6;
        dta = eta * std::pow(u / l, 1. / 10.);
    }
    double dt = dtmax;
    while (dt > dta) dt *= 0.5;
    return dt;
}

}  // namespace hb

using hb::kAuxWords;

extern "C" {

int hb_dump_write(const char *path, int order, int dumpid, int nbody, double tsys,
                  double init_energy, double prev_energy, long long steps, long long block_steps,
                  const long long *ids, const double *records, const double *aux)
{
    if (!path || (order != 4 && order != 6 && order != 8) || nbody < 0 ||
        (nbody > 0 && (!records || !aux)))
        return HB_ERR_INVALID;
    FILE *fp = std::fopen(path, "w");
    if (!fp) return HB_ERR_IO;
    const int R = 8 + 3 * (order - 2);
    std::fprintf(fp, "%d %d\n%ld\n%20.16f\n", order, dumpid, (long)nbody, tsys);
    std::fprintf(fp, "%A %A\n", init_energy, prev_energy);
    std::fprintf(fp, "%ld %ld\n", (long)steps, (long)block_steps);
    for (int i = 0; i < nbody; ++i) {
        const double *r = records + (size_t)i * R, *x = aux + (size_t)i * kAuxWords;
        std::fprintf(fp, "%8ld %A", (long)(ids ? ids[i] : i), r[3]);
        std::fprintf(fp, "   %A %A %A", r[0], r[1], r[2]);
        std::fprintf(fp, "   %A %A %A", r[4], r[5], r[6]);
        for (int k = 8; k < R; k += 3) std::fprintf(fp, "   %A %A %A", r[k], r[k + 1], r[k + 2]);
        std::fprintf(fp, "   %A %A %A", x[0], x[1], x[2]);
        std::fprintf(fp, "   %A %A %A", x[3], x[4], x[5]);
        std::fprintf(fp, "\n");
    }
    const bool ok = !std::ferror(fp);
    return (std::fclose(fp) == 0 && ok) ? HB_OK : HB_ERR_IO;
}

int hb_dump_read_header(const char *path, int *order, int *dumpid, int *nbody, double *tsys,
                        double *init_energy, double *prev_energy, long long *steps,
                        long long *block_steps)
{
    if (!path) return HB_ERR_INVALID;
    FILE *fp = std::fopen(path, "r");
    if (!fp) return HB_ERR_IO;
    int o = 0, d = 0;
    long n = 0, st = 0, bs = 0;
    double t = 0.0, e0 = 0.0, e1 = 0.0;
    const bool ok = std::fscanf(fp, "%d %d %ld %lf", &o, &d, &n, &t) == 4 &&
                    std::fscanf(fp, "%lA %lA", &e0, &e1) == 2 &&
                    std::fscanf(fp, "%ld %ld", &st, &bs) == 2;
    std::fclose(fp);
    if (!ok || n < 0 || n > (1L << 30)) return HB_ERR_IO;
    if (order) *order = o;
    if (dumpid) *dumpid = d;
    if (nbody) *nbody = (int)n;
    if (tsys) *tsys = t;
    if (init_energy) *init_energy = e0;
    if (prev_energy) *prev_energy = e1;
    if (steps) *steps = st;
    if (block_steps) *block_steps = bs;
    return HB_OK;
}

int hb_dump_read(const char *path, int order, int nbody, long long *ids, double *records,
                 double *aux)
{
    if (!path || (order != 4 && order != 6 && order != 8) || nbody < 0 ||
        (nbody > 0 && (!records || !aux)))
        return HB_ERR_INVALID;
    FILE *fp = std::fopen(path, "r");
    if (!fp) return HB_ERR_IO;
    int o = 0, d = 0;
    long n = 0, st = 0, bs = 0;
    double t = 0.0, e0 = 0.0, e1 = 0.0;
    bool ok = std::fscanf(fp, "%d %d %ld %lf", &o, &d, &n, &t) == 4 &&
              std::fscanf(fp, "%lA %lA", &e0, &e1) == 2 && std::fscanf(fp, "%ld %ld", &st, &bs) == 2 &&
              o == order && n == nbody;
    const int R = 8 + 3 * (order - 2);
    for (int i = 0; ok && i < nbody; ++i) {
        double *r = records + (size_t)i * R, *x = aux + (size_t)i * kAuxWords;
        long id = 0;
        ok = std::fscanf(fp, "%ld %lA", &id, &r[3]) == 2 &&
             std::fscanf(fp, "%lA %lA %lA", &r[0], &r[1], &r[2]) == 3 &&
             std::fscanf(fp, "%lA %lA %lA", &r[4], &r[5], &r[6]) == 3;
        r[7] = t;
        for (int k = 8; ok && k < R; k += 3)
            ok = std::fscanf(fp, "%lA %lA %lA", &r[k], &r[k + 1], &r[k + 2]) == 3;
        ok = ok && std::fscanf(fp, "%lA %lA %lA", &x[0], &x[1], &x[2]) == 3 &&
             std::fscanf(fp, "%lA %lA %lA", &x[3], &x[4], &x[5]) == 3;
        if (ids) ids[i] = id;
    }
    std::fclose(fp);
    return ok ? HB_OK : HB_ERR_IO;
}

}  // extern "C"
