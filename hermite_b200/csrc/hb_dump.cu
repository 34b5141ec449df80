// hb_dump.cu -- checkpoints and snapshots in the reference's file formats
// (host only).
//
// File layout (NbodySystem::dump / restore, SRC/nbodysystem.h:405-446):
//   "%d %d\n%ld\n%20.16f\n"   order, dumpid, nbody, tsys
//   "%A %A\n"                 initial and previous total energy
//   "%ld %ld\n"               particle steps and block steps so far
//   one line per particle (Particle::dump, SRC/hermite4.h:45-54,
//   SRC/hermite6.h:49-60, SRC/hermite8.h:61-74):
//   "%8ld %A" id, mass, then "   %A %A %A" for pos vel acc jrk snp crk
//   [d4a d5a [d6a d7a]] -- order + 2 vectors.
// Order code 9 is the 8th order with double-double positions
// (SRC/hermite8dd.h:79-114): the header says order 8 and the low part of the
// position follows the high part (posH posL vel acc ... d7a, 11 vectors).
// tlast is not stored: a dump is taken when every particle is at tsys, and
// the restore sets tlast = tsys.  Our j-particle records hold pos mass vel
// tlast acc jrk [snp crk [d4a d5a]]; the two higher vectors the corrector
// derives on top of them (snp crk at 4th order, d4a d5a at 6th, d6a d7a at
// 8th) travel in a separate 6-double "aux" row per particle.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "hermite_b200.h"
#include "hb_common.cuh"
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
    if (!path || (order != 4 && order != 6 && order != 8 && order != 9) || nbody < 0 ||
        (nbody > 0 && (!records || !aux)))
        return HB_ERR_INVALID;
    FILE *fp = std::fopen(path, "w");
    if (!fp) return HB_ERR_IO;
    const int R = 8 + 3 * (order - 2);
    const int Rd = order == 9 ? hb::kRecPosL : R;   // end of the derivative words
    std::fprintf(fp, "%d %d\n%ld\n%20.16f\n", order == 9 ? 8 : order, dumpid, (long)nbody, tsys);
    std::fprintf(fp, "%A %A\n", init_energy, prev_energy);
    std::fprintf(fp, "%ld %ld\n", (long)steps, (long)block_steps);
    for (int i = 0; i < nbody; ++i) {
        const double *r = records + (size_t)i * R, *x = aux + (size_t)i * kAuxWords;
        std::fprintf(fp, "%8ld %A", (long)(ids ? ids[i] : i), r[3]);
        std::fprintf(fp, "   %A %A %A", r[0], r[1], r[2]);
        if (order == 9)
            std::fprintf(fp, "   %A %A %A", r[hb::kRecPosL], r[hb::kRecPosL + 1], r[hb::kRecPosL + 2]);
        std::fprintf(fp, "   %A %A %A", r[4], r[5], r[6]);
        for (int k = 8; k < Rd; k += 3) std::fprintf(fp, "   %A %A %A", r[k], r[k + 1], r[k + 2]);
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
    if (!path || (order != 4 && order != 6 && order != 8 && order != 9) || nbody < 0 ||
        (nbody > 0 && (!records || !aux)))
        return HB_ERR_INVALID;
    FILE *fp = std::fopen(path, "r");
    if (!fp) return HB_ERR_IO;
    int o = 0, d = 0;
    long n = 0, st = 0, bs = 0;
    double t = 0.0, e0 = 0.0, e1 = 0.0;
    bool ok = std::fscanf(fp, "%d %d %ld %lf", &o, &d, &n, &t) == 4 &&
              std::fscanf(fp, "%lA %lA", &e0, &e1) == 2 && std::fscanf(fp, "%ld %ld", &st, &bs) == 2 &&
              o == (order == 9 ? 8 : order) && n == nbody;
    const int R = 8 + 3 * (order - 2);
    const int Rd = order == 9 ? hb::kRecPosL : R;
    for (int i = 0; ok && i < nbody; ++i) {
        double *r = records + (size_t)i * R, *x = aux + (size_t)i * kAuxWords;
        long id = 0;
        ok = std::fscanf(fp, "%ld %lA", &id, &r[3]) == 2 &&
             std::fscanf(fp, "%lA %lA %lA", &r[0], &r[1], &r[2]) == 3;
        if (ok && order == 9)
            ok = std::fscanf(fp, "%lA %lA %lA", &r[hb::kRecPosL], &r[hb::kRecPosL + 1],
                             &r[hb::kRecPosL + 2]) == 3;
        ok = ok && std::fscanf(fp, "%lA %lA %lA", &r[4], &r[5], &r[6]) == 3;
        r[7] = t;
        for (int k = 8; ok && k < Rd; k += 3)
            ok = std::fscanf(fp, "%lA %lA %lA", &r[k], &r[k + 1], &r[k + 2]) == 3;
        ok = ok && std::fscanf(fp, "%lA %lA %lA", &x[0], &x[1], &x[2]) == 3 &&
             std::fscanf(fp, "%lA %lA %lA", &x[3], &x[4], &x[5]) == 3;
        if (ids) ids[i] = id;
    }
    std::fclose(fp);
    return ok ? HB_OK : HB_ERR_IO;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Snapshots in the reference's text format (NbodySystem::read_snapshot_masaki
// and write_snapshot_masaki, SRC/nbodysystem.h:359-403): "%d\n%ld\n%f\n"
// (snapid, nbody, time), then per particle "%6ld    %A    %A %A %A    %A %A %A
// %A" (id, mass, pos, vel, potential).  Large files are the start-up cost of
// big runs, so both directions work on the whole file in memory and split the
// particle lines over host threads.

namespace {

bool slurp(const char *path, std::string &buf)
{
    FILE *fp = std::fopen(path, "rb");
    if (!fp) return false;
    std::fseek(fp, 0, SEEK_END);
    const long sz = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    if (sz < 0) {
        std::fclose(fp);
        return false;
    }
    buf.resize((size_t)sz);
    const size_t got = sz ? std::fread(&buf[0], 1, (size_t)sz, fp) : 0;
    std::fclose(fp);
    return got == (size_t)sz;
}

// Position after the header's three tokens; -1 if malformed.
long parse_snap_header(const std::string &buf, int *snapid, long *n, double *t)
{
    const char *p = buf.c_str();
    char *e = nullptr;
    const long sid = std::strtol(p, &e, 10);
    if (e == p) return -1;
    p = e;
    const long nb = std::strtol(p, &e, 10);
    if (e == p || nb < 0) return -1;
    p = e;
    const double tt = std::strtod(p, &e);
    if (e == p) return -1;
    *snapid = (int)sid;
    *n = nb;
    *t = tt;
    return (long)(e - buf.c_str());
}

}  // namespace

extern "C" {

int hb_snapshot_read_header(const char *path, int *snapid, int *nbody, double *tsys)
{
    if (!path) return HB_ERR_INVALID;
    FILE *fp = std::fopen(path, "r");
    if (!fp) return HB_ERR_IO;
    int sid = 0;
    long n = 0;
    double t = 0.0;
    const bool ok = std::fscanf(fp, "%d %ld %lf", &sid, &n, &t) == 3;
    std::fclose(fp);
    if (!ok || n < 0 || n > (1L << 30)) return HB_ERR_IO;
    if (snapid) *snapid = sid;
    if (nbody) *nbody = (int)n;
    if (tsys) *tsys = t;
    return HB_OK;
}

int hb_snapshot_read(const char *path, int nbody, long long *ids, double *mass, double *pos,
                     double *vel, double *pot)
{
    if (!path || nbody < 0 || (nbody > 0 && (!mass || !pos || !vel))) return HB_ERR_INVALID;
    std::string buf;
    if (!slurp(path, buf)) return HB_ERR_IO;
    int sid;
    long n;
    double t;
    const long body = parse_snap_header(buf, &sid, &n, &t);
    if (body < 0 || n != nbody) return HB_ERR_IO;
    // line starts of the particle records
    std::vector<long> start;
    start.reserve((size_t)nbody + 1);
    long p = body;
    const long len = (long)buf.size();
    while (p < len && (int)start.size() < nbody) {
        while (p < len && (buf[p] == '\n' || buf[p] == '\r' || buf[p] == ' ' || buf[p] == '\t')) ++p;
        if (p >= len) break;
        start.push_back(p);
        while (p < len && buf[p] != '\n') ++p;
    }
    if ((int)start.size() != nbody) return HB_ERR_IO;
    int bad = 0;
    const char *base = buf.c_str();
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int i = 0; i < nbody; ++i) {
        const char *q = base + start[i];
        char *e = nullptr;
        const long long id = std::strtoll(q, &e, 10);
        bad |= e == q;
        q = e;
        double v[8];
        for (int k = 0; k < 8; ++k) {
            v[k] = std::strtod(q, &e);
            bad |= e == q;
            q = e;
        }
        if (ids) ids[i] = id;
        mass[i] = v[0];
        for (int k = 0; k < 3; ++k) {
            pos[3 * (size_t)i + k] = v[1 + k];
            vel[3 * (size_t)i + k] = v[4 + k];
        }
        if (pot) pot[i] = v[7];
    }
    return bad ? HB_ERR_IO : HB_OK;
}

int hb_snapshot_write(const char *path, int snapid, int nbody, double tsys, const long long *ids,
                      const double *mass, const double *pos, const double *vel, const double *pot)
{
    if (!path || nbody < 0 || (nbody > 0 && (!mass || !pos || !vel))) return HB_ERR_INVALID;
    FILE *fp = std::fopen(path, "w");
    if (!fp) return HB_ERR_IO;
    std::fprintf(fp, "%d\n%ld\n%f\n", snapid, (long)nbody, tsys);
    constexpr int kBlock = 4096;   // particles formatted per task
    const int nblk = (nbody + kBlock - 1) / kBlock;
    std::vector<std::string> out((size_t)nblk);
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < nblk; ++b) {
        std::string &s = out[b];
        char line[512];
        const int i1 = std::min(nbody, (b + 1) * kBlock);
        for (int i = b * kBlock; i < i1; ++i) {
            const double *x = pos + 3 * (size_t)i, *v = vel + 3 * (size_t)i;
            const int m = std::snprintf(line, sizeof line, "%6ld    %A    %A %A %A    %A %A %A    %A\n",
                                        (long)(ids ? ids[i] : i), mass[i], x[0], x[1], x[2], v[0],
                                        v[1], v[2], pot ? pot[i] : 0.0);
            s.append(line, (size_t)m);
        }
    }
    bool ok = true;
    for (const std::string &s : out) ok = ok && std::fwrite(s.data(), 1, s.size(), fp) == s.size();
    ok = ok && !std::ferror(fp);
    return (std::fclose(fp) == 0 && ok) ? HB_OK : HB_ERR_IO;
}

}  // extern "C"
