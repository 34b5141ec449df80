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
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>
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


// ---------------------------------------------------------------------------
// "%A" text both ways, for files of millions of particles: the whole file is
// read into memory, particle lines are split over host threads, and the
// number forms that printf("%A") writes are converted by exact fast paths,
// with the C library (strtod, snprintf) for any other text.

namespace {

// A whole file in memory, NUL-terminated (the parsers stop there).
struct Text {
    std::unique_ptr<char[]> data;   // not zero-filled
    size_t size = 0;
    const char *c_str() const { return data.get(); }
};

bool slurp(const char *path, Text &buf)
{
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) return false;
    struct stat st;
    if (::fstat(fd, &st) != 0 || st.st_size < 0) {
        ::close(fd);
        return false;
    }
    const size_t sz = (size_t)st.st_size;
    buf.data.reset(new char[sz + 1]);
    buf.size = sz;
    buf.data[sz] = '\0';
    // ranges of at least 8 MiB read by host threads in parallel
    constexpr size_t kPart = (size_t)8 << 20;
    const int nt = (int)std::max<size_t>(1, std::min<size_t>(8, sz / kPart));
    const size_t per = (sz + nt - 1) / nt;
    int bad = 0;
#pragma omp parallel for num_threads(nt) schedule(static, 1) reduction(| : bad)
    for (int t = 0; t < nt; ++t) {
        size_t o = (size_t)t * per;
        const size_t e = std::min(sz, o + per);
        while (o < e) {
            const ssize_t got = ::pread(fd, buf.data.get() + o, e - o, (off_t)o);
            if (got <= 0) {
                bad = 1;
                break;
            }
            o += (size_t)got;
        }
    }
    ::close(fd);
    return !bad;
}

inline bool is_blank(char c)
{
    return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f';
}

struct HexTable {
    signed char v[256];
    HexTable()
    {
        for (int c = 0; c < 256; ++c) v[c] = -1;
        for (int c = 0; c < 10; ++c) v['0' + c] = (signed char)c;
        for (int c = 0; c < 6; ++c) v['A' + c] = v['a' + c] = (signed char)(10 + c);
    }
};
const HexTable kHex;

inline int hexdigit(char c) { return kHex.v[(unsigned char)c]; }

// The finite forms printf("%A") writes: [-]0X1[.h..h]P(+|-)d for normal
// numbers, [-]0X0.h..hP-1022 for subnormals and [-]0X0P+0 for zero, with at
// most 13 fraction digits.  These digits are the IEEE fraction bits and the
// exponent the unbiased one, so the double is assembled bit for bit, exactly.
// Returns the end of the number,
// or nullptr for any other text (decimal, more digits, NAN, INF, a leading 1
// with an exponent outside the normal range), which is left to strtod.
const char *parse_hexA(const char *p, double *out)
{
    const bool neg = *p == '-';
    if (neg || *p == '+') ++p;
    if (p[0] != '0' || (p[1] != 'X' && p[1] != 'x')) return nullptr;
    p += 2;
    const int lead = *p - '0';
    if (lead != 0 && lead != 1) return nullptr;
    ++p;
    uint64_t mant = (uint64_t)lead;
    int nd = 0;
    if (*p == '.') {
        ++p;
        for (int d; (d = hexdigit(*p)) >= 0; ++p) {
            if (++nd > 13) return nullptr;
            mant = (mant << 4) | (uint64_t)d;
        }
    }
    if (*p != 'P' && *p != 'p') return nullptr;
    ++p;
    const bool eneg = *p == '-';
    if (eneg || *p == '+') ++p;
    if (*p < '0' || *p > '9') return nullptr;
    int ex = 0;
    for (; *p >= '0' && *p <= '9'; ++p) {
        ex = ex * 10 + (*p - '0');
        if (ex > 100000) return nullptr;
    }
    if (eneg) ex = -ex;
    if (mant == 0) {
        *out = neg ? -0.0 : 0.0;
        return p;
    }
    if (lead == 1 ? (ex < -1022 || ex > 1023) : ex != -1022) return nullptr;
    // the IEEE encoding directly: the fraction digits left-aligned in 52 bits
    // under the biased exponent (0 for subnormals)
    const uint64_t frac = (mant & ((1ull << (4 * nd)) - 1)) << (52 - 4 * nd);
    const uint64_t bits = ((uint64_t)neg << 63) | ((uint64_t)(lead ? ex + 1023 : 0) << 52) | frac;
    std::memcpy(out, &bits, sizeof bits);
    return p;
}

// The next number after blanks: the exact fast path, else strtod.
inline bool next_double(const char *&p, double *v)
{
    while (is_blank(*p)) ++p;
    if (const char *e = parse_hexA(p, v)) {
        p = e;
        return true;
    }
    char *e = nullptr;
    *v = std::strtod(p, &e);
    if (e == p) return false;
    p = e;
    return true;
}

inline bool next_long(const char *&p, long long *v)
{
    while (is_blank(*p)) ++p;
    char *e = nullptr;
    *v = std::strtoll(p, &e, 10);
    if (e == p) return false;
    p = e;
    return true;
}

// nbody records of an integer and nv numbers each, from buf[body] on, into
// ids[i] (if ids) and vals[i * nv + k].  With one record per line (as every
// writer of these formats lays them out) the lines are parsed in parallel;
// any other layout is read token by token, as fscanf would.
bool parse_records(const Text &buf, size_t body, int nbody, int nv, long long *ids,
                   double *vals)
{
    const char *base = buf.c_str();
    const size_t len = buf.size;
    std::vector<size_t> start, end;
    start.reserve((size_t)nbody);
    end.reserve((size_t)nbody);
    for (size_t p = body; p < len && (int)start.size() < nbody;) {
        while (p < len && is_blank(base[p])) ++p;
        if (p >= len) break;
        const void *nl = std::memchr(base + p, '\n', len - p);
        const size_t e = nl ? (size_t)(static_cast<const char *>(nl) - base) : len;
        start.push_back(p);
        end.push_back(e);
        p = e;
    }
    bool lines_ok = (int)start.size() == nbody;
    if (lines_ok) {
        int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
        for (int i = 0; i < nbody; ++i) {
            const char *q = base + start[i], *lim = base + end[i];
            long long id = 0;
            bool ok = next_long(q, &id);
            double *v = vals + (size_t)i * nv;
            for (int k = 0; ok && k < nv; ++k) ok = next_double(q, &v[k]);
            ok = ok && q <= lim;
            while (ok && q < lim) ok = is_blank(*q++);
            if (ids) ids[i] = id;
            bad |= !ok;
        }
        lines_ok = bad == 0;
    }
    if (lines_ok) return true;
    const char *q = base + body;
    for (int i = 0; i < nbody; ++i) {
        long long id = 0;
        if (!next_long(q, &id)) return false;
        if (ids) ids[i] = id;
        for (int k = 0; k < nv; ++k)
            if (!next_double(q, &vals[(size_t)i * nv + k])) return false;
    }
    return true;
}

// printf("%A") of x, character for character as the C library writes it:
// the fraction's hex digits without trailing zeros, subnormals as
// 0X0.h..hP-1022, zero as 0X0P+0, NAN and INF with their signs.
int put_hexA(double x, char *o)
{
    uint64_t b;
    std::memcpy(&b, &x, sizeof b);
    char *const s = o;
    if (b >> 63) *o++ = '-';
    const int eb = (int)((b >> 52) & 0x7ff);
    uint64_t f = b & ((1ull << 52) - 1);
    if (eb == 0x7ff) {
        std::memcpy(o, f ? "NAN" : "INF", 3);
        return (int)(o + 3 - s);
    }
    *o++ = '0';
    *o++ = 'X';
    *o++ = eb ? '1' : '0';
    const int e = eb ? eb - 1023 : (f ? -1022 : 0);
    if (f) {
        int nd = 13;
        while ((f & 0xf) == 0) {
            f >>= 4;
            --nd;
        }
        *o++ = '.';
        for (int k = nd - 1; k >= 0; --k) *o++ = "0123456789ABCDEF"[(f >> (4 * k)) & 0xf];
    }
    *o++ = 'P';
    *o++ = e < 0 ? '-' : '+';
    unsigned a = (unsigned)(e < 0 ? -e : e);
    char d[8];
    int n = 0;
    do {
        d[n++] = (char)('0' + a % 10);
        a /= 10;
    } while (a);
    while (n) *o++ = d[--n];
    return (int)(o - s);
}

// Formats lines [0, nbody) with line(i, out) -> bytes written (at most
// max_line), in blocks over host threads, and writes them in order.
template <typename LineFn>
bool write_lines(FILE *fp, int nbody, size_t max_line, LineFn line)
{
    constexpr int kBlock = 4096;   // lines formatted per task
    const int nblk = (nbody + kBlock - 1) / kBlock;
    std::vector<std::unique_ptr<char[]>> out((size_t)nblk);   // not zero-filled
    std::vector<size_t> used((size_t)nblk, 0);
#pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < nblk; ++b) {
        const int i0 = b * kBlock, i1 = std::min(nbody, i0 + kBlock);
        out[b].reset(new char[(size_t)(i1 - i0) * max_line]);
        char *o = out[b].get();
        size_t u = 0;
        for (int i = i0; i < i1; ++i) u += (size_t)line(i, o + u);
        used[b] = u;
    }
    bool ok = true;
    for (int b = 0; b < nblk; ++b) ok = ok && std::fwrite(out[b].get(), 1, used[b], fp) == used[b];
    return ok;
}

// "%<width>ld" of v.
constexpr size_t kMaxHexA = 24;   // "-0X1.FFFFFFFFFFFFFP-1022"
constexpr size_t kMaxId = 24;     // "%8lld" of any long long, with its NUL

inline int put_id(long long v, int width, char *o)
{
    return std::snprintf(o, 32, "%*lld", width, v);
}

// " "-separated groups of three: sep then "%A %A %A".
inline int put_vec(const char *sep, const double *v, char *o)
{
    char *const s = o;
    for (const char *c = sep; *c; ++c) *o++ = *c;
    o += put_hexA(v[0], o);
    *o++ = ' ';
    o += put_hexA(v[1], o);
    *o++ = ' ';
    o += put_hexA(v[2], o);
    return (int)(o - s);
}

}  // namespace

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
    const int ngroups = 2 + (order == 9 ? 1 : 0) + (Rd - 8) / 3 + 2;   // pos [posL] vel derivs aux
    const size_t max_line = kMaxId + 1 + kMaxHexA + (size_t)ngroups * (3 + 3 * kMaxHexA + 2) + 1;
    bool ok = write_lines(fp, nbody, max_line, [&](int i, char *o) {
        const double *r = records + (size_t)i * R, *x = aux + (size_t)i * kAuxWords;
        char *const s = o;
        o += put_id(ids ? ids[i] : i, 8, o);
        *o++ = ' ';
        o += put_hexA(r[3], o);
        o += put_vec("   ", r, o);
        if (order == 9) o += put_vec("   ", r + hb::kRecPosL, o);
        o += put_vec("   ", r + 4, o);
        for (int k = 8; k < Rd; k += 3) o += put_vec("   ", r + k, o);
        o += put_vec("   ", x, o);
        o += put_vec("   ", x + 3, o);
        *o++ = '\n';
        return (int)(o - s);
    });
    ok = ok && !std::ferror(fp);
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
    Text buf;
    if (!slurp(path, buf)) return HB_ERR_IO;
    // header: order dumpid / nbody / tsys / two energies / two step counts
    const char *p = buf.c_str();
    long long o = 0, d = 0, n = 0, st = 0, bs = 0;
    double t = 0.0, e0 = 0.0, e1 = 0.0;
    const bool hdr = next_long(p, &o) && next_long(p, &d) && next_long(p, &n) && next_double(p, &t) &&
                     next_double(p, &e0) && next_double(p, &e1) && next_long(p, &st) &&
                     next_long(p, &bs);
    if (!hdr || o != (order == 9 ? 8 : order) || n != nbody) return HB_ERR_IO;
    // per particle: id, then mass, pos, [posL], vel, the record's derivatives
    // and the two aux vectors, in file order
    const int R = 8 + 3 * (order - 2);
    const int Rd = order == 9 ? hb::kRecPosL : R;
    const int nv = 1 + 3 + (order == 9 ? 3 : 0) + 3 + (Rd - 8) + 6;
    std::unique_ptr<double[]> vals(new double[(size_t)nbody * nv]);   // not zero-filled
    std::vector<long long> idv(ids ? 0 : (size_t)nbody);
    if (!parse_records(buf, (size_t)(p - buf.c_str()), nbody, nv, ids ? ids : idv.data(), vals.get()))
        return HB_ERR_IO;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nbody; ++i) {
        const double *v = vals.get() + (size_t)i * nv;
        double *r = records + (size_t)i * R, *x = aux + (size_t)i * kAuxWords;
        r[3] = *v++;
        for (int k = 0; k < 3; ++k) r[k] = *v++;
        if (order == 9)
            for (int k = 0; k < 3; ++k) r[hb::kRecPosL + k] = *v++;
        for (int k = 4; k < 7; ++k) r[k] = *v++;
        r[7] = t;
        for (int k = 8; k < Rd; ++k) r[k] = *v++;
        for (int k = 0; k < kAuxWords; ++k) x[k] = *v++;
    }
    return HB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Snapshots in the reference's text format (NbodySystem::read_snapshot_masaki
// and write_snapshot_masaki, SRC/nbodysystem.h:359-403): "%d\n%ld\n%f\n"
// (snapid, nbody, time), then per particle "%6ld    %A    %A %A %A    %A %A %A
// %A" (id, mass, pos, vel, potential).  Large files are the start-up cost of
// big runs, so both directions work on the whole file in memory and split the
// particle lines over host threads.

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
    Text buf;
    if (!slurp(path, buf)) return HB_ERR_IO;
    const char *p = buf.c_str();
    long long sid = 0, n = 0;
    double t = 0.0;
    if (!(next_long(p, &sid) && next_long(p, &n) && next_double(p, &t)) || n != nbody)
        return HB_ERR_IO;
    constexpr int nv = 8;   // mass, pos, vel, potential
    std::unique_ptr<double[]> vals(new double[(size_t)nbody * nv]);   // not zero-filled
    std::vector<long long> idv(ids ? 0 : (size_t)nbody);
    if (!parse_records(buf, (size_t)(p - buf.c_str()), nbody, nv, ids ? ids : idv.data(), vals.get()))
        return HB_ERR_IO;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nbody; ++i) {
        const double *v = vals.get() + (size_t)i * nv;
        mass[i] = v[0];
        for (int k = 0; k < 3; ++k) {
            pos[3 * (size_t)i + k] = v[1 + k];
            vel[3 * (size_t)i + k] = v[4 + k];
        }
        if (pot) pot[i] = v[7];
    }
    return HB_OK;
}

int hb_snapshot_write(const char *path, int snapid, int nbody, double tsys, const long long *ids,
                      const double *mass, const double *pos, const double *vel, const double *pot)
{
    if (!path || nbody < 0 || (nbody > 0 && (!mass || !pos || !vel))) return HB_ERR_INVALID;
    FILE *fp = std::fopen(path, "w");
    if (!fp) return HB_ERR_IO;
    std::fprintf(fp, "%d\n%ld\n%f\n", snapid, (long)nbody, tsys);
    const size_t max_line = kMaxId + 4 + kMaxHexA + 2 * (4 + 3 * kMaxHexA + 2) + 4 + kMaxHexA + 1;
    bool ok = write_lines(fp, nbody, max_line, [&](int i, char *o) {
        char *const s = o;
        o += put_id(ids ? ids[i] : i, 6, o);
        for (int k = 0; k < 4; ++k) *o++ = ' ';
        o += put_hexA(mass[i], o);
        o += put_vec("    ", pos + 3 * (size_t)i, o);
        o += put_vec("    ", vel + 3 * (size_t)i, o);
        for (int k = 0; k < 4; ++k) *o++ = ' ';
        o += put_hexA(pot ? pot[i] : 0.0, o);
        *o++ = '\n';
        return (int)(o - s);
    });
    ok = ok && !std::ferror(fp);
    return (std::fclose(fp) == 0 && ok) ? HB_OK : HB_ERR_IO;
}

}  // extern "C"
