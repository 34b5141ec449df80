"""The library's "%A" text conversions (snapshots and dumps, CPU) against the
C library they stand in for: every line the writer produces equals
snprintf's, and every number the reader parses equals strtod's, bit for bit,
over random bit patterns (normal, subnormal, signed zero, infinities, NaN
payloads) and over number forms no writer of these formats produces."""
import ctypes

import numpy as np
import pytest

import hermite_b200 as hb
from hermite_b200 import ic

LIBC = ctypes.CDLL("libc.so.6")
LIBC.strtod.restype = ctypes.c_double
LIBC.strtod.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]
SNAP_FMT = b"%6ld    %A    %A %A %A    %A %A %A    %A\n"


def c_line(fmt, ident, values):
    buf = ctypes.create_string_buffer(1024)
    n = LIBC.snprintf(buf, 1024, fmt, ctypes.c_long(int(ident)), *[ctypes.c_double(float(v)) for v in values])
    return buf.raw[:n].decode()


def random_doubles(rng, n):
    """Bit patterns from every exponent range, plus the special values."""
    bits = rng.integers(0, 2 ** 63, size=n, dtype=np.uint64) | (
        rng.integers(0, 2, size=n, dtype=np.uint64) << np.uint64(63))
    x = bits.view(np.float64).copy()
    k = n // 8
    x[:k] = rng.normal(size=k) * np.exp2(rng.integers(-1074, 1024, size=k).astype(float))
    x[k:2 * k] = (rng.integers(1, 2 ** 52, size=k, dtype=np.uint64)).view(np.float64)   # subnormals
    x[2 * k:2 * k + 8] = [0.0, -0.0, np.inf, -np.inf, np.nan, -np.nan, 5e-324, -1.7976931348623157e308]
    return x


def bits_equal(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    nan = np.isnan(a)
    return np.array_equal(nan, np.isnan(b)) and np.array_equal(a[~nan].view(np.uint64), b[~nan].view(np.uint64))


def test_snapshot_text_matches_c_library(tmp_path):
    rng = np.random.default_rng(11)
    n = 4000
    vals = random_doubles(rng, n * 8).reshape(n, 8)
    snap = ic.Snapshot(3, 0.5, rng.integers(-10 ** 9, 10 ** 9, size=n), vals[:, 0], vals[:, 1:4],
                       vals[:, 4:7], vals[:, 7])
    path = tmp_path / "s.dat"
    ic.write_snapshot(path, snap)
    lines = path.read_text().splitlines(keepends=True)
    assert lines[:3] == ["3\n", f"{n}\n", "0.500000\n"]
    for i in range(n):
        assert lines[3 + i] == c_line(SNAP_FMT, snap.ids[i], vals[i]), i
    back = ic.read_snapshot(path)
    assert np.array_equal(back.ids, snap.ids)
    for a, b in ((back.mass, snap.mass), (back.pos, snap.pos), (back.vel, snap.vel), (back.pot, snap.pot)):
        assert bits_equal(a, b)


@pytest.mark.parametrize("order", [4, 9])
def test_dump_text_matches_c_library(order, tmp_path):
    rng = np.random.default_rng(order)
    n, R = 500, hb.record_words(order)
    rec = random_doubles(rng, n * R).reshape(n, R)
    rec[:, 7] = 0.25
    aux = random_doubles(rng, n * hb.AUX_WORDS).reshape(n, hb.AUX_WORDS)
    ids = rng.integers(0, 10 ** 7, size=n)
    path = tmp_path / "d.dat"
    hb.write_dump(path, order, rec, aux, 0.25, dumpid=2, energies=(-0.25, -0.2500001), steps=(7, 3), ids=ids)
    lines = path.read_text().splitlines(keepends=True)
    pos_l = list(range(26, 29)) if order == 9 else []
    rd = 26 if order == 9 else R
    for i in range(n):
        cols = [3, 0, 1, 2] + pos_l + [4, 5, 6] + list(range(8, rd))
        v = [rec[i, c] for c in cols] + list(aux[i])
        fmt = b"%8ld %A" + b"   %A %A %A" * ((len(v) - 1) // 3) + b"\n"
        assert lines[5 + i] == c_line(fmt, ids[i], v), i
    d = hb.read_dump(path, dd=order == 9)
    assert bits_equal(d["records"], rec) and bits_equal(d["aux"], aux)
    assert np.array_equal(d["ids"], ids)


FORMS = ["0X1.8P+1", "0x1.8p+1", "-0X1.FFFFFFFFFFFFFP+1023", "0X0.0000000000001P-1022",
         "0X1.00000000000008P+0", "0X1.00000000000018P+0", "0X1.000000000000000P+0", "0X0.8P+0",
         "0X1P-1074", "0X1.8P-1075", "0X1P+1024", "+0X1P+0", "-0X0P+0", "0X0P+7", "0.125",
         "-1e-3", "3.14159265358979311599796346854", "1e-320", "INF", "-inf", "NAN", "-nan",
         "0X1.921FB54442D18P+1", "1.7976931348623157e308"]


def test_reader_handles_other_number_forms(tmp_path):
    """Text the library did not write: decimal, lowercase, more fraction
    digits (rounded), leading zeros, out-of-range exponents -- as strtod."""
    n = len(FORMS)
    body = "".join(f"{i} {f} {f} {f} {f} {f} {f} {f} {f}\n" for i, f in enumerate(FORMS))
    path = tmp_path / "s.dat"
    path.write_text(f"0\n{n}\n0.0\n" + body)
    s = ic.read_snapshot(path)
    want = np.array([LIBC.strtod(f.encode(), None) for f in FORMS])
    assert bits_equal(s.mass, want) and bits_equal(s.pot, want)
    assert bits_equal(s.pos[:, 2], want) and bits_equal(s.vel[:, 0], want)


def test_reader_accepts_records_across_lines(tmp_path):
    """Records laid out other than one per line are read token by token."""
    snap = ic.plummer(50, seed=5)
    path = tmp_path / "s.dat"
    ic.write_snapshot(path, snap)
    lines = path.read_text().splitlines()
    wrapped = lines[:3] + [t for ln in lines[3:] for t in (ln.split("    ", 2)[0] + "    " + ln.split("    ", 2)[1],
                                                          ln.split("    ", 2)[2])]
    (tmp_path / "w.dat").write_text("\n".join(wrapped) + "\n")
    back = ic.read_snapshot(tmp_path / "w.dat")
    assert bits_equal(back.pos, snap.pos) and bits_equal(back.vel, snap.vel) and bits_equal(back.mass, snap.mass)


def test_reader_rejects_short_files(tmp_path):
    snap = ic.plummer(20, seed=1)
    path = tmp_path / "s.dat"
    ic.write_snapshot(path, snap)
    text = path.read_text().splitlines()
    (tmp_path / "short.dat").write_text("\n".join(text[:-1]) + "\n")
    with pytest.raises(hb.HermiteError):
        ic.read_snapshot(tmp_path / "short.dat")
    (tmp_path / "cut.dat").write_text("\n".join(text[:-1] + [text[-1].rsplit(" ", 1)[0]]) + "\n")
    with pytest.raises(hb.HermiteError):
        ic.read_snapshot(tmp_path / "cut.dat")
