"""The force launch-shape table and the autotuner's table writer (CPU).

The table hermite_b200/csrc/hb_tuning.inc is compiled into the library and
looked up by nearest (N, nact) bucket; these tests check that the committed
table is well formed and that the tuner's merge mode replaces only the
measured entries.
"""
import math
import re

from hermite_b200 import autotune

TABLE = autotune.PKG / "csrc" / "hb_tuning.inc"
ENTRY = re.compile(r"^\{(\d+), (\d+), (\d+), (\d+), (\d+), (\d+)\},$")
NUM_VARIANTS = 20


def _entries(path):
    out = []
    for line in path.read_text().splitlines():
        if line.startswith("{"):
            m = ENTRY.match(line)
            assert m, line
            out.append(tuple(int(x) for x in m.groups()))
        else:
            assert line.startswith("//") or not line.strip(), line
    return out


def test_committed_table_is_well_formed():
    ent = _entries(TABLE)
    keys = [e[:4] for e in ent]
    assert len(keys) == len(set(keys))                       # one entry per bucket
    assert keys == sorted(keys)
    for order, mixed, log2n, log2nact, variant, jsplit in ent:
        assert order in (4, 6, 8) and mixed in (0, 1)
        assert 0 <= variant < NUM_VARIANTS and jsplit >= 1
        assert 0 <= log2nact <= log2n <= 20
    # every order and precision has entries at every N bucket
    for order in (4, 6, 8):
        for mixed in (0, 1):
            ns = {e[2] for e in ent if e[0] == order and e[1] == mixed}
            assert ns == {int(math.log2(n)) for n in autotune.N_BUCKETS}, (order, mixed, ns)


def test_merge_replaces_only_measured_entries(tmp_path):
    p = tmp_path / "t.inc"
    p.write_text("// header\n{4, 0, 16, 12, 4, 37},\n{4, 0, 16, 14, 1, 16},\n{6, 0, 18, 2, 13, 296},\n")
    res = [
        {"order": 4, "precision": "fp64", "n": 65536, "nact": 16384, "variant": 19, "jsplit": 8},
        {"order": 4, "precision": "fp64", "n": 65536, "nact": 8192, "variant": 19, "jsplit": 37},
        {"order": 4, "precision": "mixed", "n": 65536, "nact": 8192, "variant": 3, "jsplit": 10},
    ]
    autotune.merge_inc(res, p, "TEST")
    ent = _entries(p)
    assert ent == [(4, 0, 16, 12, 4, 37), (4, 0, 16, 13, 19, 37), (4, 0, 16, 14, 19, 8),
                   (4, 1, 16, 13, 3, 10), (6, 0, 18, 2, 13, 296)]
    lines = p.read_text().splitlines()
    assert lines[0] == "// header" and "TEST" in lines[1] and "nact 2^13,14" in lines[1]


def test_write_then_merge_round_trip(tmp_path):
    p = tmp_path / "t.inc"
    res = [{"order": 8, "precision": "fp64", "n": 1 << 20, "nact": 1 << k, "variant": k % NUM_VARIANTS,
            "jsplit": 1 + k} for k in range(0, 21, 2)]
    autotune.write_inc(res, p, "TEST")
    autotune.merge_inc(res[:3], p, "TEST")     # the same measurements again: no change
    assert _entries(p) == [(8, 0, 20, k, k % NUM_VARIANTS, 1 + k) for k in range(0, 21, 2)]


def test_slice_candidates():
    for nact in (1, 7, 300, 4096, 65536):
        c = autotune.s_candidates(nact, 65536, 148, 128)
        assert c == sorted(set(c)) and c[0] == 1
        assert all(1 <= s <= 65536 // 256 for s in c)


def test_bench_reads_the_tiled_shape_the_library_takes():
    """bench.py's comparison runs of the tiled kernel use the tuning table's
    shape for the bucket (nearest N, then nearest nact; slice count rescaled
    to the bucket's CTA count), as the library's automatic choice does."""
    import sys
    sys.path.insert(0, str(autotune.PKG.parent))
    import bench
    table = {e[:4]: e[4:] for e in _entries(TABLE)}
    for nact in (1, 4, 16):
        v, s = bench.tiled_shape(6, 262144, nact)
        la = min((k[3] for k in table if k[:3] == (6, 0, 18)), key=lambda b: abs(b - math.log2(nact)))
        tv, ts = table[(6, 0, 18, la)]
        assert v == tv
        # one i-tile at these nact: the slice count scales by the bucket's i-tiles
        assert s >= ts and s % ts == 0
