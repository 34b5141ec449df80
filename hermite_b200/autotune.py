"""Autotuner for the force kernel's launch shape.

For each (order, precision, N bucket, nact bucket) it times every compiled
kernel variant (threads per CTA, i-chunks per warp, in-CTA j split, tile
depth, register cap) and several j-slice counts S, on the current GPU, and
writes the fastest choice to hermite_b200/csrc/hb_tuning.inc, which the
library compiles in (hb_capi.cu looks up the nearest bucket).

    python -m hermite_b200.autotune [--out hermite_b200/csrc/hb_tuning.inc]
                                    [--json results.json] [--quick]
                                    [--orders 4,6,8] [--precisions fp64,mixed]
                                    [--n-buckets 65536] [--nact-buckets 2,8,32]
                                    [--merge] [--max-interactions X]
                                    [--variants 0,1,20] [--trials-json all.json]

--merge keeps the existing table and replaces or adds only the measured
(order, precision, N bucket, nact bucket) entries.

Timing: CUDA events on the context's stream around back-to-back force
launches (inputs resident, predicted once), median of the repeats.
Rebuild the library afterwards (python -m hermite_b200.build).
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import statistics
import sys
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
sys.path.insert(0, str(PKG.parent))

N_BUCKETS = (1024, 8192, 65536, 262144, 1048576)
NACT_BUCKETS = (1, 4, 16, 64, 256, 1024, 4096, 16384, 65536, 262144, 1048576)
MAX_INTERACTIONS = 1 << 34      # skip (N, nact) pairs beyond this per launch


def _records(order, n, seed=0):
    from hermite_b200.ic import plummer, records
    return records(plummer(n, seed), order)


def time_force(g, stream, nact, eps2, reps):
    """One block step's device work: predict_all + force (a two-pass shape
    runs the predictor pass, a fused shape predicts inside the force kernel)."""
    import torch
    g.predict_all_device(0.0)
    g.force_device(nact, eps2)              # warm-up (and first-use set-up)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    for _ in range(reps):
        e0.record(stream)
        g.predict_all_device(0.0)
        g.force_device(nact, eps2)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return statistics.median(times)


def s_candidates(nact, n, nsm, ti):
    gx = -(-nact // ti)
    nchunk = -(-n // 256) * 256 // 32
    smax = max(1, nchunk // 8)
    cands = {1}
    for mult in (0.5, 1, 2, 4, 8):
        s = int(math.ceil(mult * nsm / gx))
        cands.add(max(1, min(s, smax)))
    return sorted(cands)


def tune(orders, precisions, n_buckets, nact_buckets, quick=False, log=print,
         max_interactions=MAX_INTERACTIONS, variants=None, trials=None):
    """variants: restrict the timed shapes to these indices (None: all);
    trials: a list that receives every (shape, slice count) timing."""
    import torch
    from hermite_b200 import Gravity, load_library
    import ctypes
    lib = load_library()
    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    stream = torch.cuda.Stream()
    results = []
    for order in orders:
        for prec in precisions:
            pcode = 0 if prec == "fp64" else 1
            nvar = lib.hb_force_variant_count(order, pcode)
            tis = []
            for v in range(nvar):
                t, ni, wj = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
                lib.hb_force_variant_info(order, pcode, v, ctypes.byref(t), ctypes.byref(ni),
                                          ctypes.byref(wj))
                tis.append((t.value // 32 // wj.value) * 32 * ni.value)
            for n in n_buckets:
                eps2 = (4.0 / n) ** 2
                with torch.cuda.stream(stream):
                    g = Gravity(order, n, prec)
                    g.set_stream(stream.cuda_stream)
                    g.set_jp_records(_records(order, n))
                    g.upload()
                    g.predict_all_device(0.0)
                    for nact in nact_buckets:
                        if nact > n or nact * n > max_interactions:
                            continue
                        reps = 3 if nact * n > (1 << 30) else 7
                        best = None
                        for v in range(nvar):
                            if variants is not None and v not in variants:
                                continue
                            for s in s_candidates(nact, n, nsm, tis[v]):
                                if quick and s not in (1, s_candidates(nact, n, nsm, tis[v])[-1]):
                                    continue
                                g.set_force_shape(v, s)
                                ms = time_force(g, stream, nact, eps2, reps)
                                if trials is not None:
                                    trials.append({"order": order, "precision": prec, "n": n,
                                                   "nact": nact, "variant": v, "jsplit": s,
                                                   "ms": ms})
                                if best is None or ms < best[0]:
                                    best = (ms, v, s)
                        g.set_force_shape(-1, 0)
                        auto_ms = time_force(g, stream, nact, eps2, reps)
                        rec = {"order": order, "precision": prec, "n": n, "nact": nact,
                               "variant": best[1], "jsplit": best[2], "ms": best[0],
                               "gint_s": nact * n / best[0] * 1e-6, "auto_ms": auto_ms}
                        results.append(rec)
                        log(f"order {order} {prec:5s} N {n:8d} nact {nact:8d}: v{best[1]:2d} "
                            f"S{best[2]:4d} {best[0]*1e3:10.1f} us {rec['gint_s']:8.1f} Gint/s "
                            f"(heuristic {auto_ms*1e3:10.1f} us)")
                    g.close()
    return results


def write_inc(results, path: Path, device_name: str):
    lines = [f"// Generated by hermite_b200/autotune.py on {device_name}, "
             f"{datetime.date.today().isoformat()}.",
             "// {order, mixed, log2(N bucket), log2(nact bucket), variant, jsplit}"]
    for r in results:
        lines.append("{%d, %d, %d, %d, %d, %d}," % (
            r["order"], 1 if r["precision"] == "mixed" else 0, int(round(math.log2(r["n"]))),
            int(round(math.log2(r["nact"]))), r["variant"], r["jsplit"]))
    path.write_text("\n".join(lines) + "\n")


def merge_inc(results, path: Path, device_name: str):
    """Replace or add the measured entries in an existing table, keeping its
    other entries and comment lines; entries stay sorted by key."""
    comments, table = [], {}
    for line in path.read_text().splitlines():
        t = line.strip()
        if t.startswith("{"):
            v = [int(x) for x in t.strip("{},").split(",")]
            table[tuple(v[:4])] = tuple(v[4:])
        elif t:
            comments.append(line)
    keys = []
    for r in results:
        k = (r["order"], 1 if r["precision"] == "mixed" else 0, int(round(math.log2(r["n"]))),
             int(round(math.log2(r["nact"]))))
        table[k] = (r["variant"], r["jsplit"])
        keys.append(k)
    groups = sorted({k[:3] for k in keys})
    comments.append(f"// {datetime.date.today().isoformat()}, {device_name}: merged "
                    + ", ".join(f"(order {o}, {'mixed' if m else 'fp64'}, 2^{n})" for o, m, n in groups)
                    + " at nact 2^" + ",".join(sorted({str(k[3]) for k in keys}, key=int)))
    lines = comments + ["{%d, %d, %d, %d, %d, %d}," % (*k, *table[k]) for k in sorted(table)]
    path.write_text("\n".join(lines) + "\n")


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=str(PKG / "csrc" / "hb_tuning.inc"))
    ap.add_argument("--json", default=None)
    ap.add_argument("--orders", default="4,6,8")
    ap.add_argument("--precisions", default="fp64,mixed")
    ap.add_argument("--quick", action="store_true", help="fewer j-split candidates")
    ap.add_argument("--n-buckets", default=",".join(map(str, N_BUCKETS)))
    ap.add_argument("--nact-buckets", default=",".join(map(str, NACT_BUCKETS)))
    ap.add_argument("--merge", action="store_true", help="update only the measured entries")
    ap.add_argument("--max-interactions", type=float, default=float(MAX_INTERACTIONS),
                    help="skip buckets with more interactions per launch")
    ap.add_argument("--variants", default=None, help="time only these shapes (comma list)")
    ap.add_argument("--trials-json", default=None, help="write every timing here")
    a = ap.parse_args()
    import torch
    trials = []
    res = tune([int(x) for x in a.orders.split(",")], a.precisions.split(","),
               [int(x) for x in a.n_buckets.split(",")], [int(x) for x in a.nact_buckets.split(",")],
               quick=a.quick, max_interactions=int(a.max_interactions),
               variants=[int(v) for v in a.variants.split(",")] if a.variants else None,
               trials=trials)
    if a.trials_json:
        Path(a.trials_json).write_text(json.dumps(trials, indent=1))
    if a.merge and Path(a.out).exists():
        merge_inc(res, Path(a.out), torch.cuda.get_device_name(0))
    else:
        write_inc(res, Path(a.out), torch.cuda.get_device_name(0))
    if a.json:
        Path(a.json).write_text(json.dumps(res, indent=1))
    print(f"wrote {a.out} ({len(res)} entries)")


if __name__ == "__main__":
    main()
