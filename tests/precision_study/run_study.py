"""Per-region precision study of the adjoint (see adjoint_precision.cpp).

Runs the chained forward + adjoint of 256 synthetic tracks x 20 layers (9600-track workload's
generator, radius offsets +-100 um, random cotangents of the final state, chi2 weights
U[0.5, 1.5]) with chosen arithmetic regions rounded to FP32, and reports each gradient group's
error against the all-FP64 run with the adjoint tests' metric: per element
|g - g64| / max(|g64|, 1e-3 * max |g64| of the group); the bar is 1e-3 on every element.

    python tests/precision_study/run_study.py [--tracks 256] [--json out.json]

Test infrastructure only; builds tests/precision_study/_build/libadjstudy.so with g++.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
LIB = HERE / "_build" / "libadjstudy.so"
REGIONS = ["path", "covprop", "upd", "pathrev", "covrev", "jbar", "jent", "updrec", "updrev"]
FWD_REGIONS = ["path", "covprop", "upd"]
GROUPS = ["par0", "cov0", "hpos", "hcov", "dr", "bz"]


def build() -> ctypes.CDLL:
    src = HERE / "adjoint_precision.cpp"
    hdr = ROOT / "p2r_tests_b200" / "csrc" / "p2r_adjoint.cuh"
    if not LIB.exists() or LIB.stat().st_mtime < max(src.stat().st_mtime, hdr.stat().st_mtime):
        LIB.parent.mkdir(exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-o", str(LIB), str(src)],
                       check=True)
    lib = ctypes.CDLL(str(LIB))
    vp = ctypes.c_void_p
    lib.study_track.argtypes = [vp, vp, ctypes.c_int, vp, ctypes.c_int, vp, ctypes.c_double, vp, vp, ctypes.c_double,
                                ctypes.c_uint, ctypes.c_uint, ctypes.c_int, vp, vp, vp, vp, vp]
    return lib


def mask(names) -> int:
    m = 0
    for n in names:
        m |= 1 << REGIONS.index(n)
    return m


def workload(ntracks: int, nlayer: int = 20, seed: int = 20240003):
    from oracle.oracle import gen_helix
    bs = 32
    nb = (ntracks + bs - 1) // bs
    trk, hit = gen_helix(bs, 1, nb, nlayer, seed=seed)
    t = trk.reshape(nb, 28, bs)
    h = hit.reshape(nb, nlayer, 9, bs)
    par = t[:, 0:6, :].transpose(0, 2, 1).reshape(-1, 6).astype(np.float64)[:ntracks]
    cov = t[:, 6:27, :].transpose(0, 2, 1).reshape(-1, 21).astype(np.float64)[:ntracks]
    q = np.ascontiguousarray(t[:, 27, :]).view(np.int32).reshape(-1)[:ntracks]
    hits = h.transpose(0, 3, 1, 2).reshape(-1, nlayer, 9).astype(np.float64)[:ntracks]
    rng = np.random.default_rng(seed)
    dr = rng.uniform(-0.01, 0.01, nlayer).astype(np.float32).astype(np.float64)
    g_par = rng.normal(size=(ntracks, 6))
    g_cov = rng.normal(size=(ntracks, 21)) * 1e2
    g_chi2 = rng.uniform(0.5, 1.5, ntracks).astype(np.float32).astype(np.float64)
    return dict(par=par, cov=cov, q=q, hits=np.ascontiguousarray(hits), dr=dr, bz=3.8, g_par=g_par, g_cov=g_cov,
                g_chi2=g_chi2, nlayer=nlayer)


def run(lib, w, fwd_mask: int, rev_mask: int, tape32: bool) -> dict:
    n, nl = len(w["par"]), w["nlayer"]
    out = {"par0": np.zeros((n, 6)), "cov0": np.zeros((n, 21)), "hpos": np.zeros((n, nl, 3)),
           "hcov": np.zeros((n, nl, 6)), "dr": np.zeros(nl), "bz": 0.0}
    op, oc, oh, od, ob = np.zeros(6), np.zeros(21), np.zeros(nl * 9), np.zeros(nl), np.zeros(1)
    p = lambda a: a.ctypes.data
    for i in range(n):
        par, cov, hits = np.ascontiguousarray(w["par"][i]), np.ascontiguousarray(w["cov"][i]), w["hits"][i]
        gp, gc = np.ascontiguousarray(w["g_par"][i]), np.ascontiguousarray(w["g_cov"][i])
        lib.study_track(p(par), p(cov), int(w["q"][i]), p(hits), nl, p(w["dr"]), w["bz"], p(gp), p(gc),
                        float(w["g_chi2"][i]), fwd_mask, rev_mask, int(tape32), p(op), p(oc), p(oh), p(od), p(ob))
        out["par0"][i], out["cov0"][i] = op, oc
        out["hpos"][i] = oh.reshape(nl, 9)[:, 0:3]
        out["hcov"][i] = oh.reshape(nl, 9)[:, 3:9]
        out["dr"] += od
        out["bz"] += ob[0]
    return out


def errors(g: dict, ref: dict) -> dict:
    res = {}
    for k in GROUPS:
        a, b = np.atleast_1d(np.asarray(g[k], np.float64)), np.atleast_1d(np.asarray(ref[k], np.float64))
        scale = max(np.abs(b).max(), 1e-300)
        e = np.abs(a - b) / np.maximum(np.abs(b), 1e-3 * scale)
        res[k] = {"p99": float(np.quantile(e, 0.99)), "max": float(e.max())}
    return res


def study(ntracks: int = 256) -> list[dict]:
    lib = build()
    w = workload(ntracks)
    ref = run(lib, w, 0, 0, False)
    cases = [("reverse sweep: " + r, 0, mask([r]), False) for r in REGIONS]
    cases += [("forward pass: " + r, mask([r]), 0, False) for r in FWD_REGIONS]
    cases += [("tape stored in FP32", 0, 0, True),
              ("reverse sweep: all regions", 0, mask(REGIONS), False),
              ("reverse sweep: all but covrev, jbar", 0, mask([r for r in REGIONS if r not in ("covrev", "jbar")]),
               False),
              ("reverse sweep: covrev, jbar, updrev", 0, mask(["covrev", "jbar", "updrev"]), False),
              ("reverse sweep: pathrev, jent", 0, mask(["pathrev", "jent"]), False),
              ("forward pass: all regions", mask(FWD_REGIONS), 0, False),
              ("everything (the FP32 instance)", mask(REGIONS), mask(REGIONS), True)]
    rows = []
    for name, fm, rm, t32 in cases:
        e = errors(run(lib, w, fm, rm, t32), ref)
        rows.append({"case": name, "fwd_mask": fm, "rev_mask": rm, "tape32": t32, "errors": e,
                     "worst": max(v["max"] for v in e.values()), "meets_1e-3": all(v["max"] < 1e-3 for v in e.values())})
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--tracks", type=int, default=256)
    ap.add_argument("--json", default=None)
    a = ap.parse_args()
    rows = study(a.tracks)
    print(f"{'case (regions in FP32)':44s} " + " ".join(f"{g:>9s}" for g in GROUPS) + "  bar")
    for r in rows:
        print(f"{r['case']:44s} " + " ".join(f"{r['errors'][g]['max']:9.1e}" for g in GROUPS) +
              ("  ok" if r["meets_1e-3"] else "  FAIL"))
    if a.json:
        Path(a.json).write_text(json.dumps(rows, indent=1))


if __name__ == "__main__":
    main()
