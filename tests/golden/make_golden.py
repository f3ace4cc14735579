"""Generates the golden vectors in tests/golden/ from the reference's OWN code.

Run where the reference checkout exists (it is read only at build time, by
oracle/Makefile):  make -C oracle ref && python tests/golden/make_golden.py

Everything here comes from the reference's CPU path (src/propagate-tor-test_tbb.cpp)
compiled unmodified by oracle/ref_harness.cpp:
  fixture.npz/.txt     the seed track and 22 hits of src/input_track.h in the order the
                       reference's main uses them (TBB:818-820); .txt for the C++ driver
  ref_fixture_b{B}.npz for bsize B in 32/64/128: the reference's own generated inputs
                       (prepareTracks/prepareHits, TBB:243-293; inputs stored for B=32 only,
                       SHA-256 digests for all) and its outputs in restart mode (TBB:873-926)
                       and chained mode (cuda_v4.cu:840-846 loop over the same functions)
  ref_helix.npz        a small synthetic-helix event set at Bz = 3.8 T (inputs from this
                       package's generator) and the reference's outputs (run-time kfact
                       build) in both modes
  ref_main_b32.txt     stdout of the reference program's unmodified main at
                       -Dntrks=256 -Dnevts=2 -Dbsize=32 (the validation summary, TBB:935-1048)
"""
from __future__ import annotations

import ctypes
import hashlib
import io
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle.oracle import RefTBB  # noqa: E402

HELIX = dict(bsize=32, nevts=2, nb=8, nlayer=20, bz=3.8)


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    r32 = RefTBB(32, "v3")
    par, cov, q, hits = r32.fixture_raw()
    np.savez_compressed(HERE / "fixture.npz", par=par, cov=cov, q=np.int32(q), hits=hits)
    # the same numbers as text, the input format of the C++ driver (--input fixture FILE)
    with open(HERE / "fixture.txt", "w") as f:
        f.write(" ".join(repr(float(x)) for x in par) + "\n")
        f.write(" ".join(repr(float(x)) for x in cov) + "\n")
        f.write(f"{q}\n")
        for h in hits:
            f.write(" ".join(repr(float(x)) for x in h) + "\n")

    for bs in (32, 64, 128):
        r = RefTBB(bs, "v3")
        nev, nb, nl = r.fixture_sizes()
        trk, hit = r.prepare_fixture()
        out_restart = r.run(trk, hit, nev, nb, nl, chained=False)
        out_chained = r.run(trk, hit, nev, nb, nl, chained=True)
        payload = dict(bsize=np.int32(bs), nevts=np.int32(nev), nb=np.int32(nb), nlayer=np.int32(nl),
                       out_restart=out_restart, out_chained=out_chained,
                       trk_sha=np.bytes_(sha(trk)), hit_sha=np.bytes_(sha(hit)))
        if bs == 32:
            payload.update(trk=trk, hit=hit)
        np.savez_compressed(HERE / f"ref_fixture_b{bs}.npz", **payload)

    import p2r_tests_b200 as p2r
    cfg = p2r.Config(bsize=HELIX["bsize"], nlayer=HELIX["nlayer"], nevts=HELIX["nevts"], nb=HELIX["nb"],
                     bz=HELIX["bz"])
    trk, hit = p2r.generate_helix(cfg)
    rk = RefTBB(32, "kf")
    rk.set_bz(HELIX["bz"])
    out_restart = rk.run(trk, hit, cfg.nevts, cfg.nb, cfg.nlayer, chained=False)
    out_chained = rk.run(trk, hit, cfg.nevts, cfg.nb, cfg.nlayer, chained=True)
    np.savez_compressed(HERE / "ref_helix.npz", trk=trk, hit=hit, out_restart=out_restart,
                        out_chained=out_chained, bz=np.float64(HELIX["bz"]), bsize=np.int32(cfg.bsize),
                        nevts=np.int32(cfg.nevts), nb=np.int32(cfg.nb), nlayer=np.int32(cfg.nlayer),
                        kfact=np.float32(rk.l.ref_get_kfact()))

    # the unmodified main, in a child process so its stdout and rand() state are its own
    code = ("import sys; sys.path.insert(0, %r); from oracle.oracle import RefTBB; "
            "RefTBB(32, 'v3').l.ref_main()" % str(ROOT))
    res = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True)
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith(("track ", "number of", "done ntracks"))]
    # the timing line varies run to run; keep its shape only
    lines = [ln.split(" tot time=")[0] if ln.startswith("done ntracks") else ln for ln in lines]
    (HERE / "ref_main_b32.txt").write_text("\n".join(lines) + "\n")
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
