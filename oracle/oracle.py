"""ctypes access to the oracle libraries.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference arm, always as the checker or the timed CPU reference, never by
the product package.

  Oracle      the project's own CPU restatement (p2r_oracle.cpp), float and double
  RefTBB      the reference's CPU path compiled unmodified (ref_harness.cpp -> _ref/)
  RefGPU      the reference's own CUDA programs (cuda_v4.cu, cuda_uvm.cu) compiled
              unmodified (ref_gpu_harness.cu -> _ref/), timed beside the product's kernel
  gen_helix   the benchmark's synthetic helix inputs (helix_gen.cpp), for the timed
              reference arm, which must map no library of the product
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "_build" / "libp2r_oracle.so"
REF_DIR = HERE / "_ref"

_vp = ctypes.c_void_p


def _p(a):
    return None if a is None else a.ctypes.data


class Oracle:
    """Own restatement. run(..., prec='f32'|'f64') -> dict(out (float32 MPTRK), par, cov, chi2,
    prior = covariance entering the last update)."""

    def __init__(self, path: Path = ORACLE_LIB):
        if not path.exists():
            raise RuntimeError(f"{path} missing: build it with `make -C oracle oracle`")
        self.l = ctypes.CDLL(str(path))
        sig = [_vp, _vp, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _vp, _vp,
               _vp, _vp, _vp, _vp, _vp]
        for n in ("orc_run_f32", "orc_run_f64"):
            getattr(self.l, n).argtypes = sig
            getattr(self.l, n).restype = None
        self.l.orc_step_f64.argtypes = [_vp, _vp, ctypes.c_int, _vp, _vp, ctypes.c_double, ctypes.c_double, _vp, _vp]
        self.l.orc_step_f64.restype = ctypes.c_double
        self.l.orc_kfact_f32.argtypes = [ctypes.c_double]
        self.l.orc_kfact_f32.restype = ctypes.c_float

    def run(self, trk: np.ndarray, hit: np.ndarray, bsize: int, nlayer: int, mode: int, bz: float,
            prec: str = "f64", dr=None, nlay_lane=None) -> dict:
        trk = np.ascontiguousarray(trk, np.float32)
        hit = np.ascontiguousarray(hit, np.float32)
        nblocks = trk.size // (28 * bsize)
        ntr = nblocks * bsize
        out = np.empty_like(trk)
        par = np.empty((ntr, 6))
        cov = np.empty((ntr, 21))
        chi2 = np.empty(ntr)
        prior = np.zeros((ntr, 21))
        drv = None if dr is None else np.ascontiguousarray(dr, np.float64)
        nl = None if nlay_lane is None else np.ascontiguousarray(nlay_lane, np.int32)
        fn = self.l.orc_run_f32 if prec == "f32" else self.l.orc_run_f64
        fn(trk.ctypes.data, hit.ctypes.data, nblocks, bsize, nlayer, mode, bz, _p(drv), _p(nl), out.ctypes.data,
           par.ctypes.data, cov.ctypes.data, chi2.ctypes.data, prior.ctypes.data)
        return {"out": out, "par": par, "cov": cov, "chi2": chi2, "prior": prior}

    def step_f64(self, par, cov, q, hitpos, hitcov, dr, bz):
        par = np.ascontiguousarray(par, np.float64)
        cov = np.ascontiguousarray(cov, np.float64)
        hp = np.ascontiguousarray(hitpos, np.float64)
        hc = np.ascontiguousarray(hitcov, np.float64)
        po = np.empty(6)
        co = np.empty(21)
        chi2 = self.l.orc_step_f64(par.ctypes.data, cov.ctypes.data, int(q), hp.ctypes.data, hc.ctypes.data,
                                   float(dr), float(bz), po.ctypes.data, co.ctypes.data)
        return po, co, chi2


# The benchmark workload's generator settings: the defaults of the product's p2r_gen_params
# (include/p2r.h), in its field order after the seed.
HELIX_DEFAULTS = {"seed": 20240001, "bz": 3.8, "r_seed": 15.0, "r_first": 20.0, "r_last": 100.0, "pt": 4.0,
                  "pop_smear": 0.10, "theta_min": 0.3, "theta_max": 2.8, "cov_pos": 1e-4, "cov_ang": 1e-3,
                  "est_smear": 1.0, "hit_sigma": 1e-3}


def gen_helix(bsize: int, nevts: int, nb: int, nlayer: int, ntrk_event=None, nthreads: int = 0, **kw):
    """Synthetic helix events (helix_gen.cpp), bit-identical to the product's p2r_gen_helix for
    the same settings: returns host float32 (tracks, hits) shaped (nblocks, 28, bsize) and
    (nblocks*nlayer, 9, bsize). Keyword arguments override HELIX_DEFAULTS."""
    prm = dict(HELIX_DEFAULTS)
    for k, v in kw.items():
        if k not in prm:
            raise KeyError(k)
        prm[k] = v
    lib = ctypes.CDLL(str(ORACLE_LIB))
    fn = lib.orc_gen_helix
    fn.argtypes = [ctypes.c_uint64, _vp, ctypes.c_int, ctypes.c_long, ctypes.c_long, ctypes.c_int, _vp, _vp, _vp,
                   ctypes.c_int]
    fn.restype = ctypes.c_int
    vals = np.array([prm[k] for k in list(HELIX_DEFAULTS)[1:]], np.float64)
    nblocks = nevts * nb
    trk = np.empty((nblocks, 28, bsize), np.float32)
    hit = np.empty((nblocks * nlayer, 9, bsize), np.float32)
    nte = None if ntrk_event is None else np.ascontiguousarray(ntrk_event, np.int32)
    if nte is not None and nte.shape != (nevts,):
        raise ValueError("ntrk_event needs one entry per event")
    if fn(prm["seed"], vals.ctypes.data, bsize, nevts, nb, nlayer, _p(nte), trk.ctypes.data, hit.ctypes.data,
          nthreads) != 0:
        raise ValueError("orc_gen_helix: bad sizes or geometry")
    return trk, hit


def refgpu_available(kind: str) -> bool:
    return (REF_DIR / f"libp2r_refgpu_{kind}.so").exists()


class RefGPU:
    """The reference's own CUDA programs compiled unmodified (ref_gpu_harness.cu -> _ref/):
    kind 'v4' = GPUsequence (cuda_v4.cu:821-849, chained), 'uvm' = launch_p2r_kernel
    (cuda_uvm.cu:887-915, restart). Sizes are compile-time (sizes())."""

    def __init__(self, kind: str):
        path = REF_DIR / f"libp2r_refgpu_{kind}.so"
        if not path.exists():
            raise RuntimeError(f"{path} missing: build it with `make -C oracle refgpu REFDIR=<reference checkout>`")
        self.kind = kind
        self.l = ctypes.CDLL(str(path))
        self.l.refgpu_sizes.argtypes = [_vp, _vp, _vp, _vp]
        self.l.refgpu_run.argtypes = [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp]
        self.l.refgpu_run.restype = ctypes.c_int
        self.chained = bool(self.l.refgpu_chained())

    def sizes(self):
        """(nevts, nb, nlayer, bsize) the program was compiled for."""
        ne, nb, nl, bs = ctypes.c_long(), ctypes.c_long(), ctypes.c_int(), ctypes.c_int()
        self.l.refgpu_sizes(ctypes.byref(ne), ctypes.byref(nb), ctypes.byref(nl), ctypes.byref(bs))
        return ne.value, nb.value, nl.value, bs.value

    def run(self, trk_ptr: int, hit_ptr: int, out_ptr: int, warmup: int, iters: int, stream_ptr) -> float:
        """Launches the kernel warmup + iters times on the stream (device pointers of arrays of
        the compiled sizes); returns the CUDA-event milliseconds of the `iters` launches."""
        ms = ctypes.c_float(0)
        rc = self.l.refgpu_run(trk_ptr, hit_ptr, out_ptr, warmup, iters, stream_ptr, ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError(f"reference GPU kernel ({self.kind}) failed: CUDA error {rc}")
        return ms.value


def host_isa() -> str:
    """'v4' when the host CPU has AVX-512 (F, BW, VL, DQ, CD), else 'v3'."""
    try:
        flags = set()
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
        need = {"avx512f", "avx512bw", "avx512vl", "avx512dq", "avx512cd"}
        return "v4" if need <= flags else "v3"
    except OSError:
        return "v3"


def ref_available(bsize: int = 32, kind: str | None = None) -> bool:
    return (REF_DIR / f"libp2r_tbbref_b{bsize}_{kind or host_isa()}.so").exists()


class RefTBB:
    """The reference's own CPU functions (TBB:433-812) and driver loop, one build per bsize.

    kind: 'v3' / 'v4' = unmodified source (kfact fixed at 3.8112 T), 'kf' = run-time kfact.
    """

    def __init__(self, bsize: int = 32, kind: str | None = None):
        kind = kind or host_isa()
        path = REF_DIR / f"libp2r_tbbref_b{bsize}_{kind}.so"
        if not path.exists():
            raise RuntimeError(f"{path} missing: build it with `make -C oracle ref` where the reference exists")
        self.bsize = bsize
        self.kind = kind
        self.l = ctypes.CDLL(str(path))
        L = self.l
        L.ref_run.argtypes = [_vp, _vp, _vp, ctypes.c_long, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              ctypes.c_int]
        L.ref_run_masked.argtypes = [_vp, _vp, _vp, ctypes.c_long, ctypes.c_int, _vp]
        L.ref_set_bz.argtypes = [ctypes.c_double]
        L.ref_get_kfact.restype = ctypes.c_float
        L.ref_propagate_block.argtypes = [_vp, _vp, _vp]
        L.ref_update_block.argtypes = [_vp, _vp]
        L.ref_gain_inv_block.argtypes = [_vp, _vp, _vp]
        L.ref_gain_block.argtypes = [_vp, _vp, _vp]
        L.ref_prepare_fixture.argtypes = [_vp, _vp]
        L.ref_fixture_raw.argtypes = [_vp, _vp, _vp, _vp]
        for n in ("ref_fixture_nevts", "ref_fixture_ntrks", "ref_fixture_nb"):
            getattr(L, n).restype = ctypes.c_long

    def gain3(self, trk, hit, nblocks, nlayer, layer):
        """The reference's unused KalmanGainInv / KalmanGain (TBB:376-426) per block, with the
        hit of `layer`: returns (inv: nblocks x 9 x bsize, gain: nblocks x 18 x bsize)."""
        bs = self.bsize
        trk = np.ascontiguousarray(trk, np.float32).reshape(nblocks, 28 * bs)
        hit = np.ascontiguousarray(hit, np.float32).reshape(nblocks * nlayer, 9 * bs)
        inv = np.empty((nblocks, 9 * bs), np.float32)
        gain = np.empty((nblocks, 18 * bs), np.float32)
        for b in range(nblocks):
            self.l.ref_gain_inv_block(trk[b].ctypes.data, hit[layer + b * nlayer].ctypes.data, inv[b].ctypes.data)
            self.l.ref_gain_block(trk[b].ctypes.data, inv[b].ctypes.data, gain[b].ctypes.data)
        return inv.reshape(nblocks, 9, bs), gain.reshape(nblocks, 18, bs)

    def set_bz(self, bz: float) -> None:
        if self.l.ref_set_bz(bz) != 0:
            raise ValueError(f"this reference build has kfact fixed at 3.8112 T; use kind='kf' for bz={bz}")

    def run(self, trk, hit, nevts, nb, nlayer, chained, niter=1, nthreads=1):
        trk = np.ascontiguousarray(trk, np.float32)
        hit = np.ascontiguousarray(hit, np.float32)
        out = np.empty_like(trk)
        self.l.ref_run(trk.ctypes.data, hit.ctypes.data, out.ctypes.data, nevts, nb, nlayer, niter, nthreads,
                       1 if chained else 0)
        return out

    def run_into(self, trk, hit, out, nevts, nb, nlayer, chained, niter=1, nthreads=1):
        self.l.ref_run(trk.ctypes.data, hit.ctypes.data, out.ctypes.data, nevts, nb, nlayer, niter, nthreads,
                       1 if chained else 0)

    def run_masked(self, trk, hit, nlayer_max, nlay_lane):
        trk = np.ascontiguousarray(trk, np.float32)
        hit = np.ascontiguousarray(hit, np.float32)
        nl = np.ascontiguousarray(nlay_lane, np.int32)
        out = np.empty_like(trk)
        nblocks = trk.size // (28 * self.bsize)
        self.l.ref_run_masked(trk.ctypes.data, hit.ctypes.data, out.ctypes.data, nblocks, nlayer_max, nl.ctypes.data)
        return out

    def fixture_sizes(self):
        return int(self.l.ref_fixture_nevts()), int(self.l.ref_fixture_nb()), int(self.l.ref_fixture_nlayer())

    def prepare_fixture(self):
        nev, nb, nl = self.fixture_sizes()
        trk = np.empty(nev * nb * 28 * self.bsize, np.float32)
        hit = np.empty(nev * nb * nl * 9 * self.bsize, np.float32)
        self.l.ref_prepare_fixture(trk.ctypes.data, hit.ctypes.data)
        return trk, hit

    def fixture_raw(self):
        par = np.empty(6, np.float32)
        cov = np.empty(21, np.float32)
        q = np.zeros(1, np.int32)
        hits = np.empty((22, 9), np.float32)
        self.l.ref_fixture_raw(par.ctypes.data, cov.ctypes.data, q.ctypes.data, hits.ctypes.data)
        return par, cov, int(q[0]), hits
