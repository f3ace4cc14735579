"""Python host API over the C ABI, mirroring the reference's call shape.

The reference (cerati/p2r-tests, src/propagate-tor-test_tbb.cpp, "TBB") exposes two
per-block functions over caller-owned Matriplex arrays:

    propagateToR(inErr, inPar, inChg, msP, outErr, outPar)     TBB:656-657
    KalmanUpdate(trkErr, inPar, hitErr, msP)                   TBB:433

and a driver loop (TBB:870-926) that applies them to every block and layer. Here
`propagateToR` / `KalmanUpdate` take whole device arrays plus a layer index (one call =
one iteration of the reference's layer loop over every block), and `forward` runs the
whole loop fused in one kernel. Arrays are torch CUDA tensors of float32 with the
reference's byte layout: tracks (nblocks, 28, bsize) = par 6 | cov 21 | q 1 rows, hits
(nblocks*nlayer, 9, bsize) = pos 3 | cov 6 rows (q is an int32 row viewed as float32).

Errors raise P2RError with the library's message; the reference has no error channel
(its functions return void and its CUDA drivers abort on failure).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (CConfig, CGenParams, CSummary, FLAG_FP32_DET, FLAG_NO_STAGING, MODE_CHAINED,
                   MODE_RESTART, P2RError, check, lib)

TRK_WORDS = 28
HIT_WORDS = 9
REF_BZ = 3.8112  # field compiled into the reference (TBB:654)


@dataclass
class Config:
    """Sizes and options of one run (the reference's -D macros, TBB:15-38, at run time)."""
    bsize: int = 32
    nlayer: int = 20
    nevts: int = 1
    nb: int = 1
    bz: float = REF_BZ
    mode: int = MODE_CHAINED
    flags: int = 0
    block_threads: int = 0
    stages: int = 0

    @property
    def nblocks(self) -> int:
        return self.nevts * self.nb

    @property
    def ntracks(self) -> int:
        return self.nblocks * self.bsize

    def c(self) -> CConfig:
        return CConfig(self.bsize, self.nlayer, self.nevts, self.nb, self.bz, self.mode, self.flags,
                       self.block_threads, self.stages)


def kfact(bz: float) -> float:
    return float(lib().p2r_kfact(bz))


def _ptr(t) -> int | None:
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        if not t.is_cuda:
            raise P2RError(_lib.P2R_ERR_INVALID, "device tensor expected")
        if not t.is_contiguous():
            raise P2RError(_lib.P2R_ERR_INVALID, "contiguous tensor expected")
        return t.data_ptr()
    return int(t)


def _arg(t, dtype: str, numel: int | None, name: str) -> int | None:
    """Device pointer of an optional array argument, after checking that it is a `dtype`
    tensor of at least `numel` elements: the library reads or writes that many elements of
    that type behind the pointer and cannot see the tensor's own size or type."""
    if t is None:
        return None
    if hasattr(t, "dtype"):
        import torch
        if t.dtype != getattr(torch, dtype):
            raise P2RError(_lib.P2R_ERR_INVALID, f"{name}: {t.dtype} tensor given, torch.{dtype} expected")
        if numel is not None and t.numel() < numel:
            raise P2RError(_lib.P2R_ERR_INVALID, f"{name}: {t.numel()} elements given, {numel} needed")
    return _ptr(t)


def _stream(stream) -> int | None:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


def _check_shapes(cfg: Config, trk, hits) -> None:
    for t in (trk, hits):
        if t is not None and hasattr(t, "dtype") and str(t.dtype) != "torch.float32":
            raise P2RError(_lib.P2R_ERR_INVALID, f"Matriplex arrays are float32 tensors, {t.dtype} given")
    if trk is not None and hasattr(trk, "numel") and trk.numel() != cfg.nblocks * TRK_WORDS * cfg.bsize:
        raise P2RError(_lib.P2R_ERR_INVALID,
                       f"track array has {trk.numel()} words, expected {cfg.nblocks * TRK_WORDS * cfg.bsize}")
    if hits is not None and hasattr(hits, "numel") and hits.numel() != cfg.nblocks * cfg.nlayer * HIT_WORDS * cfg.bsize:
        raise P2RError(_lib.P2R_ERR_INVALID, "hit array size does not match nevts*nb*nlayer blocks")


# ------------------------------------------------------------------ reference call shape
def propagateToR(cfg: Config, trk_in, hits, layer: int, trk_out, dr=None, stream=None) -> None:
    """propagateToR (TBB:656-812) of every block to its hit in `layer` (TBB:894)."""
    _check_shapes(cfg, trk_in, hits)
    _check_shapes(cfg, trk_out, None)
    c = cfg.c()
    check(lib().p2r_propagate_to_r(ctypes.byref(c), _ptr(trk_in), _ptr(hits), layer, _ptr(trk_out),
                                   _arg(dr, "float32", cfg.nlayer, "dr"), _stream(stream)))


def KalmanUpdate(cfg: Config, trk, hits, layer: int, chi2_accum=None, stream=None) -> None:
    """KalmanUpdate (TBB:433-642) of every block with its hit in `layer`, in place (TBB:911)."""
    _check_shapes(cfg, trk, hits)
    c = cfg.c()
    check(lib().p2r_kalman_update(ctypes.byref(c), _ptr(trk), _ptr(hits), layer,
                                  _arg(chi2_accum, "float32", cfg.ntracks, "chi2_accum"), _stream(stream)))


def KalmanGainInv(cfg: Config, trk, hits, layer: int, inv_out, stream=None) -> None:
    """The reference's unused KalmanGainInv (TBB:376-404) of every block with its hit in
    `layer`: one MP3x3 block (9*bsize floats) per track block in inv_out."""
    _check_shapes(cfg, trk, hits)
    c = cfg.c()
    check(lib().p2r_kalman_gain_inv(ctypes.byref(c), _ptr(trk), _ptr(hits), layer,
                                    _arg(inv_out, "float32", cfg.nblocks * 9 * cfg.bsize, "inv_out"),
                                    _stream(stream)))


def KalmanGain(cfg: Config, trk, inv, gain_out, stream=None) -> None:
    """The reference's unused KalmanGain (TBB:405-426): one MP3x6 block (18*bsize floats) per
    track block in gain_out, from the track covariance and KalmanGainInv's output."""
    _check_shapes(cfg, trk, None)
    c = cfg.c()
    check(lib().p2r_kalman_gain(ctypes.byref(c), _ptr(trk), _arg(inv, "float32", cfg.nblocks * 9 * cfg.bsize, "inv"),
                                _arg(gain_out, "float32", cfg.nblocks * 18 * cfg.bsize, "gain_out"),
                                _stream(stream)))


def run_layers(cfg: Config, trk_in, hits, trk_out, stream=None) -> None:
    """The reference driver loop (TBB:878-923) issued layer by layer through the two calls."""
    trk_out.copy_(trk_in)
    for layer in range(cfg.nlayer):
        src = trk_in if cfg.mode == MODE_RESTART else trk_out
        propagateToR(cfg, src, hits, layer, trk_out, stream=stream)
        KalmanUpdate(cfg, trk_out, hits, layer, stream=stream)


# ------------------------------------------------------------------ fused
def forward(cfg: Config, trk_in, hits, trk_out, chi2=None, dr=None, nlay_lane=None, stream=None) -> None:
    """All layers of every track in one fused launch (restart or chained, cfg.mode)."""
    _check_shapes(cfg, trk_in, hits)
    _check_shapes(cfg, trk_out, None)
    c = cfg.c()
    p_chi2, p_dr = _arg(chi2, "float32", cfg.ntracks, "chi2"), _arg(dr, "float32", cfg.nlayer, "dr")
    if nlay_lane is None:
        check(lib().p2r_forward(ctypes.byref(c), _ptr(trk_in), _ptr(hits), _ptr(trk_out), p_chi2, p_dr,
                                _stream(stream)))
    else:
        check(lib().p2r_forward_masked(ctypes.byref(c), _ptr(trk_in), _ptr(hits), _ptr(trk_out),
                                       _arg(nlay_lane, "int32", cfg.ntracks, "nlay_lane"), p_chi2, p_dr,
                                       _stream(stream)))


def forward_host(cfg: Config, host_trk_in: np.ndarray, host_hits: np.ndarray, host_trk_out: np.ndarray,
                 dev_trk_in, dev_hits, dev_trk_out, nchunks: int = 8, stream=None) -> None:
    """Fused forward from HOST arrays to a HOST array, copies overlapped with kernels in chunks."""
    for a in (host_trk_in, host_hits, host_trk_out):
        if not (isinstance(a, np.ndarray) and a.flags.c_contiguous and a.dtype == np.float32):
            raise P2RError(_lib.P2R_ERR_INVALID, "host arrays must be C-contiguous float32 numpy arrays")
    _check_shapes(cfg, dev_trk_in, dev_hits)
    _check_shapes(cfg, dev_trk_out, None)
    if host_trk_in.nbytes != cfg.nblocks * TRK_WORDS * cfg.bsize * 4 or host_trk_out.nbytes != host_trk_in.nbytes \
            or host_hits.nbytes != cfg.nblocks * cfg.nlayer * HIT_WORDS * cfg.bsize * 4:
        raise P2RError(_lib.P2R_ERR_INVALID, "host array sizes do not match the config")
    c = cfg.c()
    check(lib().p2r_forward_host(ctypes.byref(c), host_trk_in.ctypes.data, host_hits.ctypes.data,
                                 host_trk_out.ctypes.data, _ptr(dev_trk_in), _ptr(dev_hits), _ptr(dev_trk_out),
                                 nchunks, _stream(stream)))


def fp32_fma_probe(out, iters: int, blocks: int, threads: int = 256, stream=None, packed: bool = False) -> int:
    """Launches the FP32 FMA probe (packed: the f32x2 form); returns the FLOPs it performs."""
    fn = lib().p2r_fp32x2_fma_probe if packed else lib().p2r_fp32_fma_probe
    check(fn(iters, blocks, threads, _arg(out, "float32", blocks * threads, "out"), _stream(stream)))
    return 64 * iters * blocks * threads


def fp64_fma_probe(out, iters: int, blocks: int, threads: int = 256, stream=None) -> int:
    """Launches the FP64 FMA probe (out: float64, blocks*threads); returns the FLOPs it performs."""
    check(lib().p2r_fp64_fma_probe(iters, blocks, threads, _arg(out, "float64", blocks * threads, "out"),
                                   _stream(stream)))
    return 64 * iters * blocks * threads


def math_variant() -> str:
    """Which division / square-root build the library is: "refined", "ieee" or "fast"."""
    return {_lib.MATH_REFINED: "refined", _lib.MATH_IEEE: "ieee", _lib.MATH_FAST: "fast"}[lib().p2r_math_variant()]


def math_check(a, b, stream=None):
    """The hot path's own a / b and sqrt(a) on the device (float32 tensors of one size)."""
    import torch
    quot, root = torch.empty_like(a), torch.empty_like(a)
    check(lib().p2r_math_check(a.numel(), _arg(a, "float32", None, "a"), _arg(b, "float32", a.numel(), "b"),
                               _ptr(quot), _ptr(root), _stream(stream)))
    return quot, root


def count_nonfinite(trk, nblocks: int, bsize: int, stream=None) -> int:
    import torch
    cnt = torch.zeros(1, dtype=torch.int64, device=trk.device)
    check(lib().p2r_count_nonfinite(_arg(trk, "float32", nblocks * TRK_WORDS * bsize, "trk"), nblocks, bsize,
                                    _ptr(cnt), _stream(stream)))
    return int(cnt.item())


# ------------------------------------------------------------------ host generators
def gen_params(**kw) -> CGenParams:
    gp = CGenParams()
    lib().p2r_gen_params_default(ctypes.byref(gp))
    for k, v in kw.items():
        if not hasattr(gp, k):
            raise KeyError(k)
        setattr(gp, k, v)
    return gp


def generate_helix(cfg: Config, params: CGenParams | None = None, ntrk_event=None, nthreads: int = 0):
    """Synthetic helices (FP64 truth) -> host float32 arrays (tracks, hits) in Matriplex layout."""
    gp = params if params is not None else gen_params(bz=cfg.bz)
    trk = np.empty((cfg.nblocks, TRK_WORDS, cfg.bsize), np.float32)
    hit = np.empty((cfg.nblocks * cfg.nlayer, HIT_WORDS, cfg.bsize), np.float32)
    nte = None
    if ntrk_event is not None:
        nte = np.ascontiguousarray(ntrk_event, dtype=np.int32)
        if nte.shape != (cfg.nevts,):
            raise P2RError(_lib.P2R_ERR_INVALID, "ntrk_event needs one entry per event")
    check(lib().p2r_gen_helix(ctypes.byref(gp), cfg.bsize, cfg.nevts, cfg.nb, cfg.nlayer,
                              None if nte is None else nte.ctypes.data, trk.ctypes.data, hit.ctypes.data, nthreads))
    return trk, hit


def generate_helix_device(cfg: Config, params: CGenParams | None = None, ntrk_event=None, stream=None,
                          device=None):
    """generate_helix on the GPU: returns flat float32 device tensors (tracks, hits) in
    Matriplex layout, the same values as the host generator (rare 1-ulp differences)."""
    import torch
    gp = params if params is not None else gen_params(bz=cfg.bz)
    dev = torch.device("cuda") if device is None else torch.device(device)
    trk = torch.empty(cfg.nblocks * TRK_WORDS * cfg.bsize, dtype=torch.float32, device=dev)
    hit = torch.empty(cfg.nblocks * cfg.nlayer * HIT_WORDS * cfg.bsize, dtype=torch.float32, device=dev)
    nte = None
    if ntrk_event is not None:
        nte = torch.as_tensor(np.asarray(ntrk_event, dtype=np.int32)).to(dev)
        if nte.shape != (cfg.nevts,):
            raise P2RError(_lib.P2R_ERR_INVALID, "ntrk_event needs one entry per event")
    check(lib().p2r_gen_helix_device(ctypes.byref(gp), cfg.bsize, cfg.nevts, cfg.nb, cfg.nlayer, _ptr(nte),
                                     _ptr(trk), _ptr(hit), _stream(stream)))
    return trk, hit


def generate_fixture(seed_par, seed_cov, seed_q: int, input_hits, cfg: Config, smear: float = 1e-5):
    """The reference's recipe (TBB:243-293) from a seed track and per-layer hits (pos 3, cov 6)."""
    par = np.ascontiguousarray(seed_par, np.float32)
    cov = np.ascontiguousarray(seed_cov, np.float32)
    hits_in = np.ascontiguousarray(input_hits, np.float32).reshape(-1, 9)
    trk = np.empty((cfg.nblocks, TRK_WORDS, cfg.bsize), np.float32)
    hit = np.empty((cfg.nblocks * cfg.nlayer, HIT_WORDS, cfg.bsize), np.float32)
    check(lib().p2r_gen_fixture(par.ctypes.data, cov.ctypes.data, seed_q, hits_in.ctypes.data, hits_in.shape[0],
                                cfg.bsize, cfg.nevts, cfg.nb, cfg.nlayer, smear, trk.ctypes.data, hit.ctypes.data))
    return trk, hit


def summary(trk_host: np.ndarray, cfg: Config, last_hit_xyz) -> dict:
    """The reference's validation printout (TBB:935-1048) as a dict."""
    t = np.ascontiguousarray(trk_host, np.float32)
    h = np.ascontiguousarray(last_hit_xyz, np.float32)
    s = CSummary()
    check(lib().p2r_summary(t.ctypes.data, cfg.bsize, cfg.nevts, cfg.nb, h.ctypes.data, ctypes.byref(s)))
    return {name: getattr(s, name) for name, _ in CSummary._fields_}


# ------------------------------------------------------------------ layout helpers
def tracks_par(trk: np.ndarray) -> np.ndarray:
    """(ntracks, 6) parameters of a (nblocks, 28, bsize) track array."""
    return np.ascontiguousarray(trk[:, 0:6, :].transpose(0, 2, 1).reshape(-1, 6))


def tracks_cov(trk: np.ndarray) -> np.ndarray:
    """(ntracks, 21) packed covariances."""
    return np.ascontiguousarray(trk[:, 6:27, :].transpose(0, 2, 1).reshape(-1, 21))


def tracks_q(trk: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(trk[:, 27, :]).view(np.int32).reshape(-1)
