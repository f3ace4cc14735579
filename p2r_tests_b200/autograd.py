"""Forward + adjoint through the C ABI, and a torch.autograd.Function over it.

`forward_backward` calls p2r_forward_backward (the chained forward with checkpoints, then
the hand-written reverse sweep). `P2RChain.apply(trk, hits, dr, bz, cfg, ckpt_stride)`
(ckpt_stride None: auto_ckpt_stride's choice) returns (trk_out, chi2) from the plain fused
forward and, on backward, runs the adjoint kernel with the incoming cotangents, giving
gradients for the Matriplex track and hit arrays (parameter and covariance rows), the
per-layer radius offsets dr and Bz.
torch is used only for device memory and streams here; the arithmetic is the library's.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import P2RError, check, lib
from .api import Config, HIT_WORDS, TRK_WORDS, _arg, _check_shapes, _ptr, _stream


def workspace_size(cfg: Config, ckpt_stride: int | None = None) -> int:
    """Workspace bytes of p2r_forward_backward: the minimum (checkpoints in thread-local
    memory) when ckpt_stride is None, else the size that also holds the checkpoint tape."""
    c = cfg.c()
    if ckpt_stride is None:
        n = lib().p2r_forward_backward_workspace_size(ctypes.byref(c))
    else:
        n = lib().p2r_forward_backward_workspace_size_tape(ctypes.byref(c), ckpt_stride)
    if n == 0:
        raise P2RError(_lib.P2R_ERR_INVALID, lib().p2r_last_error_string().decode())
    return int(n)


def auto_ckpt_stride(cfg: Config, device, tape: bool = True) -> int:
    """The checkpoint stride used when the caller names none: 1 (the whole state tape, the
    fastest reverse) when its workspace fits in half the free device memory, else 5; 5 for
    thread-local checkpoints."""
    if not tape:
        return 5
    free, _ = torch.cuda.mem_get_info(device)
    return 1 if workspace_size(cfg, 1) <= free // 2 else 5


def forward_backward(cfg: Config, trk_in, hits, dr=None, nlay_lane=None, grad_trk_out=None, grad_chi2=None,
                     ckpt_stride: int | None = None, per_event: bool = False, stream=None, out=None,
                     tape: bool = True) -> dict:
    """Returns trk_out, chi2, grad_trk_in, grad_hits, grad_dr, grad_bz (and *_event).
    tape: give the library a workspace that holds the checkpoint tape (two-kernel path);
    False keeps the checkpoints in thread-local memory (smallest workspace). ckpt_stride None:
    auto_ckpt_stride's choice, made once per `out` dict and kept with its workspace (so repeated
    calls, a CUDA-graph capture among them, run the same stride). An entry of `out` set to None
    skips that output (e.g. grad_hits for calibration-only runs)."""
    _check_shapes(cfg, trk_in, hits)
    dev = trk_in.device
    o = out if out is not None else {}
    if ckpt_stride is None:
        if o.get("ckpt_stride") is None:
            o["ckpt_stride"] = auto_ckpt_stride(cfg, dev, tape)
        ckpt_stride = o["ckpt_stride"]
    f32 = dict(dtype=torch.float32, device=dev)
    f64 = dict(dtype=torch.float64, device=dev)
    o.setdefault("trk_out", torch.empty_like(trk_in))
    o.setdefault("chi2", torch.empty(cfg.ntracks, **f32))
    o.setdefault("grad_trk_in", torch.empty_like(trk_in))
    o.setdefault("grad_hits", torch.empty_like(hits))
    o.setdefault("grad_dr", torch.empty(cfg.nlayer, **f64))
    o.setdefault("grad_bz", torch.empty(1, **f64))
    if per_event:
        o.setdefault("grad_dr_event", torch.empty(cfg.nevts, cfg.nlayer, **f64))
        o.setdefault("grad_bz_event", torch.empty(cfg.nevts, **f64))
    ws = o.get("workspace")
    need = workspace_size(cfg, ckpt_stride if tape else None)
    if ws is None or ws.numel() < need:
        ws = torch.empty(need, dtype=torch.uint8, device=dev)
        o["workspace"] = ws
    c = cfg.c()
    ntrk, nt, nh, nl = cfg.ntracks, trk_in.numel(), hits.numel(), cfg.nlayer
    check(lib().p2r_forward_backward(
        ctypes.byref(c), _ptr(trk_in), _ptr(hits), _arg(dr, "float32", nl, "dr"),
        _arg(nlay_lane, "int32", ntrk, "nlay_lane"), _arg(o["trk_out"], "float32", nt, "trk_out"),
        _arg(o["chi2"], "float32", ntrk, "chi2"), _arg(grad_trk_out, "float32", nt, "grad_trk_out"),
        _arg(grad_chi2, "float32", ntrk, "grad_chi2"), _arg(o["grad_trk_in"], "float32", nt, "grad_trk_in"),
        _arg(o["grad_hits"], "float32", nh, "grad_hits"), _arg(o["grad_dr"], "float64", nl, "grad_dr"),
        _arg(o["grad_bz"], "float64", 1, "grad_bz"),
        _arg(o.get("grad_dr_event"), "float64", cfg.nevts * nl, "grad_dr_event"),
        _arg(o.get("grad_bz_event"), "float64", cfg.nevts, "grad_bz_event"), ckpt_stride,
        _arg(ws, "uint8", need, "workspace"), ws.numel(), _stream(stream)))
    return o


class P2RChain(torch.autograd.Function):
    """(trk, hits, dr, bz) -> (trk_out, chi2) for the chained layer loop.

    trk / hits: flat float32 CUDA tensors in Matriplex layout; dr: (nlayer,) float32 CUDA;
    bz: 0-dim tensor (tesla). Gradients flow to the parameter and covariance rows of trk,
    the position and covariance rows of hits, dr and bz."""

    @staticmethod
    def forward(ctx, trk, hits, dr, bz, cfg: Config, ckpt_stride: int | None = None):
        from .api import forward
        c = Config(**{**cfg.__dict__, "bz": float(bz), "mode": _lib.MODE_CHAINED})
        trk_out = torch.empty_like(trk)
        chi2 = torch.empty(c.ntracks, dtype=torch.float32, device=trk.device)
        forward(c, trk, hits, trk_out, chi2=chi2, dr=dr)
        ctx.save_for_backward(trk, hits, dr)
        ctx.cfg, ctx.ckpt, ctx.bz_dtype, ctx.bz_device = c, ckpt_stride, bz.dtype, bz.device
        return trk_out, chi2

    @staticmethod
    def backward(ctx, g_trk_out, g_chi2):
        trk, hits, dr = ctx.saved_tensors
        g_trk_out = None if g_trk_out is None else g_trk_out.contiguous()
        g_chi2 = None if g_chi2 is None else g_chi2.contiguous()
        o = forward_backward(ctx.cfg, trk, hits, dr=dr, grad_trk_out=g_trk_out, grad_chi2=g_chi2,
                             ckpt_stride=ctx.ckpt)
        return (o["grad_trk_in"], o["grad_hits"], o["grad_dr"].to(dr.dtype),
                o["grad_bz"][0].to(dtype=ctx.bz_dtype, device=ctx.bz_device), None, None)
