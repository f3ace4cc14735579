"""Out-of-bounds writes, without a sanitizer: every output array and workspace of every entry
point is placed between two 4 KB guard regions filled with a sentinel bit pattern, and after the
call the guards must be bit-for-bit unchanged. Shapes are odd on purpose: bsize 1 and 96 (the
plain-load path), bsize 32 with ragged per-track layer counts, the restart loop, the per-layer
calls, the host-buffer pipeline, the persistent queue (plain and ordered by layer count, bsize 32,
64 and 96), the grid and persistent adjoint paths with per-event gradients, the 3x3 gain routines
and the device-side generator."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GUARD_BYTES = 4096
PATTERN = {1: 0xA5, 4: 0x7FC0DEAD, 8: 0x7FF8DEADBEEFCAFE}


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


class Guarded:
    """n elements of `dtype` on the GPU with GUARD_BYTES of sentinel on either side (the array
    itself starts filled with the sentinel too)."""

    def __init__(self, torch, n, dtype):
        self.torch = torch
        size = torch.empty(0, dtype=dtype).element_size()
        self.pad = GUARD_BYTES // size
        self.n = n
        self.buf = torch.empty(n + 2 * self.pad, dtype=dtype, device="cuda")
        ity = {1: torch.uint8, 4: torch.int32, 8: torch.int64}[size]
        pat = PATTERN[size]
        if size == 4 and pat >= 1 << 31:
            pat -= 1 << 32
        self.bits = self.buf.view(ity)
        self.bits.fill_(pat)
        self.pat = pat
        self.t = self.buf[self.pad:self.pad + n]

    def intact(self) -> bool:
        self.torch.cuda.synchronize()
        b = self.bits
        return bool((b[:self.pad] == self.pat).all() and (b[self.pad + self.n:] == self.pat).all())


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def inputs(p2r, torch, bs, nevts, nb, nlayer, seed=5):
    cfg = p2r.Config(bsize=bs, nlayer=nlayer, nevts=nevts, nb=nb, bz=3.8)
    trk, hit = p2r.generate_helix(cfg, p2r.gen_params(bz=3.8, seed=seed))
    return cfg, torch.from_numpy(trk.reshape(-1)).cuda(), torch.from_numpy(hit.reshape(-1)).cuda()


@pytest.mark.parametrize("bs,nevts,nb,nlayer,mode,ragged", [
    (1, 2, 5, 7, "chained", False), (96, 1, 3, 20, "chained", False), (32, 3, 4, 20, "restart", False),
    (32, 2, 3, 25, "chained", True), (64, 1, 2, 40, "chained", True)])
def test_forward_writes_stay_in_bounds(p2r, torch, bs, nevts, nb, nlayer, mode, ragged):
    cfg, trk, hit = inputs(p2r, torch, bs, nevts, nb, nlayer)
    cfg.mode = p2r.MODE_CHAINED if mode == "chained" else p2r.MODE_RESTART
    out = Guarded(torch, trk.numel(), torch.float32)
    chi2 = Guarded(torch, cfg.ntracks, torch.float32)
    chi2.t.zero_()
    dr = torch.linspace(-0.01, 0.01, nlayer, device="cuda")
    nlay = None
    if ragged:
        nlay = torch.randint(0, nlayer + 1, (cfg.ntracks,), dtype=torch.int32, device="cuda",
                             generator=torch.Generator("cuda").manual_seed(1))
    p2r.forward(cfg, trk, hit, out.t, chi2=chi2.t, dr=dr, nlay_lane=nlay)
    assert out.intact() and chi2.intact()


def test_per_layer_calls_and_host_pipeline_stay_in_bounds(p2r, torch):
    cfg, trk, hit = inputs(p2r, torch, 32, 2, 3, 20)
    out = Guarded(torch, trk.numel(), torch.float32)
    acc = Guarded(torch, cfg.ntracks, torch.float32)
    acc.t.zero_()
    out.t.copy_(trk)
    for layer in range(cfg.nlayer):
        p2r.propagateToR(cfg, out.t, hit, layer, out.t)
        p2r.KalmanUpdate(cfg, out.t, hit, layer, chi2_accum=acc.t)
    assert out.intact() and acc.intact()
    h_t, h_h = trk.cpu().pin_memory(), hit.cpu().pin_memory()
    h_o = torch.empty_like(h_t).pin_memory()
    d_t, d_h, d_o = (Guarded(torch, trk.numel(), torch.float32), Guarded(torch, hit.numel(), torch.float32),
                     Guarded(torch, trk.numel(), torch.float32))
    p2r.forward_host(cfg, h_t.numpy(), h_h.numpy(), h_o.numpy(), d_t.t, d_h.t, d_o.t, nchunks=3)
    assert d_t.intact() and d_h.intact() and d_o.intact()


@pytest.mark.parametrize("bs,ordered,threads", [(32, False, 64), (32, True, 0), (64, True, 128), (96, True, 0)])
def test_queue_writes_stay_in_bounds(p2r, torch, bs, ordered, threads):
    w = p2r.uneven_workload(p2r.lognormal_counts(7, median=60, sigma=1.0, lo=1, hi=400, seed=2), bsize=bs,
                            nlayer_max=25)
    q = p2r.Queue(w, blocks_per_item=3 if ordered else 2, block_threads=threads,
                  flags=p2r.FLAG_ORDER_BY_LAYERS if ordered else 0)
    ws = Guarded(torch, q.ws.numel(), torch.uint8)
    done = Guarded(torch, q.done_ns.numel(), q.done_ns.dtype)
    start = Guarded(torch, q.start_ns.numel(), q.start_ns.dtype)
    q.ws, q.done_ns, q.start_ns = ws.t, done.t, start.t
    trk = torch.from_numpy(w["trk"].reshape(-1)).cuda()
    hit = torch.from_numpy(w["hit"].reshape(-1)).cuda()
    out = Guarded(torch, trk.numel(), torch.float32)
    chi2 = Guarded(torch, trk.numel() // 28, torch.float32)
    q.run(trk, hit, out.t, chi2=chi2.t)
    assert all(g.intact() for g in (ws, done, start, out, chi2))
    assert q.error_bits() == 0


@pytest.mark.parametrize("ordered", [False, True])
def test_queue_adjoint_writes_stay_in_bounds(p2r, torch, ordered):
    w = p2r.uneven_workload(p2r.lognormal_counts(6, median=70, sigma=1.0, lo=1, hi=300, seed=4), bsize=32,
                            nlayer_max=21, lay_lo=3, lay_hi=21)
    q = p2r.Queue(w, blocks_per_item=2, flags=p2r.FLAG_ORDER_BY_LAYERS if ordered else 0)
    trk = torch.from_numpy(w["trk"].reshape(-1)).cuda()
    hit = torch.from_numpy(w["hit"].reshape(-1)).cuda()
    ntr, nl, ne = trk.numel() // 28, w["nlayer"], q.nevts
    f32, f64 = torch.float32, torch.float64
    g = {"trk_out": Guarded(torch, trk.numel(), f32), "chi2": Guarded(torch, ntr, f32),
         "grad_trk_in": Guarded(torch, trk.numel(), f32), "grad_hits": Guarded(torch, hit.numel(), f32),
         "grad_dr": Guarded(torch, nl, f64), "grad_bz": Guarded(torch, 1, f64),
         "grad_dr_event": Guarded(torch, ne * nl, f64), "grad_bz_event": Guarded(torch, ne, f64),
         "workspace": Guarded(torch, q.adjoint_workspace_size(), torch.uint8)}
    out = {k: v.t for k, v in g.items()}
    q.run_adjoint(trk, hit, dr=torch.zeros(nl, device="cuda"), grad_chi2=torch.ones(ntr, device="cuda"), out=out)
    bad = [k for k, v in g.items() if not v.intact()]
    assert not bad, bad
    assert q.error_bits() == 0


def test_gain3_writes_stay_in_bounds(p2r, torch):
    cfg, trk, hit = inputs(p2r, torch, 96, 2, 3, 11)
    inv = Guarded(torch, cfg.nblocks * 9 * 96, torch.float32)
    gain = Guarded(torch, cfg.nblocks * 18 * 96, torch.float32)
    p2r.KalmanGainInv(cfg, trk, hit, 10, inv.t)
    p2r.KalmanGain(cfg, trk, inv.t, gain.t)
    assert inv.intact() and gain.intact()


@pytest.mark.parametrize("tape,ckpt", [(True, 1), (True, 5), (False, 5)])
def test_adjoint_writes_stay_in_bounds(p2r, torch, tape, ckpt):
    cfg, trk, hit = inputs(p2r, torch, 32, 2, 3, 20)
    nlay = torch.randint(5, 21, (cfg.ntracks,), dtype=torch.int32, device="cuda",
                         generator=torch.Generator("cuda").manual_seed(3))
    f32, f64 = torch.float32, torch.float64
    g = {"trk_out": Guarded(torch, trk.numel(), f32), "chi2": Guarded(torch, cfg.ntracks, f32),
         "grad_trk_in": Guarded(torch, trk.numel(), f32), "grad_hits": Guarded(torch, hit.numel(), f32),
         "grad_dr": Guarded(torch, cfg.nlayer, f64), "grad_bz": Guarded(torch, 1, f64),
         "grad_dr_event": Guarded(torch, cfg.nevts * cfg.nlayer, f64), "grad_bz_event": Guarded(torch, cfg.nevts, f64),
         "workspace": Guarded(torch, p2r.workspace_size(cfg, ckpt if tape else None), torch.uint8)}
    out = {k: v.t for k, v in g.items()}
    out["grad_dr_event"] = out["grad_dr_event"].view(cfg.nevts, cfg.nlayer)
    p2r.forward_backward(cfg, trk, hit, dr=torch.zeros(cfg.nlayer, device="cuda"), nlay_lane=nlay,
                         grad_chi2=torch.ones(cfg.ntracks, device="cuda"), ckpt_stride=ckpt, per_event=True, out=out,
                         tape=tape)
    bad = [k for k, v in g.items() if not v.intact()]
    assert not bad, bad


def test_device_generator_writes_stay_in_bounds(p2r, torch):
    bs, nevts, nb, nlayer = 96, 2, 3, 11
    trk = Guarded(torch, nevts * nb * 28 * bs, torch.float32)
    hit = Guarded(torch, nevts * nb * nlayer * 9 * bs, torch.float32)
    gp = p2r.gen_params(bz=3.8)
    p2r._lib.check(p2r.lib().p2r_gen_helix_device(ctypes.byref(gp), bs, nevts, nb, nlayer, None, ptr(trk.t),
                                                  ptr(hit.t), None))
    assert trk.intact() and hit.intact()
