"""Forward + adjoint of uneven batches in one persistent launch (p2r_run_queue_adjoint) and its
CUDA graph, against the grid adjoint (p2r_forward_backward, stride-1 tape) and the FP64
reference gradient.

The per-lane arithmetic of both paths is the same device code in FP64, so per-track outputs
agree to rounding (1e-10 relative on the adjoint tests' metric); the shared gradients are
summed per 32-lane slice in the same fixed order by both, so the per-event dr / Bz gradients of
an evenly shaped batch agree to 1e-12.
"""
import ctypes

import numpy as np
import pytest



@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def dev(torch, a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()
    return t if dtype is None else t.to(dtype)


def grad_err(g, ref):
    g, ref = np.asarray(g, np.float64), np.asarray(ref, np.float64)
    scale = max(np.abs(ref).max(), 1e-300)
    return np.abs(g - ref) / np.maximum(np.abs(ref), 1e-3 * scale)


def seeds(torch, w, seed=11):
    rng = np.random.default_rng(seed)
    ntrk = w["nblocks"] * w["bsize"]
    g_trk = np.zeros((w["nblocks"], 28, w["bsize"]), np.float32)
    g_trk[:, 0:6, :] = rng.normal(size=(w["nblocks"], 6, w["bsize"]))
    g_trk[:, 6:27, :] = rng.normal(size=(w["nblocks"], 21, w["bsize"])) * 1e2
    g_chi2 = rng.uniform(0.5, 1.5, ntrk).astype(np.float32)
    dr = rng.uniform(-0.01, 0.01, w["nlayer"]).astype(np.float32)
    return g_trk, g_chi2, dr


def check_per_track(got, ref, what, tol=1e-10):
    for k in ("grad_trk_in", "grad_hits", "chi2", "trk_out"):
        a, b = got[k].cpu().numpy().reshape(-1), ref[k].cpu().numpy().reshape(-1)
        if k == "trk_out":  # the q row is integer bits: compare as such, the rest as values
            assert np.array_equal(np.isfinite(a), np.isfinite(b)), (what, k)
            fin = np.isfinite(a) & np.isfinite(b)
            a, b = a[fin], b[fin]
        e = grad_err(a, b)
        assert e.max() <= tol, (what, k, e.max())


def windowed_order(w, window=512):
    """The library's track order: within windows of floor(window / bsize) blocks of each event
    (window 0: whole events), tracks by layer count, longest first, ties in track order."""
    bs = w["bsize"]
    off = np.asarray(w["event_block_offset"], np.int64)
    nl = np.clip(np.asarray(w["nlay_lane"]), 0, w["nlayer"])
    wb = max(1, window // bs) if window > 0 else max(1, int(np.diff(off).max(initial=1)))
    perm = np.arange(w["nblocks"] * bs)
    for e in range(len(off) - 1):
        for b in range(off[e], off[e + 1], wb):
            a, z = b * bs, min(b + wb, off[e + 1]) * bs
            perm[a:z] = a + np.argsort(-nl[a:z], kind="stable")
    return perm


@pytest.fixture(scope="module")
def uneven(p2r):
    # 20 events, 5..400 tracks each, 10..20 layers per track (20 layer slots)
    counts = p2r.lognormal_counts(20, median=120, sigma=1.0, lo=5, hi=400, seed=21)
    return p2r.uneven_workload(counts, bsize=32, nlayer_max=20, lay_lo=10, lay_hi=20, seed=21)


@pytest.mark.gpu
def test_queue_adjoint_matches_grid_adjoint(p2r, torch, uneven):
    w = uneven
    g_trk, g_chi2, dr = seeds(torch, w)
    t, h = dev(torch, w["trk"]), dev(torch, w["hit"])
    gt, gc, d_dr = dev(torch, g_trk), dev(torch, g_chi2), dev(torch, dr)
    q = p2r.Queue(w, blocks_per_item=2)
    got = q.run_adjoint(t, h, dr=d_dr, grad_trk_out=gt, grad_chi2=gc)
    assert q.error_bits() == 0
    cfg = p2r.Config(bsize=32, nlayer=w["nlayer"], nevts=1, nb=w["nblocks"], bz=w["bz"])
    ref = p2r.forward_backward(cfg, t, h, dr=d_dr, nlay_lane=dev(torch, w["nlay_lane"]), grad_trk_out=gt,
                               grad_chi2=gc, ckpt_stride=1)
    torch.cuda.synchronize()
    check_per_track(got, ref, "uneven batch")
    for k in ("grad_dr", "grad_bz"):  # summed per event, then over events: another order
        assert grad_err(got[k].cpu().numpy(), ref[k].cpu().numpy()).max() < 1e-10, k
    # per-event sums add up to the totals
    ev = got["grad_dr_event"].sum(0)
    assert torch.allclose(ev, got["grad_dr"], rtol=1e-12, atol=0)


@pytest.mark.gpu
def test_queue_adjoint_per_event_equals_grid_path(p2r, torch):
    """Events of equal size: per-event dr / Bz gradients equal the grid adjoint's per-event sums
    (same per-slice partials, same fixed order) to 1e-12, as the calibration workload needs."""
    cfg = p2r.Config(bsize=32, nlayer=40, nevts=6, nb=5, bz=3.8)
    trk, hit = p2r.generate_helix(cfg, p2r.gen_params(bz=3.8, seed=44, r_first=4.0, r_last=110.0))
    rng = np.random.default_rng(44)
    nlay = rng.integers(20, 41, cfg.ntracks).astype(np.int32)
    off = np.arange(cfg.nevts + 1, dtype=np.int64) * cfg.nb
    w = dict(trk=trk, hit=hit, nlay_lane=nlay, event_block_offset=off, ntrk_event=np.full(cfg.nevts, cfg.nb * 32),
             nblocks=cfg.nblocks, bsize=32, nlayer=cfg.nlayer, bz=cfg.bz, updates=int(nlay.sum()))
    g_trk, g_chi2, dr = seeds(torch, w, seed=44)
    t, h = dev(torch, trk), dev(torch, hit)
    gt, gc, d_dr = dev(torch, g_trk), dev(torch, g_chi2), dev(torch, dr)
    q = p2r.Queue(w, blocks_per_item=3)
    got = q.run_adjoint(t, h, dr=d_dr, grad_trk_out=gt, grad_chi2=gc)
    ref = p2r.forward_backward(cfg, t, h, dr=d_dr, nlay_lane=dev(torch, nlay), grad_trk_out=gt, grad_chi2=gc,
                               ckpt_stride=1, per_event=True)
    torch.cuda.synchronize()
    check_per_track(got, ref, "40 layers")
    for k in ("grad_dr_event", "grad_bz_event", "grad_dr", "grad_bz"):
        a, b = got[k].cpu().numpy(), ref[k].cpu().numpy()
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max(), (k, np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.gpu
def test_queue_adjoint_matches_fp64_reference(p2r, torch):
    """The persistent adjoint against the FP64 reference gradient (torch autograd over the
    oracle's restatement) on a small uneven batch: every element within 1e-3."""
    from tests.test_adjoint_gpu import torch_reference
    counts = np.array([40, 7, 96, 33])
    w = p2r.uneven_workload(counts, bsize=32, nlayer_max=20, lay_lo=10, lay_hi=20, seed=5)
    g_trk, g_chi2, dr = seeds(torch, w, seed=5)
    q = p2r.Queue(w, blocks_per_item=1)
    got = q.run_adjoint(dev(torch, w["trk"]), dev(torch, w["hit"]), dr=dev(torch, dr), grad_trk_out=dev(torch, g_trk),
                        grad_chi2=dev(torch, g_chi2))
    torch.cuda.synchronize()
    cfg = p2r.Config(bsize=32, nlayer=w["nlayer"], nevts=1, nb=w["nblocks"], bz=w["bz"])
    ref = torch_reference(p2r, cfg, w["trk"], w["hit"], dr, g_trk, g_chi2, nlay=w["nlay_lane"])
    bs = 32
    gt = got["grad_trk_in"].cpu().numpy().reshape(cfg.nblocks, 28, bs)
    gh = got["grad_hits"].cpu().numpy().reshape(cfg.nblocks, cfg.nlayer, 9, bs)
    mine = dict(par0=gt[:, 0:6, :].transpose(0, 2, 1).reshape(-1, 6),
                cov0=gt[:, 6:27, :].transpose(0, 2, 1).reshape(-1, 21),
                hpos=gh[:, :, 0:3, :].transpose(0, 3, 1, 2).reshape(-1, cfg.nlayer, 3),
                hcov=gh[:, :, 3:9, :].transpose(0, 3, 1, 2).reshape(-1, cfg.nlayer, 6),
                dr=got["grad_dr"].cpu().numpy(), bz=float(got["grad_bz"].cpu().numpy()[0]))
    for key in ("par0", "cov0", "hpos", "hcov", "dr"):
        assert grad_err(mine[key], ref[key]).max() < 1e-3, key
    assert grad_err([mine["bz"]], [ref["bz"]])[0] < 1e-3


@pytest.mark.gpu
def test_queue_adjoint_graph_replay_and_small_workspace(p2r, torch, uneven):
    """The captured graph's replays equal the direct call bit for bit; a workspace holding only
    one CTA's tapes (fewer CTAs, the same per-slice arithmetic) gives the same results."""
    w = uneven
    g_trk, g_chi2, dr = seeds(torch, w)
    t, h = dev(torch, w["trk"]), dev(torch, w["hit"])
    gt, gc, d_dr = dev(torch, g_trk), dev(torch, g_chi2), dev(torch, dr)
    q = p2r.Queue(w, blocks_per_item=4)
    direct = {k: v.clone() for k, v in q.run_adjoint(t, h, dr=d_dr, grad_trk_out=gt, grad_chi2=gc).items()
              if k != "workspace"}
    o = q.capture_adjoint(t, h, dr=d_dr, grad_trk_out=gt, grad_chi2=gc)
    for _ in range(2):
        for v in o.values():
            if v is not None and v.dtype != torch.uint8:
                v.fill_(float("nan"))
        q.replay()
        torch.cuda.synchronize()
        for k, v in direct.items():
            assert torch.equal(o[k].view(torch.int32) if o[k].dtype == torch.float32 else o[k].view(torch.int64),
                               v.view(torch.int32) if v.dtype == torch.float32 else v.view(torch.int64)), k
    q.release()
    # a workspace with one CTA's tapes (4 warps): the sums, then 4 tapes and a little slack
    nout, nslices = w["nlayer"] + 1, w["nblocks"]
    a256 = lambda x: (x + 255) // 256 * 256
    tape_off = a256(a256(a256(256 + nslices * nout * 8) + q.nevts * nout * 8) + nout * 8)
    per_warp = w["nlayer"] * 27 * 32 * 8
    full = q.adjoint_workspace_size()
    small_ws = torch.empty(tape_off + 4 * per_warp + per_warp // 2, dtype=torch.uint8, device="cuda")
    assert small_ws.numel() < full
    q2 = p2r.Queue(w, blocks_per_item=4)
    small = {}
    args = q2._adjoint_args(t, h, d_dr, gt, gc, small)[:-2] + (small_ws.data_ptr(), small_ws.numel())
    del small["workspace"]
    lib = p2r.lib()
    from p2r_tests_b200.api import _stream
    rc = lib.p2r_run_queue_adjoint(ctypes.byref(q2.q), *args, _stream(None))
    assert rc == 0, lib.p2r_last_error_string().decode()
    torch.cuda.synchronize()
    for k, v in direct.items():
        a = small[k]
        assert torch.equal(a.view(torch.int32) if a.dtype == torch.float32 else a.view(torch.int64),
                           v.view(torch.int32) if v.dtype == torch.float32 else v.view(torch.int64)), k
    # too small for even one CTA: rejected before any launch
    tiny = torch.empty(tape_off + per_warp, dtype=torch.uint8, device="cuda")
    args = args[:-2] + (tiny.data_ptr(), tiny.numel())
    assert lib.p2r_run_queue_adjoint(ctypes.byref(q2.q), *args, _stream(None)) == p2r._lib.P2R_ERR_WORKSPACE


@pytest.mark.gpu
def test_queue_adjoint_skips_malformed_items(p2r, torch, uneven):
    """Items are device data: an out-of-range one is skipped and reported, its blocks untouched;
    every buffer is a real allocation and the out-of-range values are only compared."""
    w = uneven
    t, h = dev(torch, w["trk"]), dev(torch, w["hit"])
    q = p2r.Queue(w, blocks_per_item=2)
    items = q.d_items.cpu().numpy().view(np.dtype([("event", np.int32), ("nblk", np.int32), ("block0", np.int64)]))
    bad = items.copy()
    bad[0]["block0"] = w["nblocks"] + 100
    q.d_items.copy_(torch.from_numpy(bad.view(np.uint8).copy()))
    o = {"grad_trk_in": torch.full_like(t, float("nan"))}
    q.run_adjoint(t, h, grad_chi2=torch.ones(w["nblocks"] * 32, device="cuda"), out=o)
    assert q.error_bits() == 2
    g = o["grad_trk_in"].cpu().numpy().reshape(w["nblocks"], 28, 32)
    b0, n = int(items[0]["block0"]), int(items[0]["nblk"])
    assert np.isnan(g[b0:b0 + n]).all()
    assert np.isfinite(g[b0 + n:]).all()


@pytest.mark.usefixtures("host_only")
def test_queue_adjoint_rejects_options(p2r):
    """Host-side checks (no device work): option flags and more than 64 layers are rejected."""
    l = p2r.lib()
    for flags in (p2r.FLAG_ADJ_FP32, p2r.FLAG_SQUASH_PHI, p2r.FLAG_FP32_DET):
        q = p2r._lib.CQueue(32, 20, 1, 0, 3.8, flags, 0, 0, 0, None, None, 0, None)
        assert l.p2r_queue_adjoint_workspace_size(ctypes.byref(q)) == 0
        assert l.p2r_run_queue_adjoint(ctypes.byref(q), *([None] * 14), 0, None) == p2r._lib.P2R_ERR_UNSUPPORTED
    q = p2r._lib.CQueue(32, 65, 1, 0, 3.8, 0, 0, 0, 0, None, None, 0, None)
    assert l.p2r_run_queue_adjoint(ctypes.byref(q), *([None] * 14), 0, None) == p2r._lib.P2R_ERR_UNSUPPORTED


@pytest.mark.gpu
def test_queue_adjoint_ordered_by_layers(p2r, torch, uneven):
    """P2R_FLAG_ORDER_BY_LAYERS: the launch orders each event's tracks by layer count on the
    device, over whole events (the order equals windowed_order's), every output stays
    at its track's position and per-track results equal the unordered launch's; the shared sums
    are added in the new grouping (equal to 1e-9)."""
    w = uneven
    g_trk, g_chi2, dr = seeds(torch, w)
    t, h = dev(torch, w["trk"]), dev(torch, w["hit"])
    gt, gc, d_dr = dev(torch, g_trk), dev(torch, g_chi2), dev(torch, dr)
    plain = p2r.Queue(w, blocks_per_item=2).run_adjoint(t, h, dr=d_dr, grad_trk_out=gt, grad_chi2=gc)
    q = p2r.Queue(w, blocks_per_item=2, flags=p2r.FLAG_ORDER_BY_LAYERS)
    got = q.run_adjoint(t, h, dr=d_dr, grad_trk_out=gt, grad_chi2=gc)
    assert q.error_bits() == 0
    torch.cuda.synchronize()
    # the device order, read from its place in the workspace
    nout, nslices = w["nlayer"] + 1, w["nblocks"]
    a256 = lambda x: (x + 255) // 256 * 256
    order_off = a256(a256(256 + nslices * nout * 8) + q.nevts * nout * 8)
    order_off = a256(order_off + nout * 8)
    ntr = w["nblocks"] * 32
    order = got["workspace"][order_off:order_off + 4 * ntr].cpu().numpy().view(np.uint32)
    assert np.array_equal(order.astype(np.int64), windowed_order(w, window=0))
    check_per_track(got, plain, "ordered", tol=0.0)
    for k in ("grad_dr", "grad_bz", "grad_dr_event", "grad_bz_event"):
        a, b = got[k].cpu().numpy(), plain[k].cpu().numpy()
        assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max(), k
