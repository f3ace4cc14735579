"""Uneven batches: work-item planning (CPU) and the persistent queue launch (GPU)."""
import ctypes

import numpy as np
import pytest

from tests import parity


def test_plan_splits_events_in_order(p2r):
    off = np.array([0, 5, 5, 12, 13], np.int64)  # event 1 is empty
    items = p2r.plan(off, 3)
    assert [tuple(x) for x in items] == [(0, 3, 0), (0, 2, 3), (2, 3, 5), (2, 3, 8), (2, 1, 11), (3, 1, 12)]
    assert sum(int(x["nblk"]) for x in items) == 13


def test_plan_rejects_bad_offsets(p2r):
    l = p2r.lib()
    off = np.array([0, 4, 2], np.int64)
    assert l.p2r_queue_plan(off.ctypes.data, 2, 2, None, 0) < 0
    off = np.array([0, 4, 8], np.int64)
    assert l.p2r_queue_plan(off.ctypes.data, 2, 0, None, 0) < 0
    buf = (p2r._lib.CQueueItem * 1)()
    assert l.p2r_queue_plan(off.ctypes.data, 2, 2, ctypes.addressof(buf), 1) < 0  # capacity


def test_queue_rejects_bad_description(p2r):
    l = p2r.lib()
    q = p2r._lib.CQueue(48, 25, 1, 1, 3.8, 0, 0, 0, 0, None, None, 0, None)  # bsize not a multiple of 32
    assert l.p2r_run_queue(ctypes.byref(q), None, None, None, None, None, None, None, 0, None) == p2r._lib.P2R_ERR_QUEUE
    q = p2r._lib.CQueue(32, 25, 1, 4, 3.8, 0, 0, 0, 0, None, None, 1, None)  # blocks but no arrays
    assert l.p2r_run_queue(ctypes.byref(q), None, None, None, None, None, None, None, 0, None) == p2r._lib.P2R_ERR_QUEUE
    # the Python description is checked before anything reaches the device
    w = p2r.uneven_workload(np.array([33, 64, 1, 50]), bsize=32)
    bad = [dict(w, event_block_offset=np.array([1, 2, 4, 5, 7])), dict(w, event_block_offset=np.array([0, 2, 4, 5, 6])),
           dict(w, event_block_offset=np.array([0, 4, 2, 5, 7])), dict(w, nlay_lane=w["nlay_lane"][:-1]),
           dict(w, ntrk_event=w["ntrk_event"][:-1])]
    for b in bad:
        with pytest.raises(ValueError):
            p2r.Queue(b, device="cpu")


def test_uneven_workload_padding(p2r):
    w = p2r.uneven_workload(np.array([33, 64, 1, 50]), bsize=32)
    assert list(w["event_block_offset"]) == [0, 2, 4, 5, 7]
    nl = w["nlay_lane"].reshape(-1, 32)
    assert (nl[1, 1:] == 0).all() and (nl[1, 0] > 0)  # event 0: 33 tracks -> 1 live lane in block 1
    assert (nl[4, 1:] == 0).all()                     # event 2: 1 track
    assert ((nl[0] >= 10) & (nl[0] <= 25)).all()
    assert w["updates"] == int(nl.sum())


def test_sort_by_layers_permutation(p2r):
    """Ordering by layer count permutes tracks within events only, longest first, and
    permute_tracks with the inverse restores the arrays exactly."""
    w = p2r.uneven_workload(p2r.lognormal_counts(6, median=70, sigma=0.8, lo=5, hi=300, seed=5), bsize=32)
    ws, perm = p2r.sort_by_layers(w)
    off = w["event_block_offset"] * 32
    for e in range(len(off) - 1):
        seg = perm[off[e]:off[e + 1]]
        assert seg.min() >= off[e] and seg.max() < off[e + 1]
        nl = ws["nlay_lane"][off[e]:off[e + 1]]
        assert (np.diff(nl) <= 0).all()
    inv = p2r.inverse(perm)
    bits = lambda a: np.ascontiguousarray(a).view(np.uint32)  # the q row holds integer bits
    assert np.array_equal(bits(p2r.permute_tracks(ws["trk"], inv, 32, 28)), bits(w["trk"]))
    assert np.array_equal(bits(p2r.permute_tracks(ws["hit"], inv, 32, 9, w["nlayer"])), bits(w["hit"]))
    assert np.array_equal(ws["nlay_lane"][inv], w["nlay_lane"])
    assert int(ws["nlay_lane"].sum()) == w["updates"]


# ------------------------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()


@pytest.fixture(scope="module")
def small_batch(p2r):
    return p2r.uneven_workload(p2r.lognormal_counts(24, median=150, sigma=1.0, lo=5, hi=2000, seed=3), bsize=32)


@pytest.mark.gpu
@pytest.mark.parametrize("g,flags", [(1, 0), (4, 0), (16, 0), (4, "squash"), (4, "chi2"), (1, "order"), (8, "order"),
                                     (20, "order"), (8, "order+squash"), (8, "order+chi2"), (3, "order4"),
                                     (8, "order4+chi2")])
def test_queue_matches_masked_forward(p2r, torch, small_batch, g, flags):
    """The persistent queue performs the masked fused forward's operations: bit-identical
    tracks and chi2 (also with phi wrapped after every update, and with each CTA's tracks ordered
    by layer count: P2R_FLAG_ORDER_BY_LAYERS)."""
    w = small_batch
    fl = (p2r.FLAG_SQUASH_PHI if "squash" in str(flags) else 0) | (p2r.FLAG_ORDER_BY_LAYERS if "order" in str(flags)
                                                                   else 0)
    q = p2r.Queue(w, blocks_per_item=g, flags=fl, block_threads=128 if "order4" in str(flags) else 0)
    t, h = dev(torch, w["trk"]), dev(torch, w["hit"])
    out = torch.empty_like(t)
    with_chi2 = "chi2" in str(flags)
    ntrk = w["nblocks"] * w["bsize"]
    c2 = torch.full((ntrk,), float("nan"), device="cuda") if with_chi2 else None
    q.run(t, h, out, c2)
    cfg = p2r.Config(bsize=32, nlayer=w["nlayer"], nevts=1, nb=w["nblocks"], bz=w["bz"],
                     flags=fl & ~p2r.FLAG_ORDER_BY_LAYERS)
    ref = torch.empty_like(t)
    rc2 = torch.zeros(ntrk, device="cuda") if with_chi2 else None
    p2r.forward(cfg, t, h, ref, chi2=rc2, nlay_lane=dev(torch, w["nlay_lane"]))
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.cpu().numpy().view(np.uint32)), (g, flags)
    if with_chi2:
        assert np.array_equal(c2.cpu().numpy().view(np.uint32), rc2.cpu().numpy().view(np.uint32)), (g, flags)
    lat = q.event_latency_ns()
    assert (lat > 0).all() and (lat < 10_000_000_000).all()


@pytest.mark.gpu
def test_queue_granularity_bit_identical(p2r, torch, small_batch):
    w = small_batch
    t, h = dev(torch, w["trk"]), dev(torch, w["hit"])
    outs = []
    for g in (1, 3, 64):
        o = torch.empty_like(t)
        p2r.Queue(w, blocks_per_item=g).run(t, h, o)
        outs.append(o.cpu().numpy().view(np.uint32))
    assert all(np.array_equal(outs[0], o) for o in outs[1:])


@pytest.mark.gpu
def test_queue_matches_reference(p2r, oracle, torch, small_batch):
    from oracle.oracle import RefTBB, ref_available
    if not ref_available(32, "kf"):
        pytest.skip("reference build not present")
    w = small_batch
    ref = RefTBB(32, "kf")
    ref.set_bz(w["bz"])
    want = ref.run_masked(w["trk"], w["hit"], w["nlayer"], w["nlay_lane"])
    t, h = dev(torch, w["trk"]), dev(torch, w["hit"])
    out = torch.empty_like(t)
    p2r.Queue(w, blocks_per_item=4).run(t, h, out)
    torch.cuda.synchronize()
    f64 = oracle.run(w["trk"], w["hit"], 32, w["nlayer"], 1, w["bz"], "f64", nlay_lane=w["nlay_lane"])
    got = out.cpu().numpy()
    live = w["nlay_lane"] > 0
    sel = lambda a: a.reshape(-1, 28, 32).transpose(0, 2, 1).reshape(-1, 28)[live].reshape(-1, 1, 28).transpose(0, 2, 1).reshape(-1)
    # compare live tracks only (padding lanes keep their input), as 1-lane blocks
    parity.assert_accuracy_parity(sel(got), sel(want), f64["par"][live], f64["cov"][live], f64["prior"][live], 1,
                                  "queue vs reference (masked)")
    # padding lanes are returned unchanged
    pad = ~live
    a = got.reshape(-1, 28, 32).transpose(0, 2, 1).reshape(-1, 28)[pad]
    b = w["trk"].reshape(-1, 28, 32).transpose(0, 2, 1).reshape(-1, 28)[pad]
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.gpu
def test_queue_sorted_by_layers_same_results(p2r, torch, small_batch):
    """The same tracks ordered by layer count give bit-identical results per track."""
    w = small_batch
    ws, perm = p2r.sort_by_layers(w)
    outs = []
    for wl in (w, ws):
        q = p2r.Queue(wl, blocks_per_item=4)
        t, h = dev(torch, wl["trk"]), dev(torch, wl["hit"])
        o = torch.empty_like(t)
        q.run(t, h, o)
        torch.cuda.synchronize()
        outs.append(o.cpu().numpy())
    back = p2r.permute_tracks(outs[1], p2r.inverse(perm), 32, 28)
    assert np.array_equal(back.view(np.uint32).reshape(-1), outs[0].view(np.uint32).reshape(-1))


@pytest.mark.gpu
def test_queue_graph_replay(p2r, torch, small_batch):
    w = small_batch
    q = p2r.Queue(w, blocks_per_item=2)
    t, h = dev(torch, w["trk"]), dev(torch, w["hit"])
    direct = torch.empty_like(t)
    q.run(t, h, direct)
    out = torch.zeros_like(t)
    chi2 = torch.zeros(w["nblocks"] * 32, dtype=torch.float32, device="cuda")
    q.capture(t, h, out, chi2)
    for _ in range(3):
        out.zero_()
        q.replay()
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), direct.cpu().numpy().view(np.uint32))
    lat = q.event_latency_ns()
    assert (lat > 0).all()
    assert np.isfinite(chi2.cpu().numpy()).all()
    q.release()


@pytest.mark.gpu
def test_queue_empty_events_and_tiny(p2r, torch):
    w = p2r.uneven_workload(np.array([0, 1, 0, 40, 0]), bsize=32)
    q = p2r.Queue(w, blocks_per_item=1)
    t, h = dev(torch, w["trk"]), dev(torch, w["hit"])
    out = torch.empty_like(t)
    q.run(t, h, out)
    torch.cuda.synchronize()
    lat = q.event_latency_ns()
    assert (lat[[1, 3]] > 0).all()  # events with blocks complete; empty events have no slices
    assert np.isfinite(p2r.tracks_par(out.cpu().numpy().reshape(-1, 28, 32))[w["nlay_lane"] > 0]).all()


@pytest.mark.gpu
@pytest.mark.parametrize("bs,order", [(64, False), (128, False), (64, True), (96, True), (256, True)])
def test_queue_wide_blocks(p2r, torch, bs, order):
    w = p2r.uneven_workload(p2r.lognormal_counts(6, median=300, lo=5, hi=2000, seed=5), bsize=bs)
    t, h = dev(torch, w["trk"]), dev(torch, w["hit"])
    out, ref = torch.empty_like(t), torch.empty_like(t)
    p2r.Queue(w, blocks_per_item=2, flags=p2r.FLAG_ORDER_BY_LAYERS if order else 0).run(t, h, out)
    cfg = p2r.Config(bsize=bs, nlayer=w["nlayer"], nevts=1, nb=w["nblocks"], bz=w["bz"])
    p2r.forward(cfg, t, h, ref, nlay_lane=dev(torch, w["nlay_lane"]))
    torch.cuda.synchronize()
    parity.assert_same_arithmetic(out.cpu().numpy(), ref.cpu().numpy(), bs, f"queue bsize {bs}")


@pytest.mark.gpu
def test_queue_skips_and_reports_malformed_items(p2r, torch, small_batch):
    """Work items and event offsets are device data: the kernel range-checks each one before
    use, skips a bad one and reports it (p2r_queue_error). Every buffer here is a real
    allocation of the right size; the out-of-range values are only ever compared, never used
    as an index (checked by reading the kernel). The good items' outputs are bit-identical to
    the masked forward's, the bad items' blocks are left untouched."""
    w = small_batch
    q = p2r.Queue(w, blocks_per_item=2)
    t, h = dev(torch, w["trk"]), dev(torch, w["hit"])
    out = torch.full_like(t, float("nan"))
    q.run(t, h, out)
    assert q.error_bits() == 0
    items = q.d_items.cpu().numpy().view(np.dtype([("event", np.int32), ("nblk", np.int32), ("block0", np.int64)]))
    bad = items.copy()
    nev, nblocks = q.nevts, w["nblocks"]
    bad[1]["event"] = nev + 3                       # event out of range
    bad[2]["block0"] = nblocks + 5                  # blocks past the end
    bad[3]["nblk"] = -1                             # negative count
    off = w["event_block_offset"]
    bad[4]["event"] = (int(bad[4]["event"]) + 1) % nev  # in range, but not the event owning its blocks
    skipped = [1, 2, 3, 4]
    q.d_items.copy_(torch.from_numpy(bad.view(np.uint8).copy()))
    out2 = torch.full_like(t, float("nan"))
    q.run(t, h, out2)
    assert q.error_bits() == 1 | 2 | 4
    ref = torch.empty_like(t)
    cfg = p2r.Config(bsize=32, nlayer=w["nlayer"], nevts=1, nb=w["nblocks"], bz=w["bz"])
    p2r.forward(cfg, t, h, ref, nlay_lane=dev(torch, w["nlay_lane"]))
    torch.cuda.synchronize()
    o2 = out2.cpu().numpy().reshape(nblocks, 28, 32)
    r = ref.cpu().numpy().reshape(nblocks, 28, 32)
    untouched = np.zeros(nblocks, bool)
    for i in skipped:
        b0, n = int(items[i]["block0"]), int(items[i]["nblk"])
        untouched[b0:b0 + n] = True
    assert np.isnan(o2[untouched]).all()
    assert np.array_equal(o2[~untouched].view(np.uint32), r[~untouched].view(np.uint32))
    # decreasing event offsets are reported too (their events' items still run in range)
    q.d_items.copy_(torch.from_numpy(items.view(np.uint8).copy()))
    d_off = q.d_off.clone()
    o = off.copy()
    o[1] = -1
    q.d_off.copy_(torch.from_numpy(np.ascontiguousarray(o, np.int64)))
    q.run(t, h, torch.empty_like(t))
    assert q.error_bits() & 8
    q.d_off.copy_(d_off)
    q.run(t, h, torch.empty_like(t))
    assert q.error_bits() == 0


@pytest.mark.gpu
def test_uneven_batch_full_size(p2r, oracle, torch):
    """The 1000-event uneven batch at full size (log-normal tracks per event, median 2000,
    10-25 layers per track; 2.9e6 tracks, 5.0e7 updates) through the launch the benchmark
    times: the ordered persistent queue (bsize 32, 8 blocks per item, 4-warp CTAs) replayed from
    its CUDA graph. Size-independent properties: every track and chi2 bit-identical to the masked
    fused forward over the same arrays, padding lanes returned unchanged, no queue error; and on the
    first 40 events (7.4e4 tracks) accuracy parity with the reference's own masked chain
    against the FP64 oracle."""
    from oracle.oracle import RefTBB, ref_available
    w = p2r.uneven_workload(p2r.lognormal_counts(1000, median=2000, sigma=1.0, lo=50, hi=20000, seed=7), bsize=32,
                            nlayer_max=25)
    q = p2r.Queue(w, blocks_per_item=8, block_threads=128, flags=p2r.FLAG_ORDER_BY_LAYERS)
    t, h = dev(torch, w["trk"]), dev(torch, w["hit"])
    out = torch.full_like(t, float("nan"))
    ntrk = w["nblocks"] * w["bsize"]
    c2 = torch.full((ntrk,), float("nan"), device="cuda")
    q.capture(t, h, out, c2)
    q.replay()
    q.replay()
    torch.cuda.synchronize()
    assert q.error_bits() == 0
    q.release()
    ref = torch.empty_like(t)
    rc2 = torch.zeros(ntrk, device="cuda")
    cfg = p2r.Config(bsize=32, nlayer=w["nlayer"], nevts=1, nb=w["nblocks"], bz=w["bz"])
    p2r.forward(cfg, t, h, ref, chi2=rc2, nlay_lane=dev(torch, w["nlay_lane"]))
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    del t, h, out
    assert np.array_equal(got.view(np.uint32), ref.cpu().numpy().view(np.uint32))
    assert np.array_equal(c2.cpu().numpy().view(np.uint32), rc2.cpu().numpy().view(np.uint32))
    del ref
    live = w["nlay_lane"] > 0
    lanes = lambda a: a.reshape(-1, 28, 32).transpose(0, 2, 1).reshape(-1, 28)
    assert np.array_equal(lanes(got)[~live].view(np.uint32), lanes(w["trk"])[~live].view(np.uint32))
    if not ref_available(32, "kf"):
        pytest.skip("reference build not present")
    nb = int(w["event_block_offset"][40])
    trk, hit = w["trk"].reshape(-1)[:nb * 28 * 32], w["hit"].reshape(-1)[:nb * w["nlayer"] * 9 * 32]
    nl = w["nlay_lane"][:nb * 32]
    r = RefTBB(32, "kf")
    r.set_bz(w["bz"])
    want = r.run_masked(trk, hit, w["nlayer"], nl)
    f64 = oracle.run(trk, hit, 32, w["nlayer"], 1, w["bz"], "f64", nlay_lane=nl)
    sl = nl > 0
    one = lambda a: lanes(a)[sl].reshape(-1, 1, 28).transpose(0, 2, 1).reshape(-1)
    parity.assert_accuracy_parity(one(got[:nb * 28 * 32]), one(want), f64["par"][sl], f64["cov"][sl],
                                  f64["prior"][sl], 1, "uneven batch, first 40 events, vs reference (masked)")
