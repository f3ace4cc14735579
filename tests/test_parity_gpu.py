"""GPU parity tests: the CUDA path (through the C ABI) against the reference's own CPU code.

Comparisons use the reference's compiled functions (oracle/_ref, built from
src/propagate-tor-test_tbb.cpp) where present, and the committed golden vectors it
produced otherwise; the FP64 restatement (oracle/) measures accuracy. Tolerances and
metrics: tests/parity.py.
"""
import ctypes

import numpy as np
import pytest

from tests import parity

pytestmark = pytest.mark.gpu

MODES = {"restart": 0, "chained": 1}


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()


def host(t):
    return t.cpu().numpy()


def gpu_forward(p2r, torch, cfg, trk, hit, chi2=False, dr=None, nlay_lane=None):
    dt, dh = dev(torch, trk), dev(torch, hit)
    out = torch.empty_like(dt)
    c2 = torch.zeros(cfg.ntracks, dtype=torch.float32, device="cuda") if chi2 else None
    ddr = None if dr is None else dev(torch, np.asarray(dr, np.float32))
    dnl = None if nlay_lane is None else dev(torch, np.asarray(nlay_lane, np.int32))
    p2r.forward(cfg, dt, dh, out, chi2=c2, dr=ddr, nlay_lane=dnl)
    torch.cuda.synchronize()
    return (host(out), host(c2)) if chi2 else host(out)


def ref_or_none(bs, kind):
    from oracle.oracle import RefTBB, ref_available
    return RefTBB(bs, kind) if ref_available(bs, kind) else None


def fixture(p2r, golden_dir, bs):
    g = dict(np.load(golden_dir / f"ref_fixture_b{bs}.npz"))
    fx = dict(np.load(golden_dir / "fixture.npz"))
    cfg = p2r.Config(bsize=bs, nlayer=int(g["nlayer"]), nevts=int(g["nevts"]), nb=int(g["nb"]), bz=p2r.REF_BZ)
    ctypes.CDLL("libc.so.6").srand(1)
    trk, hit = p2r.generate_fixture(fx["par"], fx["cov"], int(fx["q"]), fx["hits"], cfg, smear=1e-5)
    return cfg, trk, hit, g


def helix(p2r, nevts, nb, nlayer=20, bs=32, bz=3.8, seed=20240001):
    cfg = p2r.Config(bsize=bs, nlayer=nlayer, nevts=nevts, nb=nb, bz=bz)
    trk, hit = p2r.generate_helix(cfg, p2r.gen_params(bz=bz, seed=seed))
    return cfg, trk, hit


def slice_layer(hit, nblocks, nlayer, layer, bs):
    return np.ascontiguousarray(hit.reshape(nblocks, nlayer, 9, bs)[:, layer:layer + 1])


# ---------------------------------------------------------------------------- fixture
@pytest.mark.parametrize("bs", [32, 64, 128])
def test_fixture_restart_matches_reference(p2r, oracle, torch, golden_dir, bs):
    cfg, trk, hit, g = fixture(p2r, golden_dir, bs)
    cfg.mode = p2r.MODE_RESTART
    out = gpu_forward(p2r, torch, cfg, trk, hit)
    f64 = oracle.run(trk, hit, bs, cfg.nlayer, 0, cfg.bz, "f64")
    parity.assert_elementwise(out, g["out_restart"], f64["prior"], bs, f"GPU restart b{bs} vs reference")


@pytest.mark.parametrize("bs", [32, 64, 128])
def test_fixture_chained_matches_reference(p2r, oracle, torch, golden_dir, bs):
    cfg, trk, hit, g = fixture(p2r, golden_dir, bs)
    out = gpu_forward(p2r, torch, cfg, trk, hit)
    f64 = oracle.run(trk, hit, bs, cfg.nlayer, 1, cfg.bz, "f64")
    tp, _, tq = parity.unpack(out, bs)
    _, _, rq = parity.unpack(g["out_chained"], bs)
    assert np.array_equal(tq, rq)
    assert np.isfinite(tp).all()
    parity.assert_accuracy_parity(out, g["out_chained"], f64["par"], f64["cov"], f64["prior"], bs,
                                  f"GPU chained b{bs} (fixture)", factor=4.0)


# ---------------------------------------------------------------------------- helix workload
@pytest.mark.parametrize("mode", list(MODES))
def test_helix_golden(p2r, oracle, torch, golden_dir, mode):
    g = dict(np.load(golden_dir / "ref_helix.npz"))
    bs, nl, bz = int(g["bsize"]), int(g["nlayer"]), float(g["bz"])
    cfg = p2r.Config(bsize=bs, nlayer=nl, nevts=int(g["nevts"]), nb=int(g["nb"]), bz=bz, mode=MODES[mode])
    out = gpu_forward(p2r, torch, cfg, g["trk"], g["hit"])
    f64 = oracle.run(g["trk"], g["hit"], bs, nl, MODES[mode], bz, "f64")
    if mode == "restart":
        parity.assert_elementwise(out, g["out_restart"], f64["prior"], bs, "GPU restart (helix golden)")
    else:
        parity.assert_accuracy_parity(out, g["out_chained"], f64["par"], f64["cov"], f64["prior"], bs,
                                      "GPU chained (helix golden)")


@pytest.mark.parametrize("bs", [32, 64, 128])
@pytest.mark.parametrize("mode", list(MODES))
def test_helix_vs_live_reference(p2r, oracle, torch, bs, mode):
    ref = ref_or_none(bs, "kf")
    if ref is None:
        pytest.skip("reference build not present")
    nb = 9600 // bs // 10  # 960 tracks per event
    cfg, trk, hit = helix(p2r, 4, nb, bs=bs)
    cfg.mode = MODES[mode]
    ref.set_bz(cfg.bz)
    rout = ref.run(trk, hit, cfg.nevts, cfg.nb, cfg.nlayer, chained=bool(MODES[mode]))
    out = gpu_forward(p2r, torch, cfg, trk, hit)
    f64 = oracle.run(trk, hit, bs, cfg.nlayer, MODES[mode], cfg.bz, "f64")
    if mode == "restart":
        parity.assert_elementwise(out, rout, f64["prior"], bs, f"GPU restart b{bs} vs live reference")
    else:
        tp, tc, _ = parity.unpack(out, bs)
        rp, rc, _ = parity.unpack(rout, bs)
        ep = parity.rel_par(tp, rp)
        ec = parity.rel_cov(tc, rc, f64["prior"])
        assert np.quantile(ep, 0.99) <= parity.PAR_RTOL
        assert np.quantile(ec, 0.99) <= parity.CHAIN_COV_P99
        parity.assert_accuracy_parity(out, rout, f64["par"], f64["cov"], f64["prior"], bs,
                                      f"GPU chained b{bs} vs live reference")


def test_stated_bar_fractions_config1_sample(p2r, oracle, torch):
    """The stated bar (relative 1e-4 on parameters, 1e-3 on covariance) at the benchmark
    workload's shape, counted element by element on 3 events x 9600 tracks x 20 layers:
    the fraction of elements beyond the bar for this library against the FP64 oracle is at most
    the reference's own (its FP32 chain against FP64), and this library's fraction beyond the
    bar against the live reference is within 10 % of the reference's own against FP64 (the two
    FP32 chains disagree about as often as the reference disagrees with the exact result)."""
    ref = ref_or_none(32, "kf")
    if ref is None:
        pytest.skip("reference build not present")
    cfg, trk, hit = helix(p2r, 3, 300)
    ref.set_bz(cfg.bz)
    rout = ref.run(trk, hit, cfg.nevts, cfg.nb, cfg.nlayer, chained=True, niter=1, nthreads=8)
    out = gpu_forward(p2r, torch, cfg, trk, hit)
    f64 = oracle.run(trk, hit, 32, cfg.nlayer, 1, cfg.bz, "f64")
    fin = np.isfinite(f64["par"]).all(1)
    tp, tc, _ = parity.unpack(out, 32)
    rp, rc, _ = parity.unpack(rout, 32)

    def frac(p, c, P, C):
        ep = parity.rel_par(p[fin], P[fin])
        ec = parity.rel_cov(c[fin], C[fin], f64["prior"][fin])
        return float((ep > parity.PAR_RTOL).mean()), float((ec > parity.COV_RTOL).mean())

    gpu = frac(tp, tc, f64["par"], f64["cov"])
    refv = frac(rp, rc, f64["par"], f64["cov"])
    cross = frac(tp, tc, rp, rc)
    assert gpu[0] <= refv[0] and gpu[1] <= refv[1], (gpu, refv)
    assert cross[0] <= 1.1 * refv[0] and cross[1] <= 1.1 * refv[1], (cross, refv)


def test_chained_step_parity_along_the_chain(p2r, oracle, torch):
    """Every step of a chained run: reference state after layer l-1 in, one GPU propagate +
    update with layer l, compared element-wise with the reference's state after layer l."""
    ref = ref_or_none(32, "kf")
    if ref is None:
        pytest.skip("reference build not present")
    cfg, trk, hit = helix(p2r, 2, 8)
    ref.set_bz(cfg.bz)
    nbk = cfg.nblocks
    state = np.ascontiguousarray(trk.reshape(-1))
    for l in range(cfg.nlayer):
        h1 = slice_layer(hit, nbk, cfg.nlayer, l, 32)
        want = ref.run(state, h1, cfg.nevts, cfg.nb, 1, chained=True)
        c1 = p2r.Config(bsize=32, nlayer=1, nevts=cfg.nevts, nb=cfg.nb, bz=cfg.bz)
        got = gpu_forward(p2r, torch, c1, state, h1)
        f64 = oracle.run(state, h1, 32, 1, 1, cfg.bz, "f64")
        parity.assert_step(got, want, f64["par"], f64["cov"], f64["prior"], 32, f"step {l}")
        state = want


@pytest.mark.parametrize("mode", list(MODES))
def test_per_layer_calls_match_reference_steps(p2r, oracle, torch, mode):
    """p2r_propagate_to_r / p2r_kalman_update: the reference's call shape, layer by layer."""
    ref = ref_or_none(32, "kf")
    if ref is None:
        pytest.skip("reference build not present")
    cfg, trk, hit = helix(p2r, 2, 8)
    cfg.mode = MODES[mode]
    ref.set_bz(cfg.bz)
    nbk = cfg.nblocks
    dt, dh = dev(torch, trk), dev(torch, hit)
    out = torch.empty_like(dt)
    out.copy_(dt)
    state = np.ascontiguousarray(trk.reshape(-1))
    for l in range(cfg.nlayer):
        src = dt if mode == "restart" else out
        p2r.propagateToR(cfg, src, dh, l, out)
        p2r.KalmanUpdate(cfg, out, dh, l)
        h1 = slice_layer(hit, nbk, cfg.nlayer, l, 32)
        inp = trk.reshape(-1) if mode == "restart" else state
        want = ref.run(inp, h1, cfg.nevts, cfg.nb, 1, chained=True)
        f64 = oracle.run(inp, h1, 32, 1, 1, cfg.bz, "f64")
        got = host(out)
        parity.assert_step(got, want, f64["par"], f64["cov"], f64["prior"], 32, f"layer {l}")
        out.copy_(dev(torch, want))  # continue from the reference state (step parity)
        state = want


def test_propagate_alone_matches_reference_block(p2r, oracle, torch):
    """propagateToR alone (no update) against the reference's function on every block."""
    ref = ref_or_none(32, "kf")
    if ref is None:
        pytest.skip("reference build not present")
    cfg, trk, hit = helix(p2r, 1, 16)
    ref.set_bz(cfg.bz)
    dt, dh = dev(torch, trk), dev(torch, hit)
    out = torch.empty_like(dt)
    for l in (0, 7, 19):
        p2r.propagateToR(cfg, dt, dh, l, out)
        got = host(out).reshape(cfg.nblocks, 28, 32)
        want = np.empty_like(got)
        for b in range(cfg.nblocks):
            tb = np.ascontiguousarray(trk[b])
            hb = np.ascontiguousarray(hit[b * cfg.nlayer + l])
            ob = tb.copy()  # the reference's propagateToR writes par and cov only; q stays
            ref.l.ref_propagate_block(tb.ctypes.data, hb.ctypes.data, ob.ctypes.data)
            want[b] = ob
        h1 = slice_layer(hit, cfg.nblocks, cfg.nlayer, l, 32)
        f64 = oracle.run(trk, h1, 32, 1, 2, cfg.bz, "f64")  # propagation only
        # no update: the propagated covariance itself is the conditioning scale
        parity.assert_step(got, want, f64["par"], f64["cov"], f64["prior"], 32, f"propagate layer {l}")


# ---------------------------------------------------------------------------- internal consistency
def test_fused_chain_equals_per_layer_chain(p2r, torch):
    cfg, trk, hit = helix(p2r, 3, 10)
    fused = gpu_forward(p2r, torch, cfg, trk, hit)
    dt, dh = dev(torch, trk), dev(torch, hit)
    out = torch.empty_like(dt)
    p2r.run_layers(cfg, dt, dh, out)
    torch.cuda.synchronize()
    a, b = fused.view(np.int32).astype(np.int64), host(out).view(np.int32).astype(np.int64)
    ulps = np.abs(a - b)
    assert np.quantile(ulps, 0.99) <= 64, np.quantile(ulps, [0.5, 0.99, 1.0])


@pytest.mark.parametrize("bs", [32, 64, 128])
def test_staged_equals_plain_loads(p2r, torch, bs):
    cfg, trk, hit = helix(p2r, 2, 12 * 32 // bs, bs=bs)
    a = gpu_forward(p2r, torch, cfg, trk, hit)
    cfg.flags = p2r.FLAG_NO_STAGING
    b = gpu_forward(p2r, torch, cfg, trk, hit)
    # every operation is explicit (no compiler contraction): the variants are bit-identical
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), "staged vs plain loads"


@pytest.mark.parametrize("mode", ["restart", "chained"])
def test_squash_phi_option(p2r, torch, mode):
    """P2R_FLAG_SQUASH_PHI (the reference's commented-out squashPhiMPlex, TBB:635): phi stays in
    [-pi, pi] and equals the unwrapped phi modulo 2 pi; the other parameters agree to the
    parity tolerance (a wrapped phi changes the rounding of the next sin/cos), and the fused
    and per-layer paths give identical results with the option."""
    cfg, trk, hit = helix(p2r, 4, 30)
    cfg.mode = MODES[mode]
    a = gpu_forward(p2r, torch, cfg, trk, hit)
    cfg.flags = p2r.FLAG_SQUASH_PHI
    b = gpu_forward(p2r, torch, cfg, trk, hit)
    pa, pb = parity.unpack(a, 32)[0], parity.unpack(b, 32)[0]
    assert (np.abs(pb[:, 4]) <= np.pi + 1e-6).all()
    d = np.remainder(pa[:, 4] - pb[:, 4] + np.pi, 2 * np.pi) - np.pi
    assert np.abs(d).max() < 1e-4
    if mode == "chained":
        assert (np.abs(pa[:, 4]) > np.pi).sum() > 0  # some tracks crossed phi = +-pi
    other = [0, 1, 2, 3, 5]
    assert np.quantile(parity.rel_par(pb, pa)[:, other], 0.999) < parity.PAR_RTOL
    dt, dh = dev(torch, trk), dev(torch, hit)
    out = torch.empty_like(dt)
    p2r.run_layers(cfg, dt, dh, out)
    torch.cuda.synchronize()
    assert np.array_equal(host(out).view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("threads,stages", [(32, 2), (64, 4), (96, 4), (128, 2)])
def test_launch_shapes_identical(p2r, torch, threads, stages):
    """The same kernel instantiation under another launch shape is bit-identical."""
    cfg, trk, hit = helix(p2r, 2, 7)
    cfg.stages = stages
    base = gpu_forward(p2r, torch, cfg, trk, hit)
    cfg.block_threads = threads
    out = gpu_forward(p2r, torch, cfg, trk, hit)
    assert np.array_equal(base.view(np.uint32), out.view(np.uint32))


@pytest.mark.parametrize("bs_other", [1, 16, 64, 96])
def test_layout_independence(p2r, torch, bs_other):
    """Each track's result is independent of the Matriplex width it is stored in (indexing)."""
    cfg32, trk, hit = helix(p2r, 1, 6, bs=32)
    out32 = gpu_forward(p2r, torch, cfg32, trk, hit)
    ntr = cfg32.ntracks
    assert ntr % bs_other == 0
    nb = ntr // bs_other

    def relayout(a, words, nl, bs_from, bs_to):
        x = a.reshape(-1, nl, words, bs_from).transpose(0, 3, 1, 2).reshape(-1, nl, words)  # (ntr, nl, words)
        return np.ascontiguousarray(x.reshape(-1, bs_to, nl, words).transpose(0, 2, 3, 1))

    trk_o = relayout(trk, 28, 1, 32, bs_other)
    hit_o = relayout(hit, 9, cfg32.nlayer, 32, bs_other)
    cfgo = p2r.Config(bsize=bs_other, nlayer=cfg32.nlayer, nevts=1, nb=nb, bz=cfg32.bz)
    outo = gpu_forward(p2r, torch, cfgo, trk_o, hit_o)
    back = relayout(outo, 28, 1, bs_other, 32)
    parity.assert_same_arithmetic(back, out32, 32, f"bsize {bs_other} vs 32")


def test_deterministic_and_q_copied(p2r, torch):
    cfg, trk, hit = helix(p2r, 2, 50)
    a = gpu_forward(p2r, torch, cfg, trk, hit)
    b = gpu_forward(p2r, torch, cfg, trk, hit)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(parity.unpack(a, 32)[2], parity.unpack(trk, 32)[2])


def test_empty_and_single_block(p2r, torch):
    cfg = p2r.Config(bsize=32, nlayer=20, nevts=0, nb=4, bz=3.8)
    e = torch.empty(0, device="cuda")
    p2r.forward(cfg, e, e, torch.empty(0, device="cuda"))
    cfg, trk, hit = helix(p2r, 1, 1)
    out = gpu_forward(p2r, torch, cfg, trk, hit)
    assert np.isfinite(parity.unpack(out, 32)[0]).all()


def test_chi2_and_radius_offsets_match_oracle(p2r, oracle, torch):
    """chi2 and the radius offsets against the FP64 oracle, with the FP32 oracle as the yardstick:
    chi2 is computed from residuals of ~10 um at radii up to 100 cm, where an FP32 position
    carries ~8e-6 cm of rounding, so any FP32 chain has ~1e-3 (median) relative chi2 error."""
    cfg, trk, hit = helix(p2r, 2, 8)
    rng = np.random.default_rng(7)
    dr = rng.uniform(-0.01, 0.01, cfg.nlayer)  # +-100 um
    for mode in (0, 1):
        cfg.mode = mode
        out, chi2 = gpu_forward(p2r, torch, cfg, trk, hit, chi2=True, dr=dr.astype(np.float32))
        drd = dr.astype(np.float32).astype(np.float64)
        f64 = oracle.run(trk, hit, 32, cfg.nlayer, mode, cfg.bz, "f64", dr=drd)
        f32 = oracle.run(trk, hit, 32, cfg.nlayer, mode, cfg.bz, "f32", dr=drd)
        rel = np.abs(chi2 - f64["chi2"]) / np.maximum(np.abs(f64["chi2"]), 1.0)
        rel32 = np.abs(f32["chi2"] - f64["chi2"]) / np.maximum(np.abs(f64["chi2"]), 1.0)
        for q in (0.5, 0.9, 0.99):
            assert np.quantile(rel, q) <= 2 * np.quantile(rel32, q) + 1e-6, (q, np.quantile(rel, q), np.quantile(rel32, q))
        tp = parity.unpack(out, 32)[0]
        assert np.quantile(parity.rel_par(tp, f64["par"]), 0.99) < parity.PAR_RTOL


def test_masked_lanes_match_reference(p2r, oracle, torch):
    ref = ref_or_none(32, "kf")
    if ref is None:
        pytest.skip("reference build not present")
    cfg, trk, hit = helix(p2r, 2, 6, nlayer=25)
    ref.set_bz(cfg.bz)
    rng = np.random.default_rng(11)
    nl = rng.integers(10, 26, cfg.ntracks).astype(np.int32)
    nl[:32] = 25
    nl[32:64] = 0  # a block whose lanes all stop at once
    out = gpu_forward(p2r, torch, cfg, trk, hit, nlay_lane=nl)
    want = ref.run_masked(trk, hit, cfg.nlayer, nl)
    f64 = oracle.run(trk, hit, 32, cfg.nlayer, 1, cfg.bz, "f64", nlay_lane=nl)
    parity.assert_accuracy_parity(out, want, f64["par"], f64["cov"], f64["prior"], 32, "masked lanes")
    # lanes with 0 layers come back unchanged
    assert np.array_equal(out.reshape(-1, 28, 32)[1].view(np.uint32), trk.reshape(-1, 28, 32)[1].view(np.uint32))


def test_fp32_determinant_option(p2r, oracle, torch):
    cfg, trk, hit = helix(p2r, 2, 20)
    f64 = oracle.run(trk, hit, 32, cfg.nlayer, 1, cfg.bz, "f64")
    d64 = gpu_forward(p2r, torch, cfg, trk, hit)
    cfg.flags = p2r.FLAG_FP32_DET
    d32 = gpu_forward(p2r, torch, cfg, trk, hit)
    # measured: the FP32 determinant roughly doubles the covariance error at the 99.9th
    # percentile, which is why the default keeps it in FP64 (as TBB:457 does)
    parity.assert_accuracy_parity(d32, d64, f64["par"], f64["cov"], f64["prior"], 32, "FP32 determinant",
                                  factor=4.0)


def test_count_nonfinite(p2r, torch):
    cfg, trk, hit = helix(p2r, 1, 4)
    trk = trk.copy()
    trk.reshape(-1, 28, 32)[2, 3, 5] = np.inf  # 1/pT of one track
    out = gpu_forward(p2r, torch, cfg, trk, hit)
    assert p2r.count_nonfinite(dev(torch, out), cfg.nblocks, 32) == 1


@pytest.mark.slow
@pytest.mark.parametrize("mode", list(MODES))
def test_full_size_sample_vs_reference(p2r, oracle, torch, mode):
    """9600 tracks x 100 events x 20 layers on the GPU, chained and restart; 300 blocks checked
    against the reference: restart element-wise at the stated bar, chained by accuracy parity."""
    cfg, trk, hit = helix(p2r, 100, 300)
    cfg.mode = MODES[mode]
    out = gpu_forward(p2r, torch, cfg, trk, hit)
    assert np.isfinite(parity.unpack(out[: 600 * 28 * 32], 32)[0]).all()
    dt = dev(torch, out)
    assert p2r.count_nonfinite(dt, cfg.nblocks, 32) == 0
    ref = ref_or_none(32, "kf")
    if ref is None:
        return
    ref.set_bz(cfg.bz)
    sel = np.random.default_rng(3).choice(cfg.nblocks, 300, replace=False)
    t_s = np.ascontiguousarray(trk[sel])
    h_s = np.ascontiguousarray(hit.reshape(cfg.nblocks, cfg.nlayer, 9, 32)[sel])
    want = ref.run(t_s, h_s, 1, 300, cfg.nlayer, chained=bool(MODES[mode]))
    got = np.ascontiguousarray(out.reshape(cfg.nblocks, 28, 32)[sel])
    f64 = oracle.run(t_s, h_s, 32, cfg.nlayer, MODES[mode], cfg.bz, "f64")
    if mode == "restart":
        parity.assert_elementwise(got, want, f64["prior"], 32, "full size sample, restart")
    else:
        parity.assert_accuracy_parity(got, want, f64["par"], f64["cov"], f64["prior"], 32, "full size sample")


def test_arrays_beyond_32_bit_offsets(p2r, torch):
    """A batch whose hit array has more than 2^31 elements (60 events x 1e5 tracks x 40 layers,
    8.6 GB, generated on the device): the tracks of the last event, whose hit offsets need 64
    bits, come out bit-identical to the same event run alone, for the fused forward and the
    masked forward."""
    nevts, nb, nl = 60, 3125, 40
    cfg = p2r.Config(bsize=32, nlayer=nl, nevts=nevts, nb=nb, bz=3.8)
    gp = p2r.gen_params(bz=3.8, seed=777, r_first=4.0, r_last=110.0)
    trk, hit = p2r.generate_helix_device(cfg, gp)
    assert hit.numel() > 2**31
    out = torch.empty_like(trk)
    p2r.forward(cfg, trk, hit, out)
    per_t, per_h = trk.numel() // nevts, hit.numel() // nevts
    one = p2r.Config(bsize=32, nlayer=nl, nevts=1, nb=nb, bz=3.8)
    t1, h1 = trk[-per_t:].clone(), hit[-per_h:].clone()
    o1 = torch.empty_like(t1)
    p2r.forward(one, t1, h1, o1)
    assert torch.equal(out[-per_t:].view(torch.int32), o1.view(torch.int32))
    nlay = torch.randint(1, nl + 1, (cfg.ntracks,), dtype=torch.int32, device="cuda",
                         generator=torch.Generator("cuda").manual_seed(5))
    p2r.forward(cfg, trk, hit, out, nlay_lane=nlay)
    p2r.forward(one, t1, h1, o1, nlay_lane=nlay[-nb * 32:].clone())
    torch.cuda.synchronize()
    assert torch.equal(out[-per_t:].view(torch.int32), o1.view(torch.int32))
    del trk, hit, out


@pytest.mark.parametrize("mode", ["chained", "restart"])
@pytest.mark.parametrize("nchunks", [1, 3, 10])
def test_host_buffer_pipeline_equals_device_run(p2r, torch, nchunks, mode):
    """p2r_forward_host (chunks of events copied in, run and copied out on the library's stream
    pool) returns exactly the device-resident forward's result, chunk count above the event
    count included; in restart mode it copies only the last layer's hits (a strided copy)."""
    cfg, trk, hit = helix(p2r, 5, 6)
    cfg.mode = MODES[mode]
    want = gpu_forward(p2r, torch, cfg, trk, hit)
    h_t = torch.from_numpy(trk.reshape(-1).copy()).pin_memory()
    h_h = torch.from_numpy(hit.reshape(-1).copy()).pin_memory()
    h_o = torch.zeros_like(h_t).pin_memory()
    d_t, d_h, d_o = torch.empty_like(h_t, device="cuda"), torch.empty_like(h_h, device="cuda"), torch.empty_like(h_t, device="cuda")
    d_h.fill_(float("nan"))  # restart: layers that are not copied must not be read either
    p2r.forward_host(cfg, h_t.numpy(), h_h.numpy(), h_o.numpy(), d_t, d_h, d_o, nchunks=nchunks)
    torch.cuda.synchronize()
    assert np.array_equal(h_o.numpy().view(np.uint32), want.reshape(-1).view(np.uint32))
    copied = np.isfinite(d_h.cpu().numpy().reshape(cfg.nblocks, cfg.nlayer, -1)).all(2)
    assert copied[:, -1].all() and (copied[:, :-1].all() if mode == "chained" else not copied[:, :-1].any())


def test_host_buffer_pipeline_from_two_threads(p2r, torch):
    """Two host threads calling p2r_forward_host at once (each with its own buffers and
    stream) both get their device-run results."""
    import threading
    cases = []
    for seed in (11, 12):
        cfg = p2r.Config(bsize=32, nlayer=20, nevts=6, nb=8, bz=3.8)
        trk, hit = p2r.generate_helix(cfg, p2r.gen_params(bz=3.8, seed=seed))
        want = gpu_forward(p2r, torch, cfg, trk, hit)
        h_t = torch.from_numpy(trk.reshape(-1).copy()).pin_memory()
        h_h = torch.from_numpy(hit.reshape(-1).copy()).pin_memory()
        h_o = torch.zeros_like(h_t).pin_memory()
        dev_bufs = (torch.empty_like(h_t, device="cuda"), torch.empty_like(h_h, device="cuda"),
                    torch.empty_like(h_t, device="cuda"))
        cases.append((cfg, h_t, h_h, h_o, dev_bufs, torch.cuda.Stream(), want))
    errors = []

    def work(c):
        cfg, h_t, h_h, h_o, (d_t, d_h, d_o), s, _ = c
        try:
            for _ in range(5):
                p2r.forward_host(cfg, h_t.numpy(), h_h.numpy(), h_o.numpy(), d_t, d_h, d_o, nchunks=4, stream=s)
            s.synchronize()
        except Exception as exc:  # reported below
            errors.append(exc)

    threads = [threading.Thread(target=work, args=(c,)) for c in cases]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for c in cases:
        assert np.array_equal(c[3].numpy().view(np.uint32), c[6].reshape(-1).view(np.uint32))


EDGE_REGIMES = {"low_pt": dict(pt=1.0), "high_pt": dict(pt=50.0),
                "forward": dict(theta_min=0.1, theta_max=0.3), "backward": dict(theta_min=2.84, theta_max=3.04),
                "bz_2T": dict(bz=2.0), "bz_4.5T": dict(bz=4.5)}


@pytest.mark.parametrize("regime", list(EDGE_REGIMES))
@pytest.mark.parametrize("mode", list(MODES))
def test_edge_regimes_accuracy_vs_live_reference(p2r, oracle, torch, regime, mode):
    """Tracks outside the default workload's ranges: pT 1 and 50 GeV, polar angles near the
    beam axis (0.1-0.3 and 2.84-3.04 rad), and fields of 2 and 4.5 T. Against the FP64 oracle the GPU is at least as accurate
    as the reference's own CPU build at every error quantile (within ACC_FACTOR), over the tracks
    that all three keep finite, and keeps at least as many tracks finite up to 0.5 % of them (near
    the axis about 1 % of chained tracks go non-finite in the reference and in FP64 as well)."""
    ref = ref_or_none(32, "kf")
    if ref is None:
        pytest.skip("reference build not present")
    kw = dict(EDGE_REGIMES[regime])
    bz = kw.pop("bz", 3.8)
    cfg = p2r.Config(bsize=32, nlayer=20, nevts=2, nb=30, bz=bz, mode=MODES[mode])
    trk, hit = p2r.generate_helix(cfg, p2r.gen_params(bz=bz, seed=77, **kw))
    ref.set_bz(cfg.bz)
    rout = ref.run(trk, hit, cfg.nevts, cfg.nb, cfg.nlayer, chained=bool(MODES[mode]))
    out = gpu_forward(p2r, torch, cfg, trk, hit)
    f64 = oracle.run(trk, hit, 32, cfg.nlayer, MODES[mode], cfg.bz, "f64")
    tp, tc, tq = parity.unpack(out, 32)
    rp, rc, rq = parity.unpack(rout, 32)
    assert np.array_equal(tq, rq)
    fin = lambda p, c: np.isfinite(p).all(1) & np.isfinite(c).all(1)
    ft, fr = fin(tp, tc), fin(rp, rc)
    assert ft.mean() >= fr.mean() - 0.005, (regime, mode, ft.mean(), fr.mean())
    both = ft & fr & fin(f64["par"], f64["cov"])
    assert both.mean() > 0.98
    qt = parity.error_quantiles(tp[both], tc[both], f64["par"][both], f64["cov"][both], f64["prior"][both])
    qr = parity.error_quantiles(rp[both], rc[both], f64["par"][both], f64["cov"][both], f64["prior"][both])
    for what, a, b in (("param", qt[0], qr[0]), ("cov", qt[1], qr[1])):
        for q, x, y in zip(parity.ACC_QUANTILES, a, b):
            assert x <= parity.ACC_FACTOR * y + 1e-7, f"{regime} {mode} {what} q{q}: GPU {x:.3e} vs reference {y:.3e}"


def test_calibration_full_size_sampled_against_fp64(p2r, oracle, torch):
    """The 40-layer calibration workload at full size (1e5 tracks x 100 events, hits on
    r = 4..110 cm, 20-40 layers per track, generated on the device; 15.5 GB of inputs), masked
    fused forward; the FP64 oracle's error sampled on 1 % of the tracks (every 100th track block)
    and compared with the reference's own masked CPU run on the same tracks: the GPU is at least as
    accurate at every error quantile and keeps every sampled track finite that the reference does.
    The launch with the tracks ordered by layer count inside it (P2R_FLAG_ORDER_BY_LAYERS) gives
    every track bit for bit the same output."""
    from oracle.oracle import RefTBB, ref_available
    if not ref_available(32, "kf"):
        pytest.skip("reference build not present")
    cfg = p2r.Config(bsize=32, nlayer=40, nevts=100, nb=3125, bz=3.8)
    gp = p2r.gen_params(bz=3.8, seed=20240004, r_first=4.0, r_last=110.0)
    trk, hit = p2r.generate_helix_device(cfg, gp)
    nlay = torch.randint(20, 41, (cfg.ntracks,), dtype=torch.int32, device="cuda",
                         generator=torch.Generator("cuda").manual_seed(4))
    out = torch.empty_like(trk)
    p2r.forward(cfg, trk, hit, out, nlay_lane=nlay)
    # the same forward with each CTA's tracks ordered by layer count inside the launch: bit-identical
    ordered = torch.full_like(trk, float("nan"))
    p2r.forward(p2r.Config(**{**cfg.__dict__, "flags": cfg.flags | p2r.FLAG_ORDER_BY_LAYERS}), trk, hit, ordered,
                nlay_lane=nlay)
    torch.cuda.synchronize()
    assert torch.equal(ordered.view(torch.int32), out.view(torch.int32))
    del ordered
    blocks = torch.arange(0, cfg.nblocks, 100, device="cuda")
    t_s = trk.view(cfg.nblocks, -1)[blocks].cpu().numpy().reshape(-1)
    h_s = hit.view(cfg.nblocks, -1)[blocks].cpu().numpy().reshape(-1)
    o_s = out.view(cfg.nblocks, -1)[blocks].cpu().numpy().reshape(-1)
    n_s = nlay.view(cfg.nblocks, -1)[blocks].cpu().numpy().reshape(-1)
    del trk, hit, out
    torch.cuda.empty_cache()
    ref = RefTBB(32, "kf")
    ref.set_bz(cfg.bz)
    rout = ref.run_masked(t_s, h_s, cfg.nlayer, n_s)
    f64 = oracle.run(t_s, h_s, 32, cfg.nlayer, 1, cfg.bz, "f64", nlay_lane=n_s)
    tp, tc, tq = parity.unpack(o_s, 32)
    rp, rc, rq = parity.unpack(rout, 32)
    assert np.array_equal(tq, rq) and len(tq) == 100000
    fin = lambda p, c: np.isfinite(p).all(1) & np.isfinite(c).all(1)
    ft, fr = fin(tp, tc), fin(rp, rc)
    assert not (fr & ~ft).any()
    both = ft & fr & fin(f64["par"], f64["cov"])
    qt = parity.error_quantiles(tp[both], tc[both], f64["par"][both], f64["cov"][both], f64["prior"][both])
    qr = parity.error_quantiles(rp[both], rc[both], f64["par"][both], f64["cov"][both], f64["prior"][both])
    for what, a, b in (("param", qt[0], qr[0]), ("cov", qt[1], qr[1])):
        for q, x, y in zip(parity.ACC_QUANTILES, a, b):
            assert x <= parity.ACC_FACTOR * y + 1e-7, f"{what} q{q}: GPU {x:.3e} vs reference {y:.3e}"


@pytest.mark.parametrize("bs,threads,opts", [(32, 0, ""), (32, 128, "chi2+dr"), (64, 0, "chi2+dr+squash"),
                                              (96, 128, "dr"), (32, 0, "chi2+dr+40")])
def test_masked_forward_ordered_by_layers_identical(p2r, torch, bs, threads, opts):
    """P2R_FLAG_ORDER_BY_LAYERS on the masked fused forward: each CTA orders its chunk's tracks by
    layer count; every output (tracks, chi2) is bit-identical to the unordered launch's."""
    nlayer = 40 if "40" in opts else 25
    cfg, trk, hit = helix(p2r, 3, 700 // bs + 1, nlayer=nlayer, bs=bs)
    rng = np.random.default_rng(bs + threads)
    nl = rng.integers(0, nlayer + 1, cfg.ntracks).astype(np.int32)
    nl[:bs] = nlayer  # a block at full length, and one with every lane empty
    nl[bs:2 * bs] = 0
    dr = rng.uniform(-0.01, 0.01, nlayer).astype(np.float32) if "dr" in opts else None
    fl = p2r.FLAG_SQUASH_PHI if "squash" in opts else 0
    outs = []
    for order in (False, True):
        c = p2r.Config(**{**cfg.__dict__, "block_threads": threads,
                          "flags": fl | (p2r.FLAG_ORDER_BY_LAYERS if order else 0)})
        outs.append(gpu_forward(p2r, torch, c, trk, hit, chi2="chi2" in opts, dr=dr, nlay_lane=nl))
    if "chi2" in opts:
        (a, ca), (b, cb) = outs
        assert np.array_equal(ca.view(np.uint32), cb.view(np.uint32))
    else:
        a, b = outs
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
