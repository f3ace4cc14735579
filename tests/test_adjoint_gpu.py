"""GPU tests of the hand-written adjoint (p2r_forward_backward) through the C ABI.

Reference gradient: torch autograd in FP64 over oracle/p2r_torch.py (pinned to the C
oracle and to central finite differences in tests/test_adjoint_cpu.py). Tolerance: each
gradient within 1e-3 relative of the FP64 reference, relative to max(|g|, 1e-3 * the
largest |g| of that gradient group) so components that are zero to rounding are measured
against the group's scale. The default adjoint runs in FP64; the FP32 mode
(P2R_FLAG_ADJ_FP32) is held to its measured accuracy instead.
"""
import numpy as np
import pytest

from tests import parity

pytestmark = pytest.mark.gpu

GRAD_RTOL = 1e-3


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def setup(p2r, torch, nevts=1, nb=8, nlayer=20, seed=20240001):
    cfg = p2r.Config(bsize=32, nlayer=nlayer, nevts=nevts, nb=nb, bz=3.8)
    trk, hit = p2r.generate_helix(cfg, p2r.gen_params(bz=3.8, seed=seed))
    rng = np.random.default_rng(seed)
    dr = rng.uniform(-0.01, 0.01, nlayer).astype(np.float32)  # +-100 um
    g_trk = np.zeros_like(trk)
    g_trk[:, 0:6, :] = rng.normal(size=(cfg.nblocks, 6, 32))
    g_trk[:, 6:27, :] = rng.normal(size=(cfg.nblocks, 21, 32)) * 1e2
    g_chi2 = rng.uniform(0.5, 1.5, cfg.ntracks).astype(np.float32)
    return cfg, trk, hit, dr, g_trk, g_chi2


def torch_reference(p2r, cfg, trk, hit, dr, g_trk, g_chi2, nlay=None):
    """FP64 reference gradients by torch autograd over the oracle restatement (CPU)."""
    import torch as T
    from oracle import p2r_torch
    bs = cfg.bsize
    t = trk.reshape(cfg.nblocks, 28, bs)
    h = hit.reshape(cfg.nblocks, cfg.nlayer, 9, bs)
    par0 = T.tensor(t[:, 0:6, :].transpose(0, 2, 1).reshape(-1, 6), dtype=T.float64, requires_grad=True)
    cov0 = T.tensor(t[:, 6:27, :].transpose(0, 2, 1).reshape(-1, 21), dtype=T.float64, requires_grad=True)
    q = T.tensor(p2r.tracks_q(t))
    hpos = T.tensor(h[:, :, 0:3, :].transpose(0, 3, 1, 2).reshape(-1, cfg.nlayer, 3), dtype=T.float64,
                    requires_grad=True)
    hcov = T.tensor(h[:, :, 3:9, :].transpose(0, 3, 1, 2).reshape(-1, cfg.nlayer, 6), dtype=T.float64,
                    requires_grad=True)
    drt = T.tensor(dr.astype(np.float64), requires_grad=True)
    bz = T.tensor(cfg.bz, dtype=T.float64, requires_grad=True)
    nl = None if nlay is None else T.tensor(nlay)
    par, cov, chi2 = p2r_torch.chained(par0, cov0, q, hpos, hcov, drt, bz, nl)
    gt = g_trk.reshape(cfg.nblocks, 28, bs)
    gp = T.tensor(gt[:, 0:6, :].transpose(0, 2, 1).reshape(-1, 6), dtype=T.float64)
    gc = T.tensor(gt[:, 6:27, :].transpose(0, 2, 1).reshape(-1, 21), dtype=T.float64)
    L = (gp * par).sum() + (gc * cov).sum() + (T.tensor(g_chi2, dtype=T.float64) * chi2).sum()
    L.backward()
    return dict(par0=par0.grad.numpy(), cov0=cov0.grad.numpy(), hpos=hpos.grad.numpy(), hcov=hcov.grad.numpy(),
                dr=drt.grad.numpy(), bz=float(bz.grad), out_par=par.detach().numpy(), chi2=chi2.detach().numpy())


def gpu_grads(p2r, torch, cfg, trk, hit, dr, g_trk, g_chi2, ckpt=5, nlay=None, per_event=False, fp32=False,
              tape=True):
    if fp32:
        cfg = p2r.Config(**{**cfg.__dict__, "flags": cfg.flags | p2r.FLAG_ADJ_FP32})
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()
    o = p2r.forward_backward(cfg, d(trk), d(hit), dr=d(dr), nlay_lane=None if nlay is None else d(nlay),
                             grad_trk_out=d(g_trk), grad_chi2=d(g_chi2), ckpt_stride=ckpt, per_event=per_event,
                             tape=tape)
    torch.cuda.synchronize()
    bs = cfg.bsize
    gt = o["grad_trk_in"].cpu().numpy().reshape(cfg.nblocks, 28, bs)
    gh = o["grad_hits"].cpu().numpy().reshape(cfg.nblocks, cfg.nlayer, 9, bs)
    res = dict(par0=gt[:, 0:6, :].transpose(0, 2, 1).reshape(-1, 6),
               cov0=gt[:, 6:27, :].transpose(0, 2, 1).reshape(-1, 21),
               hpos=gh[:, :, 0:3, :].transpose(0, 3, 1, 2).reshape(-1, cfg.nlayer, 3),
               hcov=gh[:, :, 3:9, :].transpose(0, 3, 1, 2).reshape(-1, cfg.nlayer, 6),
               dr=o["grad_dr"].cpu().numpy(), bz=float(o["grad_bz"].cpu().numpy()[0]),
               trk_out=o["trk_out"].cpu().numpy(), chi2=o["chi2"].cpu().numpy())
    if per_event:
        res["dr_event"] = o["grad_dr_event"].cpu().numpy()
        res["bz_event"] = o["grad_bz_event"].cpu().numpy()
    return res


def grad_err(g, ref):
    g, ref = np.asarray(g, np.float64), np.asarray(ref, np.float64)
    scale = max(np.abs(ref).max(), 1e-300)
    return np.abs(g - ref) / np.maximum(np.abs(ref), 1e-3 * scale)


def test_adjoint_matches_fp64_reference(p2r, torch):
    cfg, trk, hit, dr, g_trk, g_chi2 = setup(p2r, torch)
    ref = torch_reference(p2r, cfg, trk, hit, dr, g_trk, g_chi2)
    got = gpu_grads(p2r, torch, cfg, trk, hit, dr, g_trk, g_chi2)
    report = {}
    for key in ("par0", "cov0", "hpos", "hcov", "dr"):
        e = grad_err(got[key], ref[key])
        report[key] = (float(np.quantile(e, 0.99)), float(e.max()))
    report["bz"] = float(grad_err([got["bz"]], [ref["bz"]])[0])
    for key in ("par0", "cov0", "hpos", "hcov", "dr"):
        assert report[key][1] < GRAD_RTOL, report  # every element
    assert report["bz"] < GRAD_RTOL, report


@pytest.mark.parametrize("regime", ["low_pt", "high_pt", "forward", "backward", "bz_2T"])
def test_adjoint_edge_regimes_match_fp64_reference(p2r, oracle, torch, regime):
    """The FP64 adjoint against the FP64 reference gradient outside the default workload's ranges
    (pT 1 and 50 GeV, polar angles near the beam axis, a 2 T field): every element within 1e-3.
    Tracks that the FP64 chain itself takes to non-finite values (about 1 % near the axis) are
    given no layers, so that they do not poison the shared dr / Bz sums.

    At pT 50 GeV a few tracks sit where the 1 um convergence test of the helix iterations
    (TBB:714) changes outcome within rounding: the two FP64 formulations take opposite sides and
    each gradient is one of the two one-sided derivatives (central differences of either forward
    land between them and drift with the step). Near the beam axis (polar angles within 0.3 rad
    of it) the same happens to single elements now and then (one hit-position element at
    1.3e-3 on one of the GPU runs, the rest below 1e-7 at the 99th percentile). There the
    per-track gradients are held at the 99th percentile with at most 5 % of tracks off, and the
    shared dr / Bz sums at every element."""
    kw = dict(low_pt=dict(pt=1.0), high_pt=dict(pt=50.0), forward=dict(theta_min=0.1, theta_max=0.3),
              backward=dict(theta_min=2.84, theta_max=3.04), bz_2T=dict(bz=2.0))[regime]
    bz = kw.pop("bz", 3.8)
    cfg = p2r.Config(bsize=32, nlayer=20, nevts=1, nb=8, bz=bz)
    trk, hit = p2r.generate_helix(cfg, p2r.gen_params(bz=bz, seed=91, **kw))
    f64 = oracle.run(trk, hit, 32, cfg.nlayer, 1, bz, "f64")
    fin = np.isfinite(f64["par"]).all(1) & np.isfinite(f64["cov"]).all(1) & np.isfinite(f64["chi2"])
    nlay = np.where(fin, cfg.nlayer, 0).astype(np.int32)
    rng = np.random.default_rng(91)
    dr = rng.uniform(-0.01, 0.01, cfg.nlayer).astype(np.float32)
    g_trk = np.zeros_like(trk)
    g_trk[:, 0:6, :] = rng.normal(size=(cfg.nblocks, 6, 32))
    g_trk[:, 6:27, :] = rng.normal(size=(cfg.nblocks, 21, 32)) * 1e2
    g_chi2 = rng.uniform(0.5, 1.5, cfg.ntracks).astype(np.float32)
    ref = torch_reference(p2r, cfg, trk, hit, dr, g_trk, g_chi2, nlay=nlay)
    got = gpu_grads(p2r, torch, cfg, trk, hit, dr, g_trk, g_chi2, ckpt=1, nlay=nlay)
    for key in ("par0", "cov0", "hpos", "dr"):
        e = grad_err(got[key], ref[key])
        if regime in ("high_pt", "forward", "backward") and key != "dr":
            off = (e.reshape(cfg.ntracks, -1) >= GRAD_RTOL).any(1).mean()
            assert np.quantile(e, 0.99) < GRAD_RTOL and off <= 0.05, (regime, key, float(np.quantile(e, 0.99)), off)
        else:
            assert e.max() < GRAD_RTOL, (regime, key, float(np.quantile(e, 0.99)), float(e.max()))
    assert grad_err([got["bz"]], [ref["bz"]])[0] < GRAD_RTOL, regime


def test_fp32_adjoint_mode(p2r, torch):
    """The FP32 instance of the same kernel is held to its measured accuracy, not the 1e-3
    bar: per-track gradients ~1e-3 at the median; the shared Bz gradient (a sum over tracks of
    terms that largely cancel) was 17 % off on this 256-track case. It is a speed option for
    per-track hit gradients, not for calibration."""
    cfg, trk, hit, dr, g_trk, g_chi2 = setup(p2r, torch)
    ref = torch_reference(p2r, cfg, trk, hit, dr, g_trk, g_chi2)
    got = gpu_grads(p2r, torch, cfg, trk, hit, dr, g_trk, g_chi2, fp32=True)
    assert np.quantile(grad_err(got["par0"], ref["par0"]), 0.5) < 1e-2
    assert np.quantile(grad_err(got["hpos"], ref["hpos"]), 0.5) < 1e-2
    assert grad_err(got["dr"], ref["dr"]).max() < 0.2
    assert grad_err([got["bz"]], [ref["bz"]])[0] < 0.5


@pytest.mark.parametrize("ckpt", [1, 2, 4, 10])
def test_checkpoint_strides_agree(p2r, torch, ckpt):
    cfg, trk, hit, dr, g_trk, g_chi2 = setup(p2r, torch)
    base = gpu_grads(p2r, torch, cfg, trk, hit, dr, g_trk, g_chi2, ckpt=5)
    other = gpu_grads(p2r, torch, cfg, trk, hit, dr, g_trk, g_chi2, ckpt=ckpt)
    for key in ("par0", "cov0", "hpos", "hcov", "dr"):
        assert np.quantile(grad_err(other[key], base[key]), 0.999) < 1e-5, key
    assert abs(other["bz"] - base["bz"]) <= 1e-5 * abs(base["bz"])


@pytest.mark.parametrize("ckpt", [1, 4, 5])
@pytest.mark.parametrize("fp32", [False, True])
def test_tape_and_thread_local_paths_identical(p2r, torch, ckpt, fp32):
    """Checkpoints in a device-memory tape (two kernels) or in thread-local memory (one
    kernel): the same formulas, so the same results up to where the compiler fuses a
    multiply-add differently in the two kernels (FP64: float32 outputs all but identical),
    with masked lanes."""
    cfg, trk, hit, dr, g_trk, g_chi2 = setup(p2r, torch, nevts=2, nb=3, nlayer=23)
    nlay = np.random.default_rng(3).integers(5, 24, cfg.ntracks).astype(np.int32)
    a = gpu_grads(p2r, torch, cfg, trk, hit, dr, g_trk, g_chi2, ckpt=ckpt, nlay=nlay, per_event=True, fp32=fp32)
    b = gpu_grads(p2r, torch, cfg, trk, hit, dr, g_trk, g_chi2, ckpt=ckpt, nlay=nlay, per_event=True, fp32=fp32,
                  tape=False)
    for key in a:
        x, y = np.asarray(a[key], np.float64), np.asarray(b[key], np.float64)
        if key == "trk_out":  # the q row holds integer bits: compare par and cov rows as numbers
            x = x.reshape(-1, 28, 32)[:, :27]
            y = y.reshape(-1, 28, 32)[:, :27]
        e = grad_err(x.reshape(-1), y.reshape(-1))
        if fp32:  # FP32 gradients are accurate to ~1e-2 at the median only (test_fp32_adjoint_mode):
            # two compilations of that arithmetic agree to that level, their tails do not
            assert np.quantile(e, 0.5) < 1e-2, (key, np.quantile(e, [0.5, 0.99, 1]))
        elif key in ("dr", "bz", "dr_event", "bz_event"):
            # shared sums, kept in double: the two compilations' different fusing shows at ~1e-14
            assert e.max() < 1e-10, (key, e.max())
        else:
            assert np.quantile(e, 0.99) < 1e-6 and (e == 0).mean() > 0.9, (key, np.quantile(e, [0.5, 0.99, 1]))


def test_forward_outputs_are_fp64_chain(p2r, oracle, torch):
    """The FP64 kernel's forward outputs are the FP64 chain rounded to float."""
    cfg, trk, hit, dr, g_trk, g_chi2 = setup(p2r, torch)
    got = gpu_grads(p2r, torch, cfg, trk, hit, dr, g_trk, g_chi2)
    f64 = oracle.run(trk, hit, 32, cfg.nlayer, 1, cfg.bz, "f64", dr=dr.astype(np.float64))
    tp, tc, _ = parity.unpack(got["trk_out"], 32)
    assert (parity.rel_par(tp, f64["par"]) < 1e-6).all()
    assert (parity.rel_cov(tc, f64["cov"], f64["prior"]) < 1e-5).all()
    assert (np.abs(got["chi2"] - f64["chi2"]) <= 1e-6 * np.maximum(np.abs(f64["chi2"]), 1)).all()


def test_fp32_forward_outputs_match_plain_forward(p2r, oracle, torch):
    """The FP32 adjoint kernel's forward outputs are as accurate (against FP64) as the plain
    fused forward's (the two kernels need not contract or approximate identically)."""
    cfg, trk, hit, dr, g_trk, g_chi2 = setup(p2r, torch)
    got = gpu_grads(p2r, torch, cfg, trk, hit, dr, g_trk, g_chi2, fp32=True)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()
    out = torch.empty(trk.size, dtype=torch.float32, device="cuda")
    chi2 = torch.empty(cfg.ntracks, dtype=torch.float32, device="cuda")
    p2r.forward(cfg, d(trk), d(hit), out, chi2=chi2, dr=d(dr))
    f64 = oracle.run(trk, hit, 32, cfg.nlayer, 1, cfg.bz, "f64", dr=dr.astype(np.float64))
    parity.assert_accuracy_parity(got["trk_out"], out.cpu().numpy(), f64["par"], f64["cov"], f64["prior"], 32,
                                  "fwd+bwd (FP32) forward outputs vs plain forward")
    rel = lambda c: np.abs(c - f64["chi2"]) / np.maximum(np.abs(f64["chi2"]), 1.0)
    assert np.quantile(rel(got["chi2"]), 0.99) <= 2 * np.quantile(rel(chi2.cpu().numpy()), 0.99) + 1e-6


def test_per_event_gradients_sum_to_totals(p2r, torch):
    cfg, trk, hit, dr, g_trk, g_chi2 = setup(p2r, torch, nevts=3, nb=4)
    got = gpu_grads(p2r, torch, cfg, trk, hit, dr, g_trk, g_chi2, per_event=True)
    assert np.allclose(got["dr_event"].sum(0), got["dr"], rtol=1e-12, atol=0)
    assert np.isclose(got["bz_event"].sum(), got["bz"], rtol=1e-12, atol=0)
    ref = torch_reference(p2r, cfg, trk, hit, dr, g_trk, g_chi2)
    assert grad_err(got["dr"], ref["dr"]).max() < GRAD_RTOL


def test_masked_lanes_adjoint(p2r, torch):
    cfg, trk, hit, dr, g_trk, g_chi2 = setup(p2r, torch, nlayer=25)
    nlay = np.random.default_rng(9).integers(10, 26, cfg.ntracks).astype(np.int32)
    ref = torch_reference(p2r, cfg, trk, hit, dr, g_trk, g_chi2, nlay=nlay)
    got = gpu_grads(p2r, torch, cfg, trk, hit, dr, g_trk, g_chi2, nlay=nlay)
    for key in ("par0", "hpos", "dr"):
        assert np.quantile(grad_err(got[key], ref[key]), 0.99) < GRAD_RTOL, key
    # hits past a track's last layer get zero gradient
    for t in range(0, cfg.ntracks, 37):
        assert np.all(got["hpos"][t, nlay[t]:] == 0)


def test_autograd_function(p2r, torch):
    cfg, trk, hit, dr, g_trk, g_chi2 = setup(p2r, torch)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()
    t, h, r = d(trk).requires_grad_(), d(hit).requires_grad_(), d(dr).requires_grad_()
    bz = torch.tensor(3.8, dtype=torch.float64, requires_grad=True)
    out, chi2 = p2r.P2RChain.apply(t, h, r, bz, cfg, 5)
    L = (out * d(g_trk)).sum() + (chi2 * d(g_chi2)).sum()
    L.backward()
    got = gpu_grads(p2r, torch, cfg, trk, hit, dr, g_trk, g_chi2)
    gt = t.grad.cpu().numpy().reshape(cfg.nblocks, 28, 32)
    assert np.allclose(gt[:, 0:6, :].transpose(0, 2, 1).reshape(-1, 6), got["par0"], rtol=1e-6, atol=0)
    assert np.allclose(r.grad.cpu().numpy(), got["dr"].astype(np.float32), rtol=1e-6)
    assert abs(float(bz.grad) - got["bz"]) <= 1e-9 * abs(got["bz"])


def test_adjoint_rejects_bad_requests(p2r, torch):
    cfg, trk, hit, dr, g_trk, g_chi2 = setup(p2r, torch)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()
    with pytest.raises(p2r.P2RError):
        p2r.forward_backward(cfg, d(trk), d(hit), ckpt_stride=3)
    cfg.mode = p2r.MODE_RESTART
    with pytest.raises(p2r.P2RError):
        p2r.forward_backward(cfg, d(trk), d(hit))


def test_calibration_gradients_config4_shape(p2r, torch):
    """The calibration use of the adjoint in the shape of the 40-layer workload (hits on
    r = 4..110 cm, inputs generated on the device, 20-40 layers per track, radius offsets of
    +-100 um): per-event chi2 gradients w.r.t. the 40 offsets and Bz, captured in a CUDA graph
    and replayed, against the FP64 reference computed event by event."""
    nevts, nb, nlayer = 2, 4, 40
    cfg = p2r.Config(bsize=32, nlayer=nlayer, nevts=nevts, nb=nb, bz=3.8)
    gp = p2r.gen_params(bz=3.8, seed=4040, r_first=4.0, r_last=110.0)
    trk_d, hit_d = p2r.generate_helix_device(cfg, gp)
    rng = np.random.default_rng(4)
    nlay = rng.integers(20, nlayer + 1, cfg.ntracks).astype(np.int32)
    dr = rng.uniform(-0.01, 0.01, nlayer).astype(np.float32)
    d_nlay, d_dr = torch.from_numpy(nlay).cuda(), torch.from_numpy(dr).cuda()
    g_chi2 = torch.ones(cfg.ntracks, dtype=torch.float32, device="cuda")
    out = {"grad_trk_in": None, "grad_hits": None}
    p2r.forward_backward(cfg, trk_d, hit_d, dr=d_dr, nlay_lane=d_nlay, grad_chi2=g_chi2, per_event=True, out=out)
    torch.cuda.synchronize()
    direct = {k: out[k].clone() for k in ("grad_dr_event", "grad_bz_event", "chi2")}
    for k in ("grad_dr_event", "grad_bz_event", "chi2"):
        out[k].zero_()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        p2r.forward_backward(cfg, trk_d, hit_d, dr=d_dr, nlay_lane=d_nlay, grad_chi2=g_chi2, per_event=True, out=out,
                             stream=s)
    g.replay()
    torch.cuda.synchronize()
    for k in direct:  # graph replay == direct call, bit for bit (deterministic reductions)
        assert torch.equal(direct[k], out[k]), k
    trk, hit = trk_d.cpu().numpy(), hit_d.cpu().numpy()
    per_ev_trk, per_ev_hit = trk.size // nevts, hit.size // nevts
    g_trk0 = np.zeros(per_ev_trk, np.float32)
    for e in range(nevts):
        ce = p2r.Config(bsize=32, nlayer=nlayer, nevts=1, nb=nb, bz=3.8)
        te = trk[e * per_ev_trk:(e + 1) * per_ev_trk]
        he = hit[e * per_ev_hit:(e + 1) * per_ev_hit]
        ne = nlay[e * nb * 32:(e + 1) * nb * 32]
        ref = torch_reference(p2r, ce, te, he, dr, g_trk0, np.ones(nb * 32, np.float32), nlay=ne)
        got_dr = out["grad_dr_event"][e].cpu().numpy()
        assert grad_err(got_dr, ref["dr"]).max() < GRAD_RTOL, (e, grad_err(got_dr, ref["dr"]).max())
        assert grad_err([float(out["grad_bz_event"][e])], [ref["bz"]])[0] < GRAD_RTOL
    del g


@pytest.mark.parametrize("tape", [True, False])
def test_order_by_layers_flag(p2r, torch, tape):
    """P2R_FLAG_ORDER_BY_LAYERS with per-track layer counts: each event's tracks run in an order
    by layer count computed inside the call; every per-track output stays at its track's position
    and is the same arithmetic as without the flag (identical), the shared sums are added in the
    new grouping (equal to 1e-9)."""
    cfg, trk, hit, dr, g_trk, g_chi2 = setup(p2r, torch, nevts=3, nb=4, nlayer=25)
    nlay = np.random.default_rng(8).integers(3, 26, cfg.ntracks).astype(np.int32)
    a = gpu_grads(p2r, torch, cfg, trk, hit, dr, g_trk, g_chi2, ckpt=1, nlay=nlay, per_event=True, tape=tape)
    co = p2r.Config(**{**cfg.__dict__, "flags": cfg.flags | p2r.FLAG_ORDER_BY_LAYERS})
    b = gpu_grads(p2r, torch, co, trk, hit, dr, g_trk, g_chi2, ckpt=1, nlay=nlay, per_event=True, tape=tape)
    for key in a:
        x, y = np.asarray(a[key], np.float64), np.asarray(b[key], np.float64)
        if key in ("dr", "bz", "dr_event", "bz_event"):
            assert np.abs(x - y).max() <= 1e-9 * np.abs(x).max(), key
        else:
            assert np.array_equal(x.view(np.uint64), y.view(np.uint64)), key
