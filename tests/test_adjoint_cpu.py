"""CPU test of the hand-written per-layer adjoint (p2r_tests_b200/csrc/p2r_adjoint.cuh):
its double instantiation against central finite differences of its own double forward,
for every input (state, hit position and covariance, radius offset, Bz), on states taken
from a chained run of the synthetic-helix workload."""
import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
BUILD = ROOT / "tests" / "_build"


@pytest.fixture(scope="module")
def adjh():
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    BUILD.mkdir(exist_ok=True)
    so = BUILD / "libadj_host.so"
    src = ROOT / "tests" / "adjoint_host.cpp"
    hdr = ROOT / "p2r_tests_b200" / "csrc" / "p2r_adjoint.cuh"
    if not so.exists() or so.stat().st_mtime < max(src.stat().st_mtime, hdr.stat().st_mtime):
        subprocess.run([cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-Wno-unknown-pragmas",
                        "-o", str(so), str(src)], check=True)
    l = ctypes.CDLL(str(so))
    vp = ctypes.c_void_p
    l.adjh_layer_fwd.argtypes = [vp, vp, ctypes.c_int, ctypes.c_double, vp, vp, ctypes.c_double]
    l.adjh_layer_fwd.restype = ctypes.c_double
    l.adjh_layer_rev.argtypes = [vp, vp, ctypes.c_int, ctypes.c_double, vp, vp, ctypes.c_double, vp, vp,
                                 ctypes.c_double, vp, vp, vp, vp]
    return l


def states(p2r, n=24, layers=(0, 3, 9, 18)):
    """(par, cov, q, hitpos, hitcov) at several layers of a chained double-precision run."""
    cfg = p2r.Config(bsize=32, nlayer=20, nevts=1, nb=1, bz=3.8)
    trk, hit = p2r.generate_helix(cfg)
    par, cov = p2r.tracks_par(trk).astype(np.float64), p2r.tracks_cov(trk).astype(np.float64)
    q = p2r.tracks_q(trk)
    h = hit.reshape(cfg.nlayer, 9, 32).astype(np.float64)
    return cfg, par[:n], cov[:n], q[:n], h, layers


def fwd(l, p, c, q, bz, hp, hc, dr):
    p, c = p.copy(), c.copy()
    chi2 = l.adjh_layer_fwd(p.ctypes.data, c.ctypes.data, int(q), bz, hp.ctypes.data, hc.ctypes.data, dr)
    return p, c, chi2


def test_layer_adjoint_matches_finite_differences(p2r, adjh):
    cfg, par, cov, q, h, layers = states(p2r)
    rng = np.random.default_rng(5)
    bz, dr0 = 3.8, 0.004
    worst = 0.0
    for t in range(par.shape[0]):
        p, c = par[t].copy(), cov[t].copy()
        for l in range(max(layers) + 1):
            hp = np.ascontiguousarray(h[l, 0:3, t])
            hc = np.ascontiguousarray(h[l, 3:9, t])
            if l in layers:
                pbo = rng.normal(size=6)
                cbo = rng.normal(size=21) * 1e3
                chib = rng.normal()

                def loss(pp, cc, hpp, hcc, dr, bzz):
                    po, co, chi = fwd(adjh, pp, cc, q[t], bzz, hpp, hcc, dr)
                    return pbo @ po + cbo @ co + chib * chi

                pb, cb = pbo.copy(), cbo.copy()
                hpb, hcb, drb, bzb = np.zeros(3), np.zeros(6), np.zeros(1), np.zeros(1)
                adjh.adjh_layer_rev(p.ctypes.data, c.ctypes.data, int(q[t]), bz, hp.ctypes.data, hc.ctypes.data, dr0,
                                    pb.ctypes.data, cb.ctypes.data, chib, hpb.ctypes.data, hcb.ctypes.data,
                                    drb.ctypes.data, bzb.ctypes.data)
                base = dict(pp=p, cc=c, hpp=hp, hcc=hc, dr=dr0, bzz=bz)
                checks = []
                def sym_steps(m, n):  # FD step of each packed element: 1e-3 of sqrt(C_ii C_jj)
                    d = [m[i * (i + 1) // 2 + i] for i in range(n)]
                    return [1e-3 * np.sqrt(abs(d[i] * d[j])) for i in range(n) for j in range(i + 1)]

                csteps, hsteps = sym_steps(c, 6), sym_steps(hc, 3)
                for name, arr, grad, step in (("pp", p, pb, 1e-6), ("cc", c, cb, csteps), ("hpp", hp, hpb, 1e-6),
                                              ("hcc", hc, hcb, hsteps)):
                    for i in range(arr.size):
                        e = step if np.isscalar(step) else step[i]
                        a, b = arr.copy(), arr.copy()
                        a[i] += e
                        b[i] -= e
                        fd = (loss(**{**base, name: a}) - loss(**{**base, name: b})) / (2 * e)
                        checks.append((f"{name}[{i}]", grad[i], fd))
                for name, g, e in (("dr", drb[0], 1e-6), ("bzz", bzb[0], 1e-5)):
                    fd = (loss(**{**base, name: base[name] + e}) - loss(**{**base, name: base[name] - e})) / (2 * e)
                    checks.append((name, g, fd))
                scale = max(abs(fd) for _, _, fd in checks)
                for name, g, fd in checks:
                    err = abs(g - fd) / max(abs(fd), 1e-3 * scale)
                    worst = max(worst, err)
                    assert err < 2e-4, f"track {t} layer {l} {name}: adjoint {g:.6e} vs fd {fd:.6e}"
            p, c, _ = fwd(adjh, p, c, q[t], bz, hp, hc, 0.0)
    assert worst < 2e-4


# --------------------------------------------------------------------------- FP64 reference gradient
def torch_inputs(p2r, nb=2, nlayer=20, seed=20240001):
    import torch
    cfg = p2r.Config(bsize=32, nlayer=nlayer, nevts=1, nb=nb, bz=3.8)
    trk, hit = p2r.generate_helix(cfg, p2r.gen_params(bz=3.8, seed=seed))
    h = hit.reshape(cfg.nblocks, nlayer, 9, 32)
    T = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64)
    par0 = T(p2r.tracks_par(trk))
    cov0 = T(p2r.tracks_cov(trk))
    q = torch.tensor(p2r.tracks_q(trk))
    hpos = T(h[:, :, 0:3, :].transpose(0, 3, 1, 2).reshape(-1, nlayer, 3))
    hcov = T(h[:, :, 3:9, :].transpose(0, 3, 1, 2).reshape(-1, nlayer, 6))
    dr = T(np.random.default_rng(seed).uniform(-0.01, 0.01, nlayer))
    return cfg, trk, hit, par0, cov0, q, hpos, hcov, dr


def test_torch_restatement_matches_c_oracle(p2r, oracle):
    import torch
    from oracle import p2r_torch
    cfg, trk, hit, par0, cov0, q, hpos, hcov, dr = torch_inputs(p2r)
    par, cov, chi2 = p2r_torch.chained(par0, cov0, q, hpos, hcov, dr, torch.tensor(3.8, dtype=torch.float64))
    ref = oracle.run(trk, hit, 32, cfg.nlayer, 1, 3.8, "f64", dr=dr.numpy())
    assert np.allclose(par.numpy(), ref["par"], rtol=1e-10, atol=1e-12)
    assert np.allclose(cov.numpy(), ref["cov"], rtol=1e-8, atol=1e-18)
    assert np.allclose(chi2.numpy(), ref["chi2"], rtol=1e-9)


def test_reference_gradient_matches_finite_differences(p2r, oracle):
    """Autograd of the FP64 restatement against central differences: of the independent C
    oracle for the shared inputs (dr, Bz), of the restatement for per-track inputs."""
    import torch
    from oracle import p2r_torch
    cfg, trk, hit, par0, cov0, q, hpos, hcov, dr = torch_inputs(p2r)
    rng = np.random.default_rng(3)
    gp = rng.normal(size=(cfg.ntracks, 6))
    gx = rng.uniform(0.5, 1.5, cfg.ntracks)
    bz = torch.tensor(3.8, dtype=torch.float64, requires_grad=True)
    drv = dr.clone().requires_grad_()
    p0 = par0.clone().requires_grad_()
    hp = hpos.clone().requires_grad_()
    par, cov, chi2 = p2r_torch.chained(p0, cov0, q, hp, hcov, drv, bz)
    L = (torch.tensor(gp) * par).sum() + (torch.tensor(gx) * chi2).sum()
    L.backward()

    def loss_c(drx, bzx):
        r = oracle.run(trk, hit, 32, cfg.nlayer, 1, bzx, "f64", dr=drx)
        return float((gp * r["par"]).sum() + (gx * r["chi2"]).sum())

    d = dr.numpy()
    for l in (0, 7, 19):
        e = 1e-5
        a, b = d.copy(), d.copy()
        a[l] += e
        b[l] -= e
        fd = (loss_c(a, 3.8) - loss_c(b, 3.8)) / (2 * e)
        assert abs(drv.grad[l].item() - fd) <= 1e-5 * max(abs(fd), 1.0), (l, drv.grad[l].item(), fd)
    fd = (loss_c(d, 3.8 + 1e-5) - loss_c(d, 3.8 - 1e-5)) / 2e-5  # smaller steps hit the loss's roundoff
    assert abs(bz.grad.item() - fd) <= 1e-5 * abs(fd), (bz.grad.item(), fd)

    def loss_t(pp, hh):
        par, cov, chi2 = p2r_torch.chained(pp, cov0, q, hh, hcov, dr, torch.tensor(3.8, dtype=torch.float64))
        return float((torch.tensor(gp) * par).sum() + (torch.tensor(gx) * chi2).sum())

    # the chained loss carries ~1e-6 of rounding noise: steps of 1e-4 of the value keep the
    # differences well above it, at a tolerance of 1e-4 (10x below the GPU adjoint's bar)
    for (t, i) in ((0, 0), (5, 3), (17, 4), (40, 5)):
        e = 1e-4 * max(abs(par0[t, i].item()), 0.1)
        a, b = par0.clone(), par0.clone()
        a[t, i] += e
        b[t, i] -= e
        fd = (loss_t(a, hpos) - loss_t(b, hpos)) / (2 * e)
        assert abs(p0.grad[t, i].item() - fd) <= 1e-4 * max(abs(fd), 1e-3), (t, i, p0.grad[t, i].item(), fd)
    for (t, l, c) in ((1, 0, 0), (9, 10, 2), (33, 19, 1)):
        e = 1e-4
        a, b = hpos.clone(), hpos.clone()
        a[t, l, c] += e
        b[t, l, c] -= e
        fd = (loss_t(par0, a) - loss_t(par0, b)) / (2 * e)
        assert abs(hp.grad[t, l, c].item() - fd) <= 1e-4 * max(abs(fd), 1e-3), (t, l, c, hp.grad[t, l, c].item(), fd)
