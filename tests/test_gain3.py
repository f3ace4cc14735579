"""The reference's unused 3x3 routines KalmanGainInv / KalmanGain (TBB:376-426), shipped as
p2r_kalman_gain_inv / p2r_kalman_gain.

The checker is the reference's own code compiled from its source (oracle/_ref), with an FP64
restatement of the same element choice (below) as the arbiter of rounding: the routines read
the lower-triangle-packed covariances as if they were packed upper-triangle row-major, so the
3x3 they invert is [[a0+b0, a1+b1, a2+b2], [a1+b1, a6+b3, a7+b4], [a2+b2, a7+b4, a11+b5]]
(a: track covariance words, b: hit covariance words), and the inverse's third element repeats
a7+b4 where the adjugate has a6+b3 (TBB:392), as the reference writes it.
"""
import ctypes

import numpy as np
import pytest

BS = 32


def upper6(r, c):
    r, c = min(r, c), max(r, c)
    return r * 6 - r * (r - 1) // 2 + (c - r)


def gain3_f64(trk, hit, nblocks, nlayer, layer, bs=BS):
    """FP64 restatement of TBB:376-426 with the reference's element choice."""
    t = trk.reshape(nblocks, 28, bs).astype(np.float64)
    h = hit.reshape(nblocks * nlayer, 9, bs).astype(np.float64)
    a, b = t[:, 6:27, :], h[layer::nlayer][:, 3:9, :]
    s0, s1, s2 = a[:, 0] + b[:, 0], a[:, 1] + b[:, 1], a[:, 2] + b[:, 2]
    s6, s7, s11 = a[:, 6] + b[:, 3], a[:, 7] + b[:, 4], a[:, 11] + b[:, 5]
    det = s0 * (s6 * s11 - s7 * s7) - s1 * (s1 * s11 - s7 * s2) + s2 * (s1 * s7 - s2 * s6)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = np.stack([s6 * s11 - s7 * s7, -(s1 * s11 - s2 * s7), s1 * s7 - s2 * s7, -(s1 * s11 - s7 * s2),
                        s0 * s11 - s2 * s2, -(s0 * s7 - s2 * s1), s1 * s7 - s2 * s6, -(s0 * s7 - s2 * s1),
                        s0 * s6 - s1 * s1], 1) / det[:, None]
        gain = np.zeros((nblocks, 18, bs))
        for r in range(6):
            x = [a[:, upper6(r, c)] for c in range(3)]
            for c in range(3):
                gain[:, 3 * r + c] = x[0] * inv[:, c] + x[1] * inv[:, 3 + c] + x[2] * inv[:, 6 + c]
    return inv, gain


def rel_err(x, ref):
    """Element error relative to the largest |FP64| value of the same lane's matrix."""
    scale = np.abs(ref).max(axis=1, keepdims=True)
    return np.abs(x.astype(np.float64) - ref) / scale


def inputs(p2r):
    """Tracks with full covariances: the chained filter's outputs after 20 layers of synthetic
    helices (the generator's own initial covariances are diagonal, which makes the reference's
    3x3 singular), and the reference's own fixture."""
    from oracle.oracle import RefTBB, gen_helix, ref_available
    if not ref_available(BS, "v3"):
        pytest.skip("reference build oracle/_ref missing")
    ref = RefTBB(BS, "v3")
    trk, hit = gen_helix(BS, 1, 8, 20, seed=77)
    out = ref.run(trk, hit, 1, 8, 20, True, 1, 1)
    ftrk, fhit = ref.prepare_fixture()
    nev, nbf, nlf = ref.fixture_sizes()
    return ref, [(out, hit, 8, 20, (0, 19)), (ftrk, fhit, nev * nbf, nlf, (0, 7, nlf - 1))]


def test_restatement_matches_reference_build(p2r):
    """The FP64 restatement (the arbiter) agrees with the reference's compiled routines to
    float rounding on every element."""
    ref, cases = inputs(p2r)
    for trk, hit, nblocks, nlayer, layers in cases:
        for layer in layers:
            inv_r, gain_r = ref.gain3(trk, hit, nblocks, nlayer, layer)
            inv_d, gain_d = gain3_f64(trk, hit, nblocks, nlayer, layer)
            assert rel_err(inv_r, inv_d).max() < 2e-5
            assert rel_err(gain_r, gain_d).max() < 2e-5


@pytest.mark.gpu
def test_gain3_matches_reference(p2r):
    import torch
    ref, cases = inputs(p2r)
    for trk, hit, nblocks, nlayer, layers in cases:
        cfg = p2r.Config(bsize=BS, nlayer=nlayer, nevts=1, nb=nblocks, bz=3.8)
        d_trk = torch.from_numpy(np.ascontiguousarray(trk).reshape(-1)).cuda()
        d_hit = torch.from_numpy(np.ascontiguousarray(hit).reshape(-1)).cuda()
        inv = torch.empty(nblocks * 9 * BS, dtype=torch.float32, device="cuda")
        gain = torch.empty(nblocks * 18 * BS, dtype=torch.float32, device="cuda")
        for layer in layers:
            p2r.KalmanGainInv(cfg, d_trk, d_hit, layer, inv)
            p2r.KalmanGain(cfg, d_trk, inv, gain)
            torch.cuda.synchronize()
            inv_g = inv.cpu().numpy().reshape(nblocks, 9, BS)
            gain_g = gain.cpu().numpy().reshape(nblocks, 18, BS)
            inv_r, gain_r = ref.gain3(trk, hit, nblocks, nlayer, layer)
            inv_d, gain_d = gain3_f64(trk, hit, nblocks, nlayer, layer)
            for got, want, f64 in ((inv_g, inv_r, inv_d), (gain_g, gain_r, gain_d)):
                e_ref, e_gpu = rel_err(want, f64), rel_err(got, f64)
                assert e_gpu.max() <= max(2 * e_ref.max(), 1e-6), (layer, e_gpu.max(), e_ref.max())
                assert rel_err(got, want.astype(np.float64)).max() < 2e-5


@pytest.mark.gpu
def test_gain3_singular_matrix_gives_nonfinite_like_reference(p2r):
    """With diagonal covariances the reference's 3x3 has a zero row: its determinant is zero
    and the inverse non-finite. The device routine gives the same non-finite pattern."""
    import torch
    from oracle.oracle import RefTBB, gen_helix, ref_available
    if not ref_available(BS, "v3"):
        pytest.skip("reference build oracle/_ref missing")
    ref = RefTBB(BS, "v3")
    trk, hit = gen_helix(BS, 1, 2, 20, seed=5)
    cfg = p2r.Config(bsize=BS, nlayer=20, nevts=1, nb=2, bz=3.8)
    inv = torch.empty(2 * 9 * BS, dtype=torch.float32, device="cuda")
    p2r.KalmanGainInv(cfg, torch.from_numpy(trk.reshape(-1)).cuda(), torch.from_numpy(hit.reshape(-1)).cuda(), 3, inv)
    torch.cuda.synchronize()
    inv_r, _ = ref.gain3(trk, hit, 2, 20, 3)
    got = inv.cpu().numpy().reshape(2, 9, BS)
    assert np.array_equal(np.isfinite(got), np.isfinite(inv_r))
    assert not np.isfinite(got).all()


@pytest.mark.usefixtures("host_only")
def test_gain3_rejects_bad_arguments(p2r):
    l = p2r.lib()
    c = p2r.Config(bsize=32, nlayer=20, nevts=1, nb=1).c()
    base = 1 << 35
    trk, hits, inv, gain = base, base + (1 << 20), base + (2 << 20), base + (3 << 20)
    assert l.p2r_kalman_gain_inv(ctypes.byref(c), trk, hits, 20, inv, None) == 1
    assert "layer" in l.p2r_last_error_string().decode()
    assert l.p2r_kalman_gain_inv(ctypes.byref(c), trk, hits, 0, None, None) == 1
    assert l.p2r_kalman_gain_inv(ctypes.byref(c), trk, hits, 0, hits + 64, None) == 1
    assert "overlap" in l.p2r_last_error_string().decode()
    assert l.p2r_kalman_gain(ctypes.byref(c), trk, inv, trk + 256, None) == 1
    assert "overlap" in l.p2r_last_error_string().decode()
    assert l.p2r_kalman_gain(ctypes.byref(c), trk, inv + 2, gain, None) == 1
    assert "aligned" in l.p2r_last_error_string().decode()
