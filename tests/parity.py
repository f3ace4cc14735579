"""Parity metrics and the tolerances the tests apply (written here, used everywhere).

Parameters (x, y, z [cm], 1/pT [1/GeV], phi, theta [rad]):
    rel_par = |a - b| / max(|b|, floor), floor = (1, 1, 1, 0.01, 1, 1)
  The floor keeps coordinates that pass through zero (z, phi, x, y) from turning a
  micron-level difference into a large relative one.

Covariance elements C_ij:
    rel_cov = |a - b| / max(|b|, sqrt(P_ii * P_jj))
  where P is the covariance ENTERING the last Kalman update. The update C - K H C cancels
  the prior down to the (much smaller) posterior; its rounding scales with the prior, so
  this is the conditioning-aware relative error (measured: with P = the posterior the
  reference's own FP32 result is O(1) away from FP64 in restart mode).

Tolerances (the stated bar):  PAR_RTOL = 1e-4, COV_RTOL = 1e-3
  element-wise max for: single-layer steps (propagateToR, KalmanUpdate), the restart
  driver, and every step along a chained run (reference state in, one step, compare);
  for the chained end-to-end output the FP32 chain is ill-conditioned (the reference
  itself is 3e-3 away from FP64 at the 99th percentile of covariance elements, 3.3 % of them
  beyond COV_RTOL, and up to 0.13 on its tail), so there the test requires
  (a) the 99th percentile within PAR_RTOL / CHAIN_COV_P99 and
  (b) accuracy parity: every error quantile of the GPU against the FP64 oracle within
      ACC_FACTOR of the reference's own error quantile against the FP64 oracle.
q (charge) and indexing: bit-exact.

Single steps between two FP32 implementations: the reference's own FP32 result is not
exact, and where an update is ill-conditioned (a strongly correlated x-y position block,
a convergence branch decided by rounding, TBB:714) two correct FP32 evaluations can differ
by more than PAR_RTOL / COV_RTOL. `assert_step` therefore accepts an element when it is
within tolerance of the reference OR no farther from the FP64 oracle than STEP_ACC times the
reference's own distance to it (the test implementation is at least as accurate there).
"""
from __future__ import annotations

import numpy as np

PAR_RTOL = 1e-4
COV_RTOL = 1e-3
CHAIN_COV_P99 = 5e-3
ACC_FACTOR = 2.0
ACC_QUANTILES = (0.5, 0.9, 0.99, 0.999)
STEP_ACC = 2.0

PAR_FLOOR = np.array([1.0, 1.0, 1.0, 0.01, 1.0, 1.0])
DIAG = [i * (i + 1) // 2 + i for i in range(6)]


def sym(i: int, j: int) -> int:
    return i * (i + 1) // 2 + j if i >= j else j * (j + 1) // 2 + i


def unpack(trk: np.ndarray, bsize: int):
    """(par (n,6), cov (n,21), q (n,)) of a Matriplex track array of any shape."""
    t = np.ascontiguousarray(trk, np.float32).reshape(-1, 28, bsize)
    par = t[:, 0:6, :].transpose(0, 2, 1).reshape(-1, 6).astype(np.float64)
    cov = t[:, 6:27, :].transpose(0, 2, 1).reshape(-1, 21).astype(np.float64)
    q = np.ascontiguousarray(t[:, 27, :]).view(np.int32).reshape(-1)
    return par, cov, q


def rel_par(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return np.abs(a - b) / np.maximum(np.abs(b), PAR_FLOOR)


def cov_scale(prior: np.ndarray) -> np.ndarray:
    d = np.abs(prior[:, DIAG])
    sc = np.empty_like(prior)
    for i in range(6):
        for j in range(i + 1):
            sc[:, sym(i, j)] = np.sqrt(d[:, i] * d[:, j])
    return sc


def rel_cov(a: np.ndarray, b: np.ndarray, prior: np.ndarray) -> np.ndarray:
    return np.abs(a - b) / np.maximum(np.abs(b), cov_scale(prior))


def assert_elementwise(test_trk, ref_trk, prior, bsize, what="", par_rtol=PAR_RTOL, cov_rtol=COV_RTOL):
    tp, tc, tq = unpack(test_trk, bsize)
    rp, rc, rq = unpack(ref_trk, bsize)
    assert np.array_equal(tq, rq), f"{what}: charges differ"
    fin = np.isfinite(rp).all(1) & np.isfinite(rc).all(1)
    assert np.array_equal(fin, np.isfinite(tp).all(1) & np.isfinite(tc).all(1)), f"{what}: non-finite sets differ"
    ep = rel_par(tp[fin], rp[fin])
    ec = rel_cov(tc[fin], rc[fin], prior[fin])
    assert ep.max(initial=0) <= par_rtol, f"{what}: max rel param error {ep.max():.3e} > {par_rtol} at {np.unravel_index(ep.argmax(), ep.shape)}"
    assert ec.max(initial=0) <= cov_rtol, f"{what}: max rel cov error {ec.max():.3e} > {cov_rtol} at {np.unravel_index(ec.argmax(), ec.shape)}"
    return ep.max(initial=0), ec.max(initial=0)


def error_quantiles(test_par, test_cov, truth_par, truth_cov, prior):
    ep = rel_par(test_par, truth_par).reshape(-1)
    ec = rel_cov(test_cov, truth_cov, prior).reshape(-1)
    return np.quantile(ep, ACC_QUANTILES), np.quantile(ec, ACC_QUANTILES)


def assert_accuracy_parity(test_trk, ref_trk, f64_par, f64_cov, prior, bsize, what="", factor=ACC_FACTOR):
    """The test output is no less accurate (against FP64) than the reference's, per quantile."""
    tp, tc, _ = unpack(test_trk, bsize)
    rp, rc, _ = unpack(ref_trk, bsize)
    qtp, qtc = error_quantiles(tp, tc, f64_par, f64_cov, prior)
    qrp, qrc = error_quantiles(rp, rc, f64_par, f64_cov, prior)
    for q, a, b in zip(ACC_QUANTILES, qtp, qrp):
        assert a <= factor * b + 1e-7, f"{what}: param error q{q} {a:.3e} vs reference {b:.3e}"
    for q, a, b in zip(ACC_QUANTILES, qtc, qrc):
        assert a <= factor * b + 1e-7, f"{what}: cov error q{q} {a:.3e} vs reference {b:.3e}"
    return (qtp, qtc), (qrp, qrc)


def assert_same_arithmetic(a, b, bs, what):
    """Two launches of the same arithmetic: q bit-equal, values equal up to the rounding of
    differently contracted FMAs (separately compiled kernel variants may fuse a*b+c in
    different places). Most tracks come out bit-identical; the chained filter amplifies the
    rest, so the bound is the FP32 accuracy level itself (PAR_RTOL at the 99.9th percentile)."""
    ap, ac, aq = unpack(a, bs)
    bp, bc, bq = unpack(b, bs)
    assert np.array_equal(aq, bq), what
    ep = np.abs(ap - bp) / np.maximum(np.abs(bp), PAR_FLOOR)
    ec = np.abs(ac - bc) / np.maximum(np.abs(bc), cov_scale(bc))
    assert np.quantile(ep, 0.5) == 0 and np.quantile(ep, 0.999) < PAR_RTOL and ep.max() < 1e-3, \
        (what, np.quantile(ep, [0.5, 0.999, 1]))
    assert np.quantile(ec, 0.999) < COV_RTOL and ec.max() < 1e-1, (what, np.quantile(ec, [0.5, 0.999, 1]))


def assert_step(test_trk, ref_trk, f64_par, f64_cov, prior, bsize, what=""):
    """Element-wise check of one step against the reference with the FP64 oracle as arbiter."""
    tp, tc, tq = unpack(test_trk, bsize)
    rp, rc, rq = unpack(ref_trk, bsize)
    assert np.array_equal(tq, rq), f"{what}: charges differ"
    sp = np.maximum(np.abs(rp), PAR_FLOOR)
    sc = np.maximum(np.abs(rc), cov_scale(prior))
    okp = (np.abs(tp - rp) <= PAR_RTOL * sp) | (np.abs(tp - f64_par) <= STEP_ACC * np.abs(rp - f64_par) + 0.1 * PAR_RTOL * sp)
    okc = (np.abs(tc - rc) <= COV_RTOL * sc) | (np.abs(tc - f64_cov) <= STEP_ACC * np.abs(rc - f64_cov) + 0.1 * COV_RTOL * sc)
    bad_p, bad_c = np.argwhere(~okp), np.argwhere(~okc)
    assert len(bad_p) == 0, (f"{what}: {len(bad_p)} parameter elements fail; first {bad_p[:3].tolist()}: "
                             f"test {tp[tuple(bad_p[0])]:.8g} ref {rp[tuple(bad_p[0])]:.8g} f64 {f64_par[tuple(bad_p[0])]:.8g}")
    assert len(bad_c) == 0, (f"{what}: {len(bad_c)} covariance elements fail; first {bad_c[:3].tolist()}: "
                             f"test {tc[tuple(bad_c[0])]:.8g} ref {rc[tuple(bad_c[0])]:.8g} f64 {f64_cov[tuple(bad_c[0])]:.8g}")
    ep = (np.abs(tp - rp) / sp).max(initial=0)
    ec = (np.abs(tc - rc) / sc).max(initial=0)
    return ep, ec
