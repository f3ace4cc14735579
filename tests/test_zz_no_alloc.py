"""The allocation-free adjoint entry point (p2r_forward_backward_noalloc), called through
the C ABI, against the workspace entry point (p2r_forward_backward) on the same inputs.

It exists for callers that cannot allocate device memory when they need gradients (for
instance while a CUDA graph is being captured, or in an event loop that forbids allocation
after start-up); its scratch is a fixed device array inside the library. This file is
collected last so that, if it fails, a run stopping at the first failure has already run
every other test; it also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRAD_RTOL = 1e-3  # the adjoint tests' bar (tests/test_adjoint_gpu.py)


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def _grad_err(g, ref):
    g, ref = np.asarray(g, np.float64), np.asarray(ref, np.float64)
    scale = max(np.abs(ref).max(), 1e-300)
    return np.abs(g - ref) / np.maximum(np.abs(ref), 1e-3 * scale)


def test_noalloc_matches_workspace_entry_point(p2r, torch):
    cfg = p2r.Config(bsize=32, nlayer=20, nevts=3, nb=4, bz=3.8, mode=p2r.MODE_CHAINED)
    trk, hit = p2r.generate_helix(cfg, p2r.gen_params(bz=3.8, seed=4242))
    rng = np.random.default_rng(4242)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a).reshape(-1)).cuda()
    d_trk, d_hit = d(trk), d(hit)
    d_dr = d(rng.uniform(-0.01, 0.01, cfg.nlayer).astype(np.float32))
    g_trk = np.zeros_like(trk)
    g_trk[:, 0:6, :] = rng.normal(size=(cfg.nblocks, 6, 32))
    d_gtrk = d(g_trk)
    d_gchi2 = d(rng.uniform(0.5, 1.5, cfg.ntracks).astype(np.float32))

    ref = p2r.forward_backward(cfg, d_trk, d_hit, dr=d_dr, grad_trk_out=d_gtrk, grad_chi2=d_gchi2, ckpt_stride=5,
                               per_event=True)
    torch.cuda.synchronize()
    ref = {k: v.cpu().numpy() for k, v in ref.items() if k != "workspace"}

    lib = p2r.lib()
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    c = cfg.c()
    for call in range(2):  # two calls in a row share the scratch array
        out = {
            "trk_out": torch.full_like(d_trk, float("nan")), "chi2": torch.full((cfg.ntracks,), float("nan"), device="cuda"),
            "grad_trk_in": torch.full_like(d_trk, float("nan")), "grad_hits": torch.full_like(d_hit, float("nan")),
            "grad_dr": torch.full((cfg.nlayer,), float("nan"), dtype=torch.float64, device="cuda"),
            "grad_bz": torch.full((1,), float("nan"), dtype=torch.float64, device="cuda"),
            "grad_dr_event": torch.full((cfg.nevts, cfg.nlayer), float("nan"), dtype=torch.float64, device="cuda"),
            "grad_bz_event": torch.full((cfg.nevts,), float("nan"), dtype=torch.float64, device="cuda"),
        }
        rc = lib.p2r_forward_backward_noalloc(
            ctypes.byref(c), ptr(d_trk), ptr(d_hit), ptr(d_dr), None, ptr(out["trk_out"]), ptr(out["chi2"]),
            ptr(d_gtrk), ptr(d_gchi2), ptr(out["grad_trk_in"]), ptr(out["grad_hits"]), ptr(out["grad_dr"]),
            ptr(out["grad_bz"]), ptr(out["grad_dr_event"]), ptr(out["grad_bz_event"]), 5, stream)
        assert rc == 0, lib.p2r_last_error_string().decode()
        torch.cuda.synchronize()
        got = {k: v.cpu().numpy() for k, v in out.items()}
        for k in ("trk_out", "chi2"):
            a, b = got[k].reshape(-1), ref[k].reshape(-1)
            assert np.array_equal(np.isfinite(a), np.isfinite(b)), (call, k)
        for k in ("grad_trk_in", "grad_hits", "grad_dr", "grad_bz", "grad_dr_event", "grad_bz_event", "chi2"):
            e = _grad_err(got[k], ref[k])
            assert np.isfinite(got[k]).all() and e.max() < GRAD_RTOL, (call, k, e.max())
        q_in = trk.reshape(-1, 28, 32)[:, 27, :].view(np.int32)
        assert np.array_equal(got["trk_out"].reshape(-1, 28, 32)[:, 27, :].view(np.int32), q_in)


def test_noalloc_rejects_oversized_batch(p2r):
    # the size check runs before any device work; the arrays are null, so a call that got past
    # it would be rejected by the workspace entry point's null-input check, never launched
    cfg = p2r.Config(bsize=32, nlayer=64, nevts=10, nb=4000, bz=3.8, mode=p2r.MODE_CHAINED)
    lib = p2r.lib()
    c = cfg.c()
    rc = lib.p2r_forward_backward_noalloc(ctypes.byref(c), None, None, None, None, None, None, None, None, None,
                                          None, None, None, None, None, 5, None)
    assert rc == p2r._lib.P2R_ERR_WORKSPACE
    assert "scratch" in lib.p2r_last_error_string().decode()
