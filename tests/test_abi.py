"""CPU tests of the C ABI: the library loads, exports what include/p2r.h declares, and
rejects bad arguments with status codes (checked before any CUDA call, so no GPU needed)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    text = (ROOT / "include" / "p2r.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(p2r_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(p2r):
    lib = ctypes.CDLL(str(p2r.LIB_PATH))
    names = declared_functions()
    assert len(names) >= 12
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared in include/p2r.h but not exported: {missing}"


def test_binding_covers_header(p2r):
    from p2r_tests_b200 import _lib
    assert set(declared_functions()) == set(_lib.exported_symbols())


def test_abi_version_and_kfact(p2r):
    assert p2r.lib().p2r_abi_version() == 1
    header = (ROOT / "include" / "p2r.h").read_text()
    assert f"#define P2R_ABI_VERSION {p2r._lib.ABI_VERSION}" in header
    # kfact as the reference rounds its constant (TBB:654): float(100/(-0.299792458*3.8112))
    assert np.float32(p2r.kfact(3.8112)) == np.float32(100 / (-0.299792458 * 3.8112))
    assert p2r.kfact(0.0) == p2r.kfact(3.8112)


def _cfg(p2r, **kw):
    c = p2r.Config(bsize=32, nlayer=20, nevts=1, nb=1)
    for k, v in kw.items():
        setattr(c, k, v)
    return c.c()


@pytest.mark.usefixtures("host_only")
@pytest.mark.parametrize("bad,code", [
    (dict(bsize=0), 1), (dict(bsize=5000), 1), (dict(nlayer=0), 1), (dict(nevts=-1), 1), (dict(mode=7), 1),
    (dict(block_threads=100), 1), (dict(stages=9), 1),
])
def test_forward_rejects_bad_config(p2r, bad, code):
    l = p2r.lib()
    c = _cfg(p2r, **bad)
    rc = l.p2r_forward(ctypes.byref(c), 16, 32, 48, None, None, None)
    assert rc == code
    assert l.p2r_last_error_string().decode()


@pytest.mark.usefixtures("host_only")
def test_forward_rejects_null_and_alias(p2r):
    l = p2r.lib()
    c = _cfg(p2r)
    assert l.p2r_forward(ctypes.byref(c), None, 32, 48, None, None, None) == 1
    assert l.p2r_forward(ctypes.byref(c), 16, 32, 16, None, None, None) == 1
    assert "alias" in l.p2r_last_error_string().decode()
    assert l.p2r_forward(None, 16, 32, 48, None, None, None) == 1


@pytest.mark.usefixtures("host_only")
def test_per_layer_rejects_bad_layer(p2r):
    l = p2r.lib()
    c = _cfg(p2r)
    assert l.p2r_propagate_to_r(ctypes.byref(c), 16, 32, 20, 48, None, None) == 1
    assert l.p2r_kalman_update(ctypes.byref(c), 16, 32, -1, None, None) == 1
    assert "layer" in l.p2r_last_error_string().decode()


@pytest.mark.usefixtures("host_only")
def test_masked_needs_chained_and_counts(p2r):
    l = p2r.lib()
    c = _cfg(p2r, mode=0)
    assert l.p2r_forward_masked(ctypes.byref(c), 16, 32, 48, 64, None, None, None) == 1
    c = _cfg(p2r)
    assert l.p2r_forward_masked(ctypes.byref(c), 16, 32, 48, None, None, None, None) == 1


@pytest.mark.usefixtures("host_only")
def test_empty_work_is_ok_without_gpu(p2r):
    """nevts*nb == 0 returns OK before touching the device (an empty batch is valid)."""
    l = p2r.lib()
    c = _cfg(p2r, nevts=0)
    assert l.p2r_forward(ctypes.byref(c), 16, 32, 48, None, None, None) == 0


@pytest.mark.usefixtures("host_only")
def test_generators_reject_bad_args(p2r):
    l = p2r.lib()
    gp = p2r.gen_params()
    assert l.p2r_gen_helix(ctypes.byref(gp), 0, 1, 1, 20, None, 16, 32, 1) == 1
    assert l.p2r_gen_fixture(None, None, 1, None, 22, 32, 1, 1, 20, 1e-5, None, None) == 1
    buf = np.zeros(100, np.float32)
    assert l.p2r_gen_fixture(buf.ctypes.data, buf.ctypes.data, 1, buf.ctypes.data, 2, 32, 1, 1, 20, 1e-5,
                             buf.ctypes.data, buf.ctypes.data) == 1  # nlayer > input hits


@pytest.mark.usefixtures("host_only")
def test_adjoint_rejects_forward_only_options(p2r):
    """squash-phi is a forward-only option; the adjoint refuses it before any device work,
    and the tape workspace size grows with the tape and is reported for valid strides only."""
    l = p2r.lib()
    c = _cfg(p2r, flags=p2r.FLAG_SQUASH_PHI)
    rc = l.p2r_forward_backward(ctypes.byref(c), 16, 32, None, None, 48, None, None, None, None, None, None, None,
                                None, None, 5, 256, 1 << 20, None)
    assert rc == 4 and "SQUASH" in l.p2r_last_error_string().decode()
    c = _cfg(p2r, nevts=10, nb=30)
    small = l.p2r_forward_backward_workspace_size(ctypes.byref(c))
    tape1 = l.p2r_forward_backward_workspace_size_tape(ctypes.byref(c), 1)
    tape5 = l.p2r_forward_backward_workspace_size_tape(ctypes.byref(c), 5)
    assert small < tape5 < tape1
    assert tape1 >= small + 20 * 27 * 8 * 10 * 30 * 32  # 20 FP64 checkpoints per track
    assert l.p2r_forward_backward_workspace_size_tape(ctypes.byref(c), 3) == 0


@pytest.mark.usefixtures("host_only")
def test_misaligned_device_arrays_rejected(p2r):
    """Device arrays are read as 4-byte words (8-byte for doubles and 64-bit counters): a
    misaligned pointer is an INVALID argument on the host, before any launch (runs without a GPU)."""
    l = p2r.lib()
    c = _cfg(p2r)
    odd, ok = 0x10002, 0x10000  # fake device addresses: only their alignment is looked at

    def rejected(rc):
        return rc == 1 and "aligned" in l.p2r_last_error_string().decode()

    assert rejected(l.p2r_forward(ctypes.byref(c), odd, ok, ok + 64, None, None, None))
    assert rejected(l.p2r_forward(ctypes.byref(c), ok, ok + 64, ok + 128, odd, None, None))     # chi2_out
    assert rejected(l.p2r_forward_masked(ctypes.byref(c), ok, ok + 64, ok + 128, odd, None, None, None))
    assert rejected(l.p2r_propagate_to_r(ctypes.byref(c), ok, odd, 0, ok + 128, None, None))
    assert rejected(l.p2r_kalman_update(ctypes.byref(c), ok, ok + 64, 0, odd, None))
    assert rejected(l.p2r_count_nonfinite(odd, 1, 32, ok, None))
    assert rejected(l.p2r_count_nonfinite(ok, 1, 32, ok + 4, None))                             # 64-bit counter
    assert rejected(l.p2r_forward_backward(ctypes.byref(c), ok, ok + 64, None, None, ok + 128, None, None, None, None,
                                           None, ok + 4, None, None, None, 5, 256, 1 << 20, None))  # double grad_dr
    assert rejected(l.p2r_forward_host(ctypes.byref(c), ok, ok, ok, odd, ok, ok, 4, None))
    gp = p2r.gen_params()
    assert rejected(l.p2r_gen_helix_device(ctypes.byref(gp), 32, 1, 1, 20, None, odd, ok, None))
    assert rejected(l.p2r_fp64_fma_probe(1, 1, 32, ok + 4, None))


@pytest.mark.usefixtures("host_only")
def test_bindings_check_array_types_and_sizes(p2r, monkeypatch):
    """The library sees bare pointers, so the Python bindings check each tensor's type and
    size first: a float16 track array or a short radius-offset vector would otherwise be read
    or written past its end. Pointer and stream extraction are replaced by None here (no GPU), so a call
    whose tensors pass the checks reaches the library and stops at its null-pointer check."""
    import torch
    from p2r_tests_b200 import api, autograd
    for mod in (api, autograd):
        monkeypatch.setattr(mod, "_ptr", lambda t: None)
        monkeypatch.setattr(mod, "_stream", lambda s: None)
    cfg = p2r.Config(bsize=32, nlayer=4, nevts=1, nb=2)
    f32 = lambda n, dt=torch.float32: torch.zeros(n, dtype=dt)
    trk, hit = f32(cfg.nblocks * 28 * 32), f32(cfg.nblocks * 4 * 9 * 32)
    out, chi2, dr, nlay = torch.zeros_like(trk), f32(cfg.ntracks), f32(4), torch.zeros(cfg.ntracks, dtype=torch.int32)

    def fails(fn, *words):
        with pytest.raises(p2r.P2RError) as e:
            fn()
        msg = str(e.value)
        assert all(w in msg for w in words), msg

    fails(lambda: p2r.forward(cfg, trk, hit, out, chi2=chi2, dr=dr, nlay_lane=nlay), "null")  # checks pass
    fails(lambda: p2r.forward(cfg, trk.half().repeat(2)[:trk.numel()], hit, out), "float32", "float16")
    fails(lambda: p2r.forward(cfg, trk, hit, out.double()), "float64")
    fails(lambda: p2r.forward(cfg, trk, hit, out, dr=dr.double()), "dr", "float64")
    fails(lambda: p2r.forward(cfg, trk, hit, out, dr=dr[:3]), "dr", "3 elements", "4 needed")
    fails(lambda: p2r.forward(cfg, trk, hit, out, chi2=chi2[:-1]), "chi2")
    fails(lambda: p2r.forward(cfg, trk, hit, out, nlay_lane=nlay.long()), "nlay_lane", "int64")
    fails(lambda: p2r.propagateToR(cfg, trk, hit, 0, out, dr=dr.half()), "dr")
    fails(lambda: p2r.KalmanUpdate(cfg, out, hit, 0, chi2_accum=chi2.double()), "chi2_accum")
    fails(lambda: p2r.count_nonfinite(trk[:-1], cfg.nblocks, 32), "trk", "needed")
    fails(lambda: p2r.fp64_fma_probe(f32(256), 1, 1, 256), "out", "float32")

    h_trk, h_hit = trk.numpy(), hit.numpy()
    fails(lambda: p2r.forward_host(cfg, h_trk, h_hit, h_trk.copy(), trk, hit, out), "null")  # checks pass
    fails(lambda: p2r.forward_host(cfg, h_trk.view(np.float64), h_hit, h_trk.copy(), trk, hit, out), "float32")

    def adj(**out_entries):
        o = {"grad_hits": None, **out_entries}
        return p2r.forward_backward(cfg, trk, hit, dr=dr, grad_chi2=chi2, ckpt_stride=5, out=o)
    fails(lambda: adj(), "null input")  # checks pass
    fails(lambda: adj(grad_dr=f32(4)), "grad_dr", "float32")
    fails(lambda: adj(grad_trk_in=f32(trk.numel() - 1)), "grad_trk_in", "needed")
    fails(lambda: p2r.forward_backward(cfg, trk, hit, dr=dr, grad_chi2=chi2, ckpt_stride=5, per_event=True,
                                       out={"grad_bz_event": f32(0, torch.float64)}), "grad_bz_event")


@pytest.mark.usefixtures("host_only")
def test_overlapping_arrays_rejected(p2r):
    """A written array may not share bytes with another array of the same call (one track's
    writes would land in another's inputs); the per-layer propagation may run exactly in place.
    Only the fake addresses' byte ranges are compared, on the host (runs without a GPU)."""
    l = p2r.lib()
    c = _cfg(p2r)  # one block of 32 tracks, 20 layers
    tb, hb, lb = 28 * 32 * 4, 20 * 9 * 32 * 4, 32 * 4
    base = 1 << 32
    t_in, hits, t_out = base, base + (1 << 20), base + (2 << 20)

    def overlap(rc, *words):
        msg = l.p2r_last_error_string().decode()
        return rc == 1 and "overlap" in msg and all(w in msg for w in words)

    assert overlap(l.p2r_forward(ctypes.byref(c), t_in, hits, t_in + 256, None, None, None), "trk_in")
    assert overlap(l.p2r_forward(ctypes.byref(c), t_in, hits, hits + hb - 256, None, None, None), "hits")
    assert overlap(l.p2r_forward(ctypes.byref(c), t_in, hits, t_out, t_out + tb - 64, None, None), "chi2_out")
    assert overlap(l.p2r_forward(ctypes.byref(c), t_in, hits, t_out, t_in, None, None), "chi2_out", "trk_in")
    assert overlap(l.p2r_forward_masked(ctypes.byref(c), t_in, hits, t_out, t_out + 64, None, None, None), "nlay")
    assert overlap(l.p2r_propagate_to_r(ctypes.byref(c), t_in, hits, 0, t_in + 128, None, None), "trk_in")
    assert overlap(l.p2r_propagate_to_r(ctypes.byref(c), t_out, hits, 0, t_out, t_out + 64, None), "dr")
    assert overlap(l.p2r_kalman_update(ctypes.byref(c), t_out, t_out + tb - 256, 0, None, None), "hits")
    assert overlap(l.p2r_kalman_update(ctypes.byref(c), t_out, hits, 0, hits + lb, None), "chi2_accum")
    h = np.zeros(tb + hb, np.uint8)  # host buffers are never dereferenced before the device checks
    assert overlap(l.p2r_forward_host(ctypes.byref(c), h.ctypes.data, h.ctypes.data, h.ctypes.data, t_in, t_in + tb - 4,
                                      t_out, 4, None), "dev_trk_in", "dev_hits")
    assert overlap(l.p2r_forward_host(ctypes.byref(c), h.ctypes.data, h.ctypes.data, h.ctypes.data, t_in, hits,
                                      hits + 4096, 4, None), "dev_hits", "dev_trk_out")
    # adjacent ranges do not overlap. A call that passed every check would launch, so the
    # boundary is shown with a launch shape that is rejected after the overlap checks.
    bad_shape = _cfg(p2r, block_threads=100)
    a_in, a_out, a_hit, a_chi2 = base, base + tb, base + 2 * tb, base + 2 * tb + hb  # end to end
    assert l.p2r_forward(ctypes.byref(bad_shape), a_in, a_hit, a_out, a_chi2, None, None) == 1
    assert "block_threads" in l.p2r_last_error_string().decode()
    assert overlap(l.p2r_forward(ctypes.byref(bad_shape), a_in, a_hit, a_out - 4, None, None, None))


@pytest.mark.usefixtures("host_only")
def test_adjoint_overlapping_arrays_rejected(p2r):
    """p2r_forward_backward (and so its allocation-free variant): no written array (outputs,
    gradients, workspace) may share a byte with another array of the call. Fake addresses,
    compared on the host only."""
    l = p2r.lib()
    c = _cfg(p2r)  # one block of 32 tracks, 20 layers
    c.mode = p2r.MODE_CHAINED
    tb, hb, lb = 28 * 32 * 4, 20 * 9 * 32 * 4, 32 * 4
    need = l.p2r_forward_backward_workspace_size(ctypes.byref(c))
    base = 1 << 33
    a = {n: base + i * (1 << 20) for i, n in enumerate(
        ("trk_in", "hits", "dr", "nlay", "trk_out", "chi2", "g_out", "g_chi2", "g_in", "g_hits", "g_dr", "g_bz",
         "g_dr_ev", "g_bz_ev", "ws"))}

    def call(**over):
        v = {**a, **over}
        return l.p2r_forward_backward(ctypes.byref(c), v["trk_in"], v["hits"], v["dr"], v["nlay"], v["trk_out"],
                                      v["chi2"], v["g_out"], v["g_chi2"], v["g_in"], v["g_hits"], v["g_dr"],
                                      v["g_bz"], v["g_dr_ev"], v["g_bz_ev"], 5, v["ws"], need, None)

    def overlap(rc, *words):
        msg = l.p2r_last_error_string().decode()
        return rc == 1 and "overlap" in msg and all(w in msg for w in words)

    assert overlap(call(trk_out=a["trk_in"] + 256), "trk_in", "trk_out")
    assert overlap(call(g_in=a["hits"] + hb - 4), "hits", "grad_trk_in")
    assert overlap(call(g_hits=a["trk_out"] + tb - 8), "trk_out", "grad_hits")
    assert overlap(call(chi2=a["g_chi2"]), "grad_chi2", "chi2_out")
    assert overlap(call(g_dr=a["dr"]), "dr", "grad_dr")
    assert overlap(call(g_bz=a["g_dr"] + 8 * 19), "grad_dr", "grad_bz")
    assert overlap(call(g_bz_ev=a["g_dr_ev"]), "grad_dr_event", "grad_bz_event")
    assert overlap(call(ws=a["g_out"]), "grad_trk_out", "workspace")
    assert overlap(call(nlay=a["chi2"] + lb - 4), "nlay_lane", "chi2_out")
    # two read-only arrays may share memory (the same hits passed twice is harmless) ...
    assert not overlap(call(g_out=a["trk_in"], trk_in=a["trk_in"], ws=a["ws"] + 1))
    # ... that call was rejected by the workspace alignment check after the overlap checks
    assert "256-byte" in l.p2r_last_error_string().decode()


@pytest.mark.usefixtures("host_only")
def test_queue_overlapping_arrays_rejected(p2r):
    """p2r_run_queue: outputs, timestamps and workspace may not overlap any array of the call."""
    from p2r_tests_b200._lib import CQueue
    l = p2r.lib()
    base = 1 << 34
    off, items, nlay = base, base + (1 << 20), base + (2 << 20)
    t_in, hits, t_out = base + (3 << 20), base + (4 << 20), base + (5 << 20)
    chi2, done, start, ws = base + (6 << 20), base + (7 << 20), base + (8 << 20), base + (9 << 20)
    q = CQueue(32, 20, 2, 2, 3.8, 0, 0, 0, 0, off, items, 2, nlay)
    need = l.p2r_queue_workspace_size(ctypes.byref(q))

    def call(**over):
        v = dict(t_in=t_in, hits=hits, t_out=t_out, chi2=chi2, done=done, start=start, ws=ws)
        v.update(over)
        return l.p2r_run_queue(ctypes.byref(q), v["t_in"], v["hits"], v["t_out"], v["chi2"], v["done"], v["start"],
                               v["ws"], need, None)

    def overlap(rc, *words):
        msg = l.p2r_last_error_string().decode()
        return rc == 1 and "overlap" in msg and all(w in msg for w in words)

    assert overlap(call(t_out=t_in + 64), "trk_in", "trk_out")
    assert overlap(call(chi2=nlay), "nlay_lane", "chi2_out")
    assert overlap(call(done=items), "items", "event_done_ns")
    assert overlap(call(start=off + 8), "event_block_offset", "start_ns")
    assert overlap(call(ws=t_out + 256), "trk_out", "workspace")
    assert overlap(call(ws=hits), "hits", "workspace")
