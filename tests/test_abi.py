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


def test_forward_rejects_null_and_alias(p2r):
    l = p2r.lib()
    c = _cfg(p2r)
    assert l.p2r_forward(ctypes.byref(c), None, 32, 48, None, None, None) == 1
    assert l.p2r_forward(ctypes.byref(c), 16, 32, 16, None, None, None) == 1
    assert "alias" in l.p2r_last_error_string().decode()
    assert l.p2r_forward(None, 16, 32, 48, None, None, None) == 1


def test_per_layer_rejects_bad_layer(p2r):
    l = p2r.lib()
    c = _cfg(p2r)
    assert l.p2r_propagate_to_r(ctypes.byref(c), 16, 32, 20, 48, None, None) == 1
    assert l.p2r_kalman_update(ctypes.byref(c), 16, 32, -1, None, None) == 1
    assert "layer" in l.p2r_last_error_string().decode()


def test_masked_needs_chained_and_counts(p2r):
    l = p2r.lib()
    c = _cfg(p2r, mode=0)
    assert l.p2r_forward_masked(ctypes.byref(c), 16, 32, 48, 64, None, None, None) == 1
    c = _cfg(p2r)
    assert l.p2r_forward_masked(ctypes.byref(c), 16, 32, 48, None, None, None, None) == 1


def test_empty_work_is_ok_without_gpu(p2r):
    """nevts*nb == 0 returns OK before touching the device (an empty batch is valid)."""
    l = p2r.lib()
    c = _cfg(p2r, nevts=0)
    assert l.p2r_forward(ctypes.byref(c), 16, 32, 48, None, None, None) == 0


def test_generators_reject_bad_args(p2r):
    l = p2r.lib()
    gp = p2r.gen_params()
    assert l.p2r_gen_helix(ctypes.byref(gp), 0, 1, 1, 20, None, 16, 32, 1) == 1
    assert l.p2r_gen_fixture(None, None, 1, None, 22, 32, 1, 1, 20, 1e-5, None, None) == 1
    buf = np.zeros(100, np.float32)
    assert l.p2r_gen_fixture(buf.ctypes.data, buf.ctypes.data, 1, buf.ctypes.data, 2, 32, 1, 1, 20, 1e-5,
                             buf.ctypes.data, buf.ctypes.data) == 1  # nlayer > input hits


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
