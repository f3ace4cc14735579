"""The reference's own CUDA kernels (src/propagate-tor-test_cuda_v4.cu GPUsequence, chained;
src/propagate-tor-test_cuda_uvm.cu launch_p2r_kernel, restart), compiled unmodified into
oracle/_ref for the benchmark workload's sizes (9600 tracks x 100 events x 20 layers, bsize 32),
run on the same device inputs as this library's fused forward.

They are a timed comparison point in bench.py; here they are checked to run on this GPU and to
agree with this library's output as two FP32 implementations of the same arithmetic do: each
error quantile of this library against the FP64 oracle within 2x of the reference GPU kernel's
(event 0; the kernels are compiled for the whole workload). The reference's kfact is its
compiled-in 3.8112 T, so the inputs are generated for that field."""
import numpy as np
import pytest

from tests import parity

pytestmark = pytest.mark.gpu

NTRK, NEV, NL, BS, BZ = 9600, 100, 20, 32, 3.8112


@pytest.fixture(scope="module")
def inputs(p2r):
    import torch
    from oracle.oracle import refgpu_available
    if not (refgpu_available("v4") and refgpu_available("uvm")):
        pytest.skip("reference GPU builds (oracle/_ref/libp2r_refgpu_*.so) missing")
    cfg = p2r.Config(bsize=BS, nlayer=NL, nevts=NEV, nb=NTRK // BS, bz=BZ)
    t, h = p2r.generate_helix_device(cfg, p2r.gen_params(bz=BZ, seed=20240011))
    torch.cuda.synchronize()
    return cfg, t, h


@pytest.mark.parametrize("kind", ["v4", "uvm"])
def test_reference_gpu_kernel_agrees(p2r, oracle, inputs, kind):
    import torch
    from oracle.oracle import RefGPU
    cfg, t, h = inputs
    r = RefGPU(kind)
    assert r.sizes() == (cfg.nevts, cfg.nb, cfg.nlayer, cfg.bsize)
    ref_out = torch.empty_like(t)
    ms = r.run(t.data_ptr(), h.data_ptr(), ref_out.data_ptr(), 1, 2, torch.cuda.current_stream().cuda_stream)
    assert ms > 0
    mode = p2r.MODE_CHAINED if r.chained else p2r.MODE_RESTART
    c = p2r.Config(**{**cfg.__dict__, "mode": mode})
    ours = torch.empty_like(t)
    p2r.forward(c, t, h, ours)
    torch.cuda.synchronize()
    tw, hw = 28 * BS * cfg.nb, 9 * BS * cfg.nb * NL
    trk0, hit0 = t[:tw].cpu().numpy(), h[:hw].cpu().numpy()
    f64 = oracle.run(trk0, hit0, BS, NL, mode, BZ, "f64")
    a, b = ours[:tw].cpu().numpy(), ref_out[:tw].cpu().numpy()
    assert np.array_equal(parity.unpack(a, BS)[2], parity.unpack(b, BS)[2])  # charges
    fin = np.isfinite(f64["par"]).all(1)
    assert fin.mean() > 0.98
    ap, ac, _ = parity.unpack(a, BS)
    bp, bc, _ = parity.unpack(b, BS)
    qa = parity.error_quantiles(ap[fin], ac[fin], f64["par"][fin], f64["cov"][fin], f64["prior"][fin])
    qb = parity.error_quantiles(bp[fin], bc[fin], f64["par"][fin], f64["cov"][fin], f64["prior"][fin])
    for x, y in zip(np.concatenate(qa), np.concatenate(qb)):
        assert x <= parity.ACC_FACTOR * y + 1e-7, (kind, qa, qb)
