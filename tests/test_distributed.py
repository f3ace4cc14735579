"""Multi-process host logic on CPU: world_size-2 gloo ranks shard events and all-reduce the
calibration gradients; the result must equal a single-process computation over all tracks
(FP64 reference gradient of the oracle restatement standing in for the GPU adjoint)."""
import os
import socket

import numpy as np
import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_events_partitions():
    from p2r_tests_b200.distributed import shard_events, shard_uneven
    for nevts in (0, 1, 7, 100):
        for world in (1, 2, 3, 8):
            ranges = [shard_events(nevts, world, r) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == nevts
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            assert max(e - s for s, e in ranges) - min(e - s for s, e in ranges) <= 1
    counts = np.array([5000, 10, 10, 10, 3000, 2000, 50, 50])
    ranges = [shard_uneven(counts, 2, r) for r in range(2)]
    assert ranges[0][0] == 0 and ranges[-1][1] == len(counts) and ranges[0][1] == ranges[1][0]
    load = [counts[s:e].sum() for s, e in ranges]
    assert max(load) <= counts.sum() * 0.5 + counts.max()
    rng = np.random.default_rng(4)
    for world in (1, 3, 8):
        c = rng.integers(0, 500, 37)
        ranges = [shard_uneven(c, world, r) for r in range(world)]
        assert ranges[0][0] == 0 and ranges[-1][1] == len(c)
        assert all(a[1] == b[0] and a[0] <= a[1] for a, b in zip(ranges, ranges[1:]))
        assert max(c[s:e].sum() for s, e in ranges) <= c.sum() / world + c.max()
    for bad in ((counts, 0, 0), (counts, 2, 2), (counts, 2, -1), ([3, -1], 1, 0)):
        with pytest.raises(ValueError):
            shard_uneven(*bad)


def test_event_slice_is_the_events_byte_range():
    from p2r_tests_b200.distributed import event_slice
    a = np.arange(5 * 12, dtype=np.float32).reshape(5, 12)
    assert np.array_equal(event_slice(a, 1, 3, 5), a[1:3].reshape(-1))
    assert event_slice(a, 2, 2, 5).size == 0
    for bad in ((0, 1, 0), (0, 6, 5), (3, 2, 5), (0, 1, 7)):
        with pytest.raises(ValueError):
            event_slice(a, *bad)


def _grad_on_tracks(par0, cov0, q, hpos, hcov, dr, bz):
    import torch
    from oracle import p2r_torch
    drt = torch.tensor(dr, dtype=torch.float64, requires_grad=True)
    bzt = torch.tensor(bz, dtype=torch.float64, requires_grad=True)
    T = lambda a: torch.tensor(a, dtype=torch.float64)
    _, _, chi2 = p2r_torch.chained(T(par0), T(cov0), torch.tensor(q), T(hpos), T(hcov), drt, bzt)
    chi2.sum().backward()
    return drt.grad.detach().clone(), bzt.grad.detach().reshape(1).clone()


def _inputs():
    import p2r_tests_b200 as p2r
    cfg = p2r.Config(bsize=32, nlayer=12, nevts=4, nb=1, bz=3.8)
    trk, hit = p2r.generate_helix(cfg, p2r.gen_params(bz=3.8, seed=99, r_last=60.0))
    h = hit.reshape(cfg.nblocks, cfg.nlayer, 9, 32)
    par0, cov0, q = p2r.tracks_par(trk), p2r.tracks_cov(trk), p2r.tracks_q(trk)
    hpos = h[:, :, 0:3, :].transpose(0, 3, 1, 2).reshape(-1, cfg.nlayer, 3)
    hcov = h[:, :, 3:9, :].transpose(0, 3, 1, 2).reshape(-1, cfg.nlayer, 6)
    dr = np.linspace(-0.005, 0.005, cfg.nlayer)
    return cfg, par0, cov0, q, hpos, hcov, dr


def _worker(rank, world, port, out_path):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch
    import torch.distributed as dist
    from p2r_tests_b200.distributed import allreduce_calibration, shard_events
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        cfg, par0, cov0, q, hpos, hcov, dr = _inputs()
        e0, e1 = shard_events(cfg.nevts, world, rank)
        sel = slice(e0 * cfg.nb * 32, e1 * cfg.nb * 32)  # tracks of this rank's events
        gdr, gbz = _grad_on_tracks(par0[sel], cov0[sel], q[sel], hpos[sel], hcov[sel], dr, cfg.bz)
        allreduce_calibration(gdr, gbz)
        if rank == 0:
            np.save(out_path, np.concatenate([gdr.numpy(), gbz.numpy()]))
    finally:
        dist.destroy_process_group()


def test_two_rank_calibration_gradient_matches_single_process(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    out = str(tmp_path / "grad.npy")
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    got = np.load(out)
    cfg, par0, cov0, q, hpos, hcov, dr = _inputs()
    gdr, gbz = _grad_on_tracks(par0, cov0, q, hpos, hcov, dr, cfg.bz)
    want = np.concatenate([gdr.numpy(), gbz.numpy()])
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
