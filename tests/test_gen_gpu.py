"""The device-side helix generator against the host generator: same random streams and
arithmetic, so the arrays agree bit for bit except where CUDA's and the C library's
double-precision transcendentals round differently (then by one float ulp), including
per-event track counts (padding lanes) and several bsize / layer counts."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bs,nevts,nb,nlayer", [(32, 3, 7, 20), (1, 2, 5, 3), (64, 2, 3, 40), (96, 1, 2, 25)])
def test_device_generator_matches_host(bs, nevts, nb, nlayer):
    import torch
    import p2r_tests_b200 as p2r
    cfg = p2r.Config(bsize=bs, nlayer=nlayer, nevts=nevts, nb=nb, bz=3.8)
    gp = p2r.gen_params(bz=3.8, seed=1234 + bs, r_first=4.0, r_last=110.0)
    counts = None if bs == 1 else np.array([nb * bs - 5 - e for e in range(nevts)], np.int32)
    trk_h, hit_h = p2r.generate_helix(cfg, gp, ntrk_event=counts)
    trk_d, hit_d = p2r.generate_helix_device(cfg, gp, ntrk_event=counts)
    torch.cuda.synchronize()
    for host, dev in ((trk_h.reshape(-1), trk_d.cpu().numpy()), (hit_h.reshape(-1), hit_d.cpu().numpy())):
        a, b = host.view(np.int32).astype(np.int64), dev.view(np.int32).astype(np.int64)
        ulps = np.abs(a - b)
        assert ulps.max() <= 1, ulps.max()
        assert (ulps > 0).mean() < 1e-4, (ulps > 0).mean()


def test_device_generator_feeds_the_forward():
    """Generated on the device, the chained forward runs and every track stays finite."""
    import torch
    import p2r_tests_b200 as p2r
    cfg = p2r.Config(bsize=32, nlayer=20, nevts=4, nb=30, bz=3.8)
    trk, hit = p2r.generate_helix_device(cfg)
    out = torch.empty_like(trk)
    p2r.forward(cfg, trk, hit, out)
    assert p2r.count_nonfinite(out, cfg.nblocks, cfg.bsize) == 0


def test_device_generator_empty_and_invalid():
    import torch
    import p2r_tests_b200 as p2r
    cfg = p2r.Config(bsize=32, nlayer=20, nevts=0, nb=4, bz=3.8)
    p2r.generate_helix_device(cfg)  # empty batch: no launch
    with pytest.raises(p2r.P2RError):
        p2r.generate_helix_device(p2r.Config(bsize=32, nlayer=20, nevts=1, nb=1, bz=0.0))


def test_device_sort_by_layers_matches_host():
    """sort_by_layers_device orders each event's tracks like the host sort_by_layers, and the
    masked forward on the sorted arrays gives each track its unsorted result bit for bit."""
    import torch
    import p2r_tests_b200 as p2r
    cfg = p2r.Config(bsize=32, nlayer=12, nevts=3, nb=4, bz=3.8)
    trk, hit = p2r.generate_helix_device(cfg)
    nlay = torch.randint(1, 13, (cfg.ntracks,), dtype=torch.int32, device="cuda",
                         generator=torch.Generator("cuda").manual_seed(2))
    ts, hs, ns, perm = p2r.sort_by_layers_device(cfg, trk, hit, nlay)
    w = dict(trk=trk.cpu().numpy().reshape(cfg.nblocks, 28, 32), hit=hit.cpu().numpy(),
             nlay_lane=nlay.cpu().numpy(), event_block_offset=np.arange(cfg.nevts + 1) * cfg.nb, bsize=32,
             nlayer=cfg.nlayer, nblocks=cfg.nblocks)
    wh, ph = p2r.sort_by_layers(w)
    assert np.array_equal(perm.cpu().numpy(), ph)
    bits = lambda a: np.ascontiguousarray(a).reshape(-1).view(np.uint32)
    assert np.array_equal(bits(ts.cpu().numpy()), bits(wh["trk"])) and np.array_equal(bits(hs.cpu().numpy()), bits(wh["hit"]))
    a, b = torch.empty_like(trk), torch.empty_like(trk)
    p2r.forward(cfg, trk, hit, a, nlay_lane=nlay)
    p2r.forward(cfg, ts, hs, b, nlay_lane=ns)
    back = p2r.permute_tracks(b.cpu().numpy(), p2r.inverse(ph), 32, 28)
    assert np.array_equal(bits(back), bits(a.cpu().numpy()))
    # the same round trip on the device, for tracks and hits
    inv = p2r.inverse_device(perm)
    assert np.array_equal(bits(p2r.permute_tracks_device(b, inv, 32, 28).cpu().numpy()), bits(a.cpu().numpy()))
    assert torch.equal(p2r.permute_tracks_device(hs, inv, 32, 9, cfg.nlayer), hit)
