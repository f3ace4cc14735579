"""The autotuner: re-layout and cache on the CPU; on the GPU, that each tuner returns the
fastest of the candidates it timed, and that the shape it picks computes the same results as
the default launch (launch shape and bsize are performance choices only)."""
import ctypes

import numpy as np
import pytest


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)  # the q row holds integer bits


def test_relayout_round_trip_and_placement(p2r):
    from p2r_tests_b200.autotune import relayout
    rng = np.random.default_rng(0)
    nblk, nslots, words = 6, 3, 9
    a = rng.standard_normal((nblk, nslots, words, 32)).astype(np.float32)
    b = relayout(a, words, nslots, 32, 64)
    assert b.shape == (3, nslots, words, 64)
    for t in (0, 31, 32, 77, 191):  # track t: lane t % bs of block t // bs
        assert np.array_equal(b[t // 64, :, :, t % 64], a[t // 32, :, :, t % 32])
    assert np.array_equal(relayout(b, words, nslots, 64, 32), a)
    assert np.array_equal(relayout(relayout(a, words, nslots, 32, 1), words, nslots, 1, 32), a)


def test_relayout_rejects_partial_blocks(p2r):
    from p2r_tests_b200.autotune import relayout
    with pytest.raises(ValueError):
        relayout(np.zeros((3, 1, 28, 32), np.float32), 28, 1, 32, 64)  # 96 tracks, blocks of 64


def test_cache_store_load_and_corrupt_file(p2r, tmp_path, monkeypatch):
    from p2r_tests_b200 import autotune
    f = tmp_path / "sub" / "tune.json"
    monkeypatch.setenv("P2R_TUNE_CACHE", str(f))
    assert autotune._load_cache() == {}
    autotune._store("gpu|forward|x", {"bsize": 64, "ms": 0.5})
    autotune._store("gpu|queue|y", {"bsize": 32, "ms": 1.5})
    assert autotune._load_cache() == {"gpu|forward|x": {"bsize": 64, "ms": 0.5}, "gpu|queue|y": {"bsize": 32, "ms": 1.5}}
    assert sorted(x.name for x in f.parent.iterdir()) == ["tune.json"]  # no temporary file left
    f.write_text("{not json")
    assert autotune._load_cache() == {}


def test_tune_forward_rejects_widths_that_split_events(p2r):
    from p2r_tests_b200 import autotune
    cfg = p2r.Config(bsize=32, nlayer=4, nevts=2, nb=3)  # 96 tracks per event
    with pytest.raises(ValueError, match="divides"):
        autotune.tune_forward(cfg, None, None, bsizes=(64, 128))


def test_native_tuner_rejects_bad_arguments(p2r):
    """Argument errors come back before any CUDA call (runs without a GPU)."""
    l = p2r.lib()
    c = p2r.Config(bsize=32, nlayer=20, nevts=1, nb=1).c()
    th = np.array([64], np.int32)
    st = np.array([4], np.int32)
    r = p2r._lib.CTuneResult()
    E = p2r._lib.P2R_ERR_INVALID
    assert l.p2r_autotune_forward(None, None, None, None, th.ctypes.data, 1, st.ctypes.data, 1, 1, ctypes.byref(r), None) == E
    assert l.p2r_autotune_forward(ctypes.byref(c), None, None, None, th.ctypes.data, 0, st.ctypes.data, 1, 1,
                                  ctypes.byref(r), None) == E
    assert l.p2r_autotune_forward(ctypes.byref(c), None, None, None, th.ctypes.data, 1, st.ctypes.data, 1, 0,
                                  ctypes.byref(r), None) == E
    assert l.p2r_autotune_forward(ctypes.byref(c), None, None, None, th.ctypes.data, 1, st.ctypes.data, 1, 1,
                                  None, None) == E


@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


@pytest.fixture(scope="module")
def helix(p2r):
    cfg = p2r.Config(bsize=32, nlayer=20, nevts=4, nb=12, bz=3.8, mode=p2r.MODE_CHAINED)
    trk, hit = p2r.generate_helix(cfg, p2r.gen_params(bz=3.8, seed=11))
    return cfg, trk, hit


@pytest.mark.gpu
def test_native_tuner_times_every_candidate(p2r, torch, helix):
    cfg, trk, hit = helix
    d_trk = torch.from_numpy(trk.reshape(-1)).cuda()
    d_hit = torch.from_numpy(hit.reshape(-1)).cuda()
    d_out = torch.empty_like(d_trk)
    th = np.array([32, 64, 128], np.int32)
    st = np.array([2, 4], np.int32)
    r = p2r._lib.CTuneResult()
    c = cfg.c()
    p2r._lib.check(p2r.lib().p2r_autotune_forward(ctypes.byref(c), d_trk.data_ptr(), d_hit.data_ptr(),
                                                  d_out.data_ptr(), th.ctypes.data, 3, st.ctypes.data, 2, 2,
                                                  ctypes.byref(r), None))
    torch.cuda.synchronize()
    assert r.n_tried == 6
    tried = [(r.tried_threads[i], r.tried_stages[i], r.tried_ms[i]) for i in range(6)]
    assert sorted((a, b) for a, b, _ in tried) == sorted((a, b) for a in (32, 64, 128) for b in (2, 4))
    assert all(ms > 0 for _, _, ms in tried)
    assert r.best_ms == min(ms for _, _, ms in tried)
    assert (r.block_threads, r.stages) in [(a, b) for a, b, ms in tried if ms == r.best_ms]
    # the buffer holds the last candidate's output: the same bits as the default launch
    ref = torch.empty_like(d_trk)
    p2r.forward(cfg, d_trk, d_hit, ref)
    assert np.array_equal(bits(d_out.cpu().numpy()), bits(ref.cpu().numpy()))
    # an invalid candidate is an error, not a silent skip
    bad = np.array([48], np.int32)
    assert p2r.lib().p2r_autotune_forward(ctypes.byref(c), d_trk.data_ptr(), d_hit.data_ptr(), d_out.data_ptr(),
                                          bad.ctypes.data, 1, st.ctypes.data, 1, 1, ctypes.byref(r), None) \
        == p2r._lib.P2R_ERR_INVALID


@pytest.mark.gpu
def test_tune_forward_choice_reproduces_default_results(p2r, torch, helix, tmp_path, monkeypatch):
    from p2r_tests_b200 import autotune
    monkeypatch.setenv("P2R_TUNE_CACHE", str(tmp_path / "tune.json"))
    from p2r_tests_b200.api import HIT_WORDS, TRK_WORDS
    cfg, trk, hit = helix
    t = autotune.tune_forward(cfg, trk, hit, bsizes=(32, 64, 128), threads=(64, 128), stages=(2, 4), reps=2,
                              use_cache=False)
    assert len(t["tried"]) == 3 * 2 * 2
    assert t["ms"] == min(x["ms"] for x in t["tried"])
    ref = torch.empty(trk.size, dtype=torch.float32, device="cuda")
    p2r.forward(cfg, torch.from_numpy(trk.reshape(-1)).cuda(), torch.from_numpy(hit.reshape(-1)).cuda(), ref)
    bs = t["bsize"]
    c = p2r.Config(**{**cfg.__dict__, "bsize": bs, "nb": cfg.nb * cfg.bsize // bs,
                      "block_threads": t["block_threads"], "stages": t["stages"]})
    tt = autotune.relayout(trk, TRK_WORDS, 1, cfg.bsize, bs)
    hh = autotune.relayout(hit, HIT_WORDS, cfg.nlayer, cfg.bsize, bs)
    out = torch.empty(tt.size, dtype=torch.float32, device="cuda")
    p2r.forward(c, torch.from_numpy(tt.reshape(-1)).cuda(), torch.from_numpy(hh.reshape(-1)).cuda(), out)
    back = autotune.relayout(out.cpu().numpy(), TRK_WORDS, 1, bs, cfg.bsize)
    assert np.array_equal(bits(back), bits(ref.cpu().numpy().reshape(back.shape)))


@pytest.mark.gpu
def test_tune_queue_choice_reproduces_results(p2r, torch, tmp_path, monkeypatch):
    from p2r_tests_b200 import autotune
    monkeypatch.setenv("P2R_TUNE_CACHE", str(tmp_path / "tune.json"))
    counts = p2r.lognormal_counts(8, median=120, sigma=0.8, lo=5, hi=600, seed=9)
    t = autotune.tune_queue(counts, bsizes=(32, 64), granularity=(1, 4), threads=(64, 128), stages=(4,), reps=1,
                            use_cache=False)
    # per bsize: 2 granularities x 2 block shapes, plus 2 granularities x 2 CTA sizes with
    # in-launch ordering
    assert len(t["tried"]) == 2 * (2 * 2 + 2 * 2)
    assert sum(1 for x in t["tried"] if x["order"]) == 8
    assert t["ms"] == min(x["ms"] for x in t["tried"])
    assert all(x["p50_event_ms"] <= x["p99_event_ms"] for x in t["tried"])
    w = p2r.uneven_workload(counts, bsize=t["bsize"], nlayer_max=25)
    dt = torch.from_numpy(w["trk"].reshape(-1)).cuda()
    dh = torch.from_numpy(w["hit"].reshape(-1)).cuda()
    outs = []
    fl = p2r.FLAG_ORDER_BY_LAYERS if t["order"] else 0
    for g, nt, f in ((t["blocks_per_item"], t["block_threads"], fl), (1, 64, 0)):
        o = torch.empty_like(dt)
        p2r.Queue(w, blocks_per_item=g, block_threads=nt, stages=t["stages"], flags=f).run(dt, dh, o)
        outs.append(bits(o.cpu().numpy()))
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.gpu
def test_tune_adjoint_picks_a_timed_stride(p2r, torch, helix, tmp_path, monkeypatch):
    from p2r_tests_b200 import autotune
    monkeypatch.setenv("P2R_TUNE_CACHE", str(tmp_path / "tune.json"))
    cfg, trk, hit = helix
    d_trk = torch.from_numpy(trk.reshape(-1)).cuda()
    d_hit = torch.from_numpy(hit.reshape(-1)).cuda()
    t = autotune.tune_adjoint(cfg, d_trk, d_hit, strides=(1, 5, 10), reps=1, use_cache=False)
    assert [x["ckpt_stride"] for x in t["tried"]] == [1, 5, 10]
    assert t["ckpt_stride"] in (1, 5, 10) and t["ms"] == min(x["ms"] for x in t["tried"])
    # a workspace budget below the stride-1 tape leaves only the larger strides
    budget = max(p2r.workspace_size(cfg, 5), p2r.workspace_size(cfg, 10))  # 10 keeps a 9-slot segment buffer
    assert p2r.workspace_size(cfg, 1) > budget
    t = autotune.tune_adjoint(cfg, d_trk, d_hit, strides=(1, 5, 10), reps=1, use_cache=False,
                              max_workspace_bytes=budget)
    assert [x["ckpt_stride"] for x in t["tried"]] == [5, 10]
    with pytest.raises(ValueError):
        autotune.tune_adjoint(cfg, d_trk, d_hit, strides=(1,), reps=1, use_cache=False, max_workspace_bytes=budget)
