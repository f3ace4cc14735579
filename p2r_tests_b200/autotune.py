"""Autotuner: picks bsize, block shape, hit-staging depth, queue granularity and checkpoint
stride by timing the library's own launches on the target GPU.

The launch-shape sweep of the fused forward runs natively (p2r_autotune_forward); bsize is
a data-layout choice, so it is tuned here by re-laying the same tracks out at each width.
Results are cached in a JSON file keyed by GPU name, kind and workload signature
($P2R_TUNE_CACHE, default ~/.cache/p2r_b200/tune.json).
"""
from __future__ import annotations

import ctypes
import json
import os
import time
from pathlib import Path

import numpy as np

from ._lib import FLAG_ORDER_BY_LAYERS, CTuneResult, check, lib
from .api import Config, HIT_WORDS, TRK_WORDS, _stream


def cache_path() -> Path:
    return Path(os.environ.get("P2R_TUNE_CACHE", Path.home() / ".cache" / "p2r_b200" / "tune.json"))


def _load_cache() -> dict:
    try:
        return json.loads(cache_path().read_text())
    except (OSError, ValueError):
        return {}


def _store(key: str, value: dict) -> None:
    c = _load_cache()
    c[key] = value
    p = cache_path()
    try:
        p.parent.mkdir(parents=True, exist_ok=True)
        tmp = p.with_suffix(f".{os.getpid()}.tmp")  # one per process: ranks may store at once
        tmp.write_text(json.dumps(c, indent=1, sort_keys=True))
        os.replace(tmp, p)
    except OSError:
        pass  # a read-only home only loses the cache


def _gpu_name() -> str:
    import torch
    return torch.cuda.get_device_name()


def relayout(a: np.ndarray, words: int, nslots: int, bs_from: int, bs_to: int) -> np.ndarray:
    """Same tracks, another Matriplex width: (nblk, nslots, words, bs_from) -> (.., bs_to)."""
    x = np.ascontiguousarray(a).reshape(-1, nslots, words, bs_from).transpose(0, 3, 1, 2).reshape(-1, nslots, words)
    if x.shape[0] % bs_to:
        raise ValueError(f"{x.shape[0]} tracks do not fill blocks of {bs_to}")
    return np.ascontiguousarray(x.reshape(-1, bs_to, nslots, words).transpose(0, 2, 3, 1))


def tune_forward(cfg: Config, trk: np.ndarray, hit: np.ndarray, bsizes=(32, 64, 128), threads=(32, 64, 96, 128),
                 stages=(2, 4), reps: int = 20, use_cache: bool = True) -> dict:
    """Best (bsize, block_threads, stages) for p2r_forward on this workload (tracks per event
    must be divisible by every bsize tried)."""
    import torch
    ntr_ev = cfg.nb * cfg.bsize
    if not any(ntr_ev % bs == 0 for bs in bsizes):
        raise ValueError(f"no bsize of {tuple(bsizes)} divides the {ntr_ev} tracks per event")
    key = (f"{_gpu_name()}|forward|ntr_ev={ntr_ev}|nevts={cfg.nevts}|nlayer={cfg.nlayer}|mode={cfg.mode}"
           f"|flags={cfg.flags}|space={tuple(bsizes)}x{tuple(threads)}x{tuple(stages)}")
    if use_cache and key in _load_cache():
        return _load_cache()[key]
    th = np.array(threads, np.int32)
    stg = np.array(stages, np.int32)
    results = []
    for bs in bsizes:
        if ntr_ev % bs:
            continue
        t = relayout(trk, TRK_WORDS, 1, cfg.bsize, bs)
        h = relayout(hit, HIT_WORDS, cfg.nlayer, cfg.bsize, bs)
        c = Config(**{**cfg.__dict__, "bsize": bs, "nb": ntr_ev // bs})
        dt = torch.from_numpy(t.reshape(-1)).cuda()
        dh = torch.from_numpy(h.reshape(-1)).cuda()
        do = torch.empty_like(dt)
        r = CTuneResult()
        cc = c.c()
        check(lib().p2r_autotune_forward(ctypes.byref(cc), dt.data_ptr(), dh.data_ptr(), do.data_ptr(),
                                         th.ctypes.data, len(th), stg.ctypes.data, len(stg), reps, ctypes.byref(r),
                                         _stream(None)))
        for i in range(min(r.n_tried, 64)):
            results.append({"bsize": bs, "block_threads": r.tried_threads[i], "stages": r.tried_stages[i],
                            "ms": r.tried_ms[i]})
        del dt, dh, do
    best = min(results, key=lambda x: x["ms"])
    out = {**best, "tried": results, "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    _store(key, out)
    return out


def tune_queue(ntrk_event, bsizes=(32, 64, 128), granularity=(1, 2, 4, 8, 16), threads=(64, 128), stages=(4,),
               reps: int = 5, nlayer_max: int = 25, use_cache: bool = True, workloads: dict | None = None,
               order=(False, True)) -> dict:
    """Best (bsize, blocks_per_item, block_threads, stages, order) for the persistent queue launch.
    order True: each CTA orders its tracks by layer count (P2R_FLAG_ORDER_BY_LAYERS; block_threads
    0 = 8 warps per CTA or 128 = 4 warps, the hit-staging depth does not apply)."""
    import torch

    from .uneven import Queue, uneven_workload
    counts = np.asarray(ntrk_event, np.int64)
    sig = f"nevts={len(counts)}|ntr={int(counts.sum())}|median={int(np.median(counts))}|nlay={nlayer_max}"
    key = (f"{_gpu_name()}|queue|{sig}|space={tuple(bsizes)}x{tuple(granularity)}x{tuple(threads)}x{tuple(stages)}"
           f"x{tuple(order)}")
    if use_cache and key in _load_cache():
        return _load_cache()[key]
    results = []
    for bs in bsizes:
        w = (workloads or {}).get(bs) or uneven_workload(counts, bsize=bs, nlayer_max=nlayer_max)
        dt = torch.from_numpy(w["trk"].reshape(-1)).cuda()
        dh = torch.from_numpy(w["hit"].reshape(-1)).cuda()
        do = torch.empty_like(dt)
        shapes = [(g, nt, st, False) for g in granularity for nt in threads for st in stages if False in order]
        # ordered: 8 warps per CTA (block_threads 0, chunks of 512 tracks) or 4 (128, 256 tracks)
        shapes += [(g, nt, st, True) for g in granularity for nt in (0, 128) for st in stages[:1]
                   if True in order and bs <= 2 * (nt or 256)]
        for g, nt, st, ordered in shapes:
            q = Queue(w, blocks_per_item=g, block_threads=nt, stages=st,
                      flags=FLAG_ORDER_BY_LAYERS if ordered else 0)
            q.run(dt, dh, do)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                q.run(dt, dh, do)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            lat = q.event_latency_ns()
            results.append({"bsize": bs, "blocks_per_item": g, "block_threads": nt, "stages": st,
                            "order": ordered, "ms": ms, "updates_per_s": w["updates"] / (ms / 1e3),
                            "p50_event_ms": float(np.percentile(lat, 50)) / 1e6,
                            "p99_event_ms": float(np.percentile(lat, 99)) / 1e6})
        del dt, dh, do
    best = min(results, key=lambda x: x["ms"])
    out = {**best, "tried": results, "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    _store(key, out)
    return out


def tune_adjoint(cfg: Config, d_trk, d_hit, strides=(1, 2, 4, 5, 10), reps: int = 3, use_cache: bool = True,
                 max_workspace_bytes: int | None = None) -> dict:
    """Best checkpoint stride for p2r_forward_backward on device arrays d_trk / d_hit.
    A smaller stride keeps more of the state on the tape (faster reverse, larger workspace:
    27 values per track per checkpoint); strides whose workspace exceeds max_workspace_bytes
    are not tried (None: no limit)."""
    import torch

    from .autograd import forward_backward, workspace_size
    fits = [ck for ck in strides if max_workspace_bytes is None or workspace_size(cfg, ck) <= max_workspace_bytes]
    if not fits:
        raise ValueError(f"no checkpoint stride in {tuple(strides)} fits {max_workspace_bytes} bytes of workspace")
    key = (f"{_gpu_name()}|adjoint|ntr={cfg.ntracks}|nlayer={cfg.nlayer}|flags={cfg.flags}|strides={fits}")
    if use_cache and key in _load_cache():
        return _load_cache()[key]
    g_chi2 = torch.ones(cfg.ntracks, dtype=torch.float32, device=d_trk.device)
    results, ws = [], {}
    for ck in fits:
        forward_backward(cfg, d_trk, d_hit, grad_chi2=g_chi2, ckpt_stride=ck, out=ws)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            forward_backward(cfg, d_trk, d_hit, grad_chi2=g_chi2, ckpt_stride=ck, out=ws)
        e1.record()
        torch.cuda.synchronize()
        results.append({"ckpt_stride": ck, "ms": e0.elapsed_time(e1) / reps})
    best = min(results, key=lambda x: x["ms"])
    out = {**best, "tried": results, "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    _store(key, out)
    return out
