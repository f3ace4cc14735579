"""Uneven batches through the persistent work-queue launch (p2r_run_queue) and its CUDA graph.

`uneven_workload` builds the batched workload: events with log-normal track counts (blocks
padded to bsize, padding lanes given zero layers) and uniform per-track layer counts, hits
on nlayer_max cylinders. `Queue` holds the device-side description, the workspace and the
per-event completion timestamps, and runs the launch directly or through a captured graph.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import CQueue, CQueueItem, P2RError, check, lib
from .api import Config, HIT_WORDS, TRK_WORDS, _arg, _ptr, _stream, gen_params, generate_helix


def lognormal_counts(nevts: int, median: float = 2000.0, sigma: float = 1.0, lo: int = 50, hi: int = 20000,
                     seed: int = 7) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.clip(np.round(median * np.exp(sigma * rng.standard_normal(nevts))), lo, hi).astype(np.int64)


def uneven_workload(ntrk_event, bsize: int = 32, nlayer_max: int = 25, lay_lo: int = 10, lay_hi: int = 25,
                    bz: float = 3.8, seed: int = 20240002, r_first: float = 20.0, r_last: float = 100.0) -> dict:
    """Host arrays of an uneven batch. Returns dict(trk, hit, nlay_lane, event_block_offset,
    ntrk_event, nblocks, updates)."""
    ntrk_event = np.asarray(ntrk_event, np.int64)
    nb_event = (ntrk_event + bsize - 1) // bsize
    off = np.zeros(len(ntrk_event) + 1, np.int64)
    off[1:] = np.cumsum(nb_event)
    nblocks = int(off[-1])
    cfg = Config(bsize=bsize, nlayer=nlayer_max, nevts=1, nb=nblocks, bz=bz)
    trk, hit = generate_helix(cfg, gen_params(bz=bz, seed=seed, r_first=r_first, r_last=r_last))
    rng = np.random.default_rng(seed)
    nlay = rng.integers(lay_lo, lay_hi + 1, nblocks * bsize).astype(np.int32)
    # lanes past an event's track count are padding: no layers
    lane_in_event = np.arange(nblocks * bsize) - np.repeat(off[:-1] * bsize, nb_event * bsize)
    nlay[lane_in_event >= np.repeat(ntrk_event, nb_event * bsize)] = 0
    return dict(trk=trk, hit=hit, nlay_lane=nlay, event_block_offset=off, ntrk_event=ntrk_event,
                nblocks=nblocks, bsize=bsize, nlayer=nlayer_max, bz=bz, updates=int(nlay.sum()))


def permute_tracks(arr: np.ndarray, perm: np.ndarray, bsize: int, words: int, nlayer: int = 1) -> np.ndarray:
    """Matriplex array (tracks: words=28, nlayer=1; hits: words=9, nlayer layers per block)
    with its tracks reordered: track i of the result is track perm[i] of arr."""
    a = np.ascontiguousarray(arr).reshape(-1, nlayer, words, bsize)
    nblocks = a.shape[0]
    t = a.transpose(0, 3, 1, 2).reshape(nblocks * bsize, nlayer, words)[perm]
    return np.ascontiguousarray(t.reshape(nblocks, bsize, nlayer, words).transpose(0, 2, 3, 1)).reshape(arr.shape)


def sort_by_layers(w: dict) -> tuple[dict, np.ndarray]:
    """The same uneven workload with each event's tracks ordered by layer count, longest first.

    A warp runs until the longest of its 32 tracks is done, so with layer counts spread over
    10-25 about a third of the lanes idle at the end; grouping tracks of similar length in the
    same 32-lane slices keeps them busy. Events stay where they are (padding lanes, which have
    no layers, stay at the end of their event), and every track's result is bit-identical in
    either order. Returns (workload, perm): track i of the new arrays is track perm[i] of the
    old ones; permute_tracks(out, inverse(perm), ...) puts outputs back in the old order."""
    bs, nl = w["bsize"], w["nlayer"]
    off = np.asarray(w["event_block_offset"], np.int64)
    nlay = np.asarray(w["nlay_lane"])
    perm = np.arange(w["nblocks"] * bs)
    for e in range(len(off) - 1):
        a, b = off[e] * bs, off[e + 1] * bs
        perm[a:b] = a + np.argsort(-nlay[a:b], kind="stable")
    out = dict(w)
    out["trk"] = permute_tracks(w["trk"], perm, bs, 28)
    out["hit"] = permute_tracks(w["hit"], perm, bs, 9, nl)
    out["nlay_lane"] = np.ascontiguousarray(nlay[perm])
    return out, perm


def sort_by_layers_device(cfg: Config, trk, hits, nlay_lane):
    """sort_by_layers for device arrays of cfg's regular layout (nevts events of nb blocks):
    returns (trk, hits, nlay_lane, perm) as new device tensors, each event's tracks ordered by
    layer count, longest first; perm[i] is the old index of new track i."""
    import torch
    bs, nl, nblocks = cfg.bsize, cfg.nlayer, cfg.nblocks
    n = nblocks * bs
    ev = torch.arange(n, device=nlay_lane.device, dtype=torch.int64) // (cfg.nb * bs)
    key = ev * (nl + 2) + (nl - nlay_lane.to(torch.int64).clamp(0, nl))
    perm = torch.argsort(key, stable=True)
    t = trk.view(nblocks, 28, bs).permute(0, 2, 1).reshape(n, 28)[perm]
    t = t.reshape(nblocks, bs, 28).permute(0, 2, 1).contiguous().view(-1)
    h = hits.view(nblocks, nl, 9, bs).permute(0, 3, 1, 2).reshape(n, nl, 9)[perm]
    h = h.reshape(nblocks, bs, nl, 9).permute(0, 2, 3, 1).contiguous().view(-1)
    return t, h, nlay_lane[perm].contiguous(), perm


def permute_tracks_device(arr, perm, bsize: int, words: int, nlayer: int = 1):
    """permute_tracks for a flat device tensor (torch): track i of the result is track perm[i]
    of arr. With perm = inverse_device(p) it undoes the ordering p of sort_by_layers_device,
    e.g. to return trk_out, grad_trk_in (words 28) or grad_hits (words 9, nlayer) of an ordered
    run in the caller's track order."""
    n = perm.numel()
    nblocks = n // bsize
    t = arr.view(nblocks, nlayer, words, bsize).permute(0, 3, 1, 2).reshape(n, nlayer, words)[perm]
    return t.reshape(nblocks, bsize, nlayer, words).permute(0, 2, 3, 1).contiguous().view(-1)


def inverse_device(perm):
    """Inverse of a device permutation (torch): inv[perm[i]] = i."""
    import torch
    inv = torch.empty_like(perm)
    inv[perm] = torch.arange(perm.numel(), device=perm.device, dtype=perm.dtype)
    return inv


def inverse(perm: np.ndarray) -> np.ndarray:
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    return inv


def plan(event_block_offset: np.ndarray, blocks_per_item: int) -> np.ndarray:
    """Work items (event, nblk, block0) as a structured numpy array."""
    off = np.ascontiguousarray(event_block_offset, np.int64)
    nevts = len(off) - 1
    n = lib().p2r_queue_plan(off.ctypes.data, nevts, blocks_per_item, None, 0)
    if n < 0:
        raise P2RError(-n, lib().p2r_last_error_string().decode())
    items = (CQueueItem * max(n, 1))()
    m = lib().p2r_queue_plan(off.ctypes.data, nevts, blocks_per_item, ctypes.addressof(items), n)
    if m < 0:
        raise P2RError(-m, lib().p2r_last_error_string().decode())
    dt = np.dtype([("event", np.int32), ("nblk", np.int32), ("block0", np.int64)])
    return np.frombuffer(bytes(items), dtype=dt, count=n).copy()


class Queue:
    """Device description of an uneven batch for p2r_run_queue / p2r_queue_graph_create."""

    def __init__(self, w: dict, blocks_per_item: int = 4, block_threads: int = 0, stages: int = 0,
                 ctas_per_sm: int = 0, flags: int = 0, device="cuda"):
        import torch
        self.torch = torch
        self.w = w
        self.dev = torch.device(device)
        # the kernel reads int64 offsets and int32 layer counts and trusts the block ranges
        off = np.ascontiguousarray(w["event_block_offset"], np.int64)
        nlay = np.ascontiguousarray(w["nlay_lane"], np.int32).reshape(-1)
        if off.ndim != 1 or len(off) < 1 or off[0] != 0 or off[-1] != w["nblocks"] or (np.diff(off) < 0).any():
            raise ValueError("event_block_offset must rise from 0 to nblocks")
        if nlay.size != w["nblocks"] * w["bsize"]:
            raise ValueError(f"nlay_lane has {nlay.size} entries, nblocks * bsize = {w['nblocks'] * w['bsize']}")
        items = plan(off, blocks_per_item)
        self.n_items = len(items)
        self.d_off = torch.from_numpy(off).to(self.dev)
        self.d_items = torch.from_numpy(items.view(np.uint8).copy()).to(self.dev)
        self.d_nlay = torch.from_numpy(nlay).to(self.dev)
        self.nevts = len(off) - 1
        if "ntrk_event" in w and len(w["ntrk_event"]) != self.nevts:
            raise ValueError("ntrk_event and event_block_offset disagree on the event count")
        self.q = CQueue(w["bsize"], w["nlayer"], self.nevts, w["nblocks"], w["bz"], flags, block_threads, stages,
                        ctas_per_sm, self.d_off.data_ptr(), self.d_items.data_ptr(), self.n_items,
                        self.d_nlay.data_ptr())
        ws = lib().p2r_queue_workspace_size(ctypes.byref(self.q))
        self.ws = torch.empty(max(int(ws), 256), dtype=torch.uint8, device=self.dev)
        self.done_ns = torch.zeros(self.nevts, dtype=torch.int64, device=self.dev)
        self.start_ns = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self.graph = None

    def _arrays(self, trk_in, hits, trk_out, chi2):
        """The four array pointers, each checked for type and size against the workload."""
        w = self.w
        ntrk = w["nblocks"] * w["bsize"]
        return (_arg(trk_in, "float32", ntrk * TRK_WORDS, "trk_in"),
                _arg(hits, "float32", ntrk * w["nlayer"] * HIT_WORDS, "hits"),
                _arg(trk_out, "float32", ntrk * TRK_WORDS, "trk_out"), _arg(chi2, "float32", ntrk, "chi2"))

    def run(self, trk_in, hits, trk_out, chi2=None, stream=None) -> None:
        self._last_ws = self.ws
        check(lib().p2r_run_queue(ctypes.byref(self.q), *self._arrays(trk_in, hits, trk_out, chi2),
                                  _ptr(self.done_ns), _ptr(self.start_ns), _ptr(self.ws), self.ws.numel(),
                                  _stream(stream)))

    def capture(self, trk_in, hits, trk_out, chi2=None) -> None:
        """Captures the launch sequence into a CUDA graph (pointers are baked in)."""
        self.release()
        self._last_ws = self.ws
        g = ctypes.c_void_p()
        check(lib().p2r_queue_graph_create(ctypes.byref(self.q), *self._arrays(trk_in, hits, trk_out, chi2),
                                           _ptr(self.done_ns), _ptr(self.start_ns), _ptr(self.ws), self.ws.numel(),
                                           ctypes.byref(g)))
        self.graph = g

    def replay(self, stream=None) -> None:
        if self.graph is None:
            raise P2RError(_lib.P2R_ERR_INVALID, "no graph captured")
        check(lib().p2r_graph_launch(self.graph, _stream(stream)))

    def release(self) -> None:
        if self.graph is not None:
            lib().p2r_graph_destroy(self.graph)
            self.graph = None

    # ------------------------------------------------------------ forward + adjoint
    def adjoint_workspace_size(self) -> int:
        n = lib().p2r_queue_adjoint_workspace_size(ctypes.byref(self.q))
        if n == 0:
            raise P2RError(_lib.P2R_ERR_INVALID, lib().p2r_last_error_string().decode())
        return int(n)

    def _adjoint_args(self, trk_in, hits, dr, grad_trk_out, grad_chi2, o: dict):
        """The argument list of p2r_run_queue_adjoint / p2r_queue_adjoint_graph_create after
        the queue, each array checked for type and size against the workload."""
        torch = self.torch
        w = self.w
        ntrk = w["nblocks"] * w["bsize"]
        nt, nh, nl = ntrk * TRK_WORDS, ntrk * w["nlayer"] * HIT_WORDS, w["nlayer"]
        dev = trk_in.device
        f32 = dict(dtype=torch.float32, device=dev)
        f64 = dict(dtype=torch.float64, device=dev)
        o.setdefault("trk_out", torch.empty_like(trk_in))
        o.setdefault("chi2", torch.empty(ntrk, **f32))
        o.setdefault("grad_trk_in", torch.empty_like(trk_in))
        o.setdefault("grad_hits", torch.empty_like(hits))
        o.setdefault("grad_dr", torch.empty(nl, **f64))
        o.setdefault("grad_bz", torch.empty(1, **f64))
        o.setdefault("grad_dr_event", torch.empty(self.nevts, nl, **f64))
        o.setdefault("grad_bz_event", torch.empty(self.nevts, **f64))
        need = self.adjoint_workspace_size()
        ws = o.get("workspace")
        if ws is None or ws.numel() < need:
            ws = torch.empty(need, dtype=torch.uint8, device=dev)
            o["workspace"] = ws
        return (_arg(trk_in, "float32", nt, "trk_in"), _arg(hits, "float32", nh, "hits"),
                _arg(dr, "float32", nl, "dr"), _arg(o["trk_out"], "float32", nt, "trk_out"),
                _arg(o["chi2"], "float32", ntrk, "chi2"), _arg(grad_trk_out, "float32", nt, "grad_trk_out"),
                _arg(grad_chi2, "float32", ntrk, "grad_chi2"), _arg(o["grad_trk_in"], "float32", nt, "grad_trk_in"),
                _arg(o["grad_hits"], "float32", nh, "grad_hits"), _arg(o["grad_dr"], "float64", nl, "grad_dr"),
                _arg(o["grad_bz"], "float64", 1, "grad_bz"),
                _arg(o["grad_dr_event"], "float64", self.nevts * nl, "grad_dr_event"),
                _arg(o["grad_bz_event"], "float64", self.nevts, "grad_bz_event"), _ptr(ws), ws.numel())

    def run_adjoint(self, trk_in, hits, dr=None, grad_trk_out=None, grad_chi2=None, out=None, stream=None) -> dict:
        """Forward + adjoint of the batch in one persistent launch (p2r_run_queue_adjoint):
        returns trk_out, chi2, grad_trk_in, grad_hits, grad_dr, grad_bz, grad_dr_event,
        grad_bz_event (an entry of `out` set to None skips that output) and the workspace."""
        o = out if out is not None else {}
        args = self._adjoint_args(trk_in, hits, dr, grad_trk_out, grad_chi2, o)
        self._last_ws = o["workspace"]
        check(lib().p2r_run_queue_adjoint(ctypes.byref(self.q), *args, _stream(stream)))
        return o

    def capture_adjoint(self, trk_in, hits, dr=None, grad_trk_out=None, grad_chi2=None, out=None) -> dict:
        """Captures the forward + adjoint launch sequence into a CUDA graph (replay()); returns
        the output dict the replays write."""
        self.release()
        o = out if out is not None else {}
        args = self._adjoint_args(trk_in, hits, dr, grad_trk_out, grad_chi2, o)
        self._last_ws = o["workspace"]
        g = ctypes.c_void_p()
        check(lib().p2r_queue_adjoint_graph_create(ctypes.byref(self.q), *args, ctypes.byref(g)))
        self.graph = g
        self.adjoint_out = o
        return o

    def error_bits(self, stream=None) -> int:
        """Synchronises `stream` and returns the device-side check bits of the last launch
        (0: every work item and event offset was in range; see p2r_queue_error)."""
        bits = ctypes.c_uint32(0)
        ws = getattr(self, "_last_ws", None)
        rc = lib().p2r_queue_error(_ptr(self.ws if ws is None else ws), ctypes.byref(bits), _stream(stream))
        if rc not in (_lib.P2R_OK, _lib.P2R_ERR_QUEUE):
            check(rc)
        return int(bits.value)

    def event_latency_ns(self) -> np.ndarray:
        """Per-event completion time relative to the earliest CTA start of the last launch."""
        return (self.done_ns - self.start_ns).cpu().numpy()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass
