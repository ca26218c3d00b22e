"""Autotuner for the delay-and-sum schedule (kernel variant, voxel tile, window, event chunk).

    cfg = autotune(x, srcpos, dstpos, offsets, weights)       # times candidates on these inputs
    with schedule(cfg): ffdas_b200.das(...)                    # or handle.set_config(cfg)

Candidates are timed with CUDA events on the caller's own inputs (the
geometry decides which voxel tile keeps each tile's sample windows narrow).
The winner is cached per problem signature in a JSON file
($FFDAS_B200_TUNE_CACHE, default ~/.cache/ffdas_b200/tune.json) and reused.
"""
from __future__ import annotations

import contextlib
import json
import os
import threading
from pathlib import Path

import numpy as np
import torch

from .library import get_library_handle

_lock = threading.Lock()


def cache_path() -> Path:
    p = os.environ.get("FFDAS_B200_TUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "ffdas_b200" / "tune.json"


def signature(x, dstpos, offsets, sparse_indices=None, use_fp16=False, use_bf16=False) -> str:
    dev = torch.cuda.get_device_name(x.device)
    comp = "f16" if use_fp16 else ("bf16" if use_bf16 else "default")
    sp = "sparse" if sparse_indices is not None else "dense"
    return f"{dev}|{tuple(x.shape)}|{x.dtype}|{tuple(dstpos.shape)}|{tuple(offsets.shape)}|{sp}|{comp}"


def _grid_dims(dstpos) -> tuple[int, int]:
    dims = [int(d) for d in dstpos.shape[:-1] if d != 1]
    d0 = dims[-1] if dims else 1
    d1 = dims[-2] if len(dims) >= 2 else 1
    return d0, d1


# Largest problem (voxels x channels x events x items) for which the direct
# kernel is among the candidates: twice the planner's own threshold.
DIRECT_UNITS_MAX = 2 << 25


def candidates(x, dstpos, offsets, sparse_indices=None) -> list[dict]:
    d0, d1 = _grid_dims(dstpos)
    B = x.shape[0] if x.ndim == 4 else 1
    real = not x.is_complex() and x.dtype != torch.float64
    tiles = []
    for t0 in (256, 128, 64, 32, 16, 8):
        t1 = 256 // t0
        if t0 <= max(d0, 8) * 2 and (t1 == 1 or t1 <= max(d1, 1) * 2):
            tiles.append((t0, t1))
    out = []
    for t0, t1 in tiles:
        for bt in sorted({1, min(4, B), min(8, B)} if real else {1}):
            if bt & (bt - 1):
                continue
            out.append(dict(variant=1, tile_x=t0, tile_y=t1, batch_tile=bt))
            if real and sparse_indices is not None and bt <= 4:
                # event chunks of 8 and 4: fewer registers, more resident warps for latency-bound lists
                for ec in (8, 4):
                    out.append(dict(variant=1, tile_x=t0, tile_y=t1, batch_tile=bt, event_chunk=ec))
                    for mb in (8, 16, 32):   # channel-slice targets around the default of 16 CTAs per SM
                        out.append(dict(variant=1, tile_x=t0, tile_y=t1, batch_tile=bt, event_chunk=ec,
                                        min_blocks=mb))
        if real and sparse_indices is None:
            n_ev = offsets.shape[0]
            chunks = sorted({min(c, max(n_ev, 1)) for c in (4, 8, 16)})
            for wb in (32, 64):
                for ec in chunks:
                    for ce in (1, 2):   # TMA tile loads / per-thread cp.async copies
                        out.append(dict(variant=2, tile_x=t0, tile_y=t1, window=wb, event_chunk=ec, copy_engine=ce,
                                        batch_tile=1))
                # batch tiles: BT items per CTA share each window's delays
                for bt in (2, 4, 8):
                    if bt > B:
                        continue
                    for ec in sorted({4, 8} if bt <= 4 else {4}):
                        out.append(dict(variant=2, tile_x=t0, tile_y=t1, window=wb, event_chunk=ec, copy_engine=1,
                                        batch_tile=bt))
    if real and sparse_indices is None and x.dtype != torch.float64:
        # direct kernel (one launch, no pair workspace) for small problems
        V = int(np.prod(dstpos.shape[:-1]))
        C, S = x.shape[-3], offsets.shape[0]
        if V * C * S * B <= DIRECT_UNITS_MAX:
            for bt in sorted({1, min(2, B), min(4, B)}):
                if bt & (bt - 1) == 0:
                    out.append(dict(variant=5, batch_tile=bt))   # lanes per voxel from the occupancy
                    for lanes in (2, 4, 8, 16, 32):
                        if lanes <= C:
                            out.append(dict(variant=5, batch_tile=bt, tile_x=lanes))
    if real and sparse_indices is not None and x.dtype != torch.float64:
        # das_sparse as one persistent launch over bucketed lists (256-voxel tiles)
        for t0, t1 in tiles:
            for wb in (32, 64):
                for ec in (4, 8):
                    for mb in (4, 8, 16):   # channel slicing: about mb work items per SM
                        out.append(dict(variant=6, tile_x=t0, tile_y=t1, window=wb, event_chunk=ec, min_blocks=mb))
        # das_sparse on the staged kernel: 512-voxel tiles, passes over x's events
        S = x.shape[-2]
        for t0 in (128, 64, 32, 16, 8):
            t1 = 512 // t0
            if t0 <= max(d0, 8) * 2 and t1 <= max(d1, 1) * 2:
                for wb in (32, 64):
                    for ec in sorted({min(c, max(S, 1)) for c in (4, 8)}):
                        out.append(dict(variant=2, tile_x=t0, tile_y=t1, window=wb, event_chunk=ec, copy_engine=1,
                                        batch_tile=1))
    if real and sparse_indices is None:
        # staged kernel with 512-voxel tiles (two voxels per thread)
        n_ev = offsets.shape[0]
        chunks = sorted({min(c, max(n_ev, 1)) for c in (4, 8)})
        for t0 in (128, 64, 32, 16, 8):
            t1 = 512 // t0
            if t0 <= max(d0, 8) * 2 and t1 <= max(d1, 1) * 2:
                for wb in (32, 64):
                    for ec in chunks:
                        out.append(dict(variant=2, tile_x=t0, tile_y=t1, window=wb, event_chunk=ec, copy_engine=1,
                                        batch_tile=1))
    return out


@contextlib.contextmanager
def schedule(cfg: dict | None, device=None):
    """Apply a schedule to the device's library handle for the duration of a block."""
    h = get_library_handle(device)
    prev = h.get_config().as_dict()
    h.set_config(cfg)
    try:
        yield
    finally:
        h.set_config(prev if any(prev.values()) else None)


_MIN_TIMED_MS = 2.0      # a timed run of a small call repeats it until about this much device time
_MAX_REPS = 256
_GRAPH_BELOW_MS = 0.1    # calls shorter than this are timed as CUDA graph replays


def _time_graph(fn, n: int) -> float:
    """Per-call milliseconds of `n` calls captured into one CUDA graph (the
    device time of the call itself: no host launch overhead between calls)."""
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        fn()
    s.synchronize()
    with torch.cuda.graph(g, stream=s):
        for _ in range(n):
            fn()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)

    def run():
        with torch.cuda.stream(s):
            a.record(s)
            g.replay()
            b.record(s)
        b.synchronize()
        return a.elapsed_time(b) / n

    run()
    best = min(run(), run(), run())
    del g
    return best


def _time(fn, reps: int) -> float:
    """Per-call milliseconds: the best of three timed runs of at least `reps` calls.

    Calls of a few microseconds are repeated until a run holds about 2 ms of
    device time, so that launch jitter does not decide between schedules whose
    difference is a few percent.  Calls under 0.1 ms are timed as replays of a
    CUDA graph holding the repeated calls: issued one by one from Python they
    are bound by the host, and every schedule would time the same; under a
    graph (the way `DASRunner` runs them) the device time decides."""
    fn()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)

    def run(n):
        a.record()
        for _ in range(n):
            fn()
        b.record()
        b.synchronize()
        return a.elapsed_time(b) / n

    first = run(reps)
    n = reps
    if first * reps < _MIN_TIMED_MS:
        n = min(_MAX_REPS, max(reps, int(_MIN_TIMED_MS / max(first, 1e-3))))
    if first < _GRAPH_BELOW_MS:
        try:
            return _time_graph(fn, n)
        except RuntimeError:
            torch.cuda.synchronize()
    return min(first if n == reps else run(n), run(n), run(n))


def autotune(x, srcpos, dstpos, offsets, weights, sparse_indices=None, *, use_fp16=False, use_bf16=False,
             reps: int = 3, use_cache: bool = True, max_candidates: int | None = None) -> dict:
    """Time the candidate schedules on these inputs; return {'config', 'ms', 'table'}."""
    from .das import das, das_sparse
    key = signature(x, dstpos, offsets, sparse_indices, use_fp16, use_bf16)
    path = cache_path()
    if use_cache and path.exists():
        try:
            cached = json.loads(path.read_text()).get(key)
            if cached:
                return cached
        except Exception:
            pass
    out = torch.empty((x.shape[0], *dstpos.shape[:-1]) if x.ndim == 4 else tuple(dstpos.shape[:-1]),
                      dtype=torch.float64 if x.dtype in (torch.float64, torch.complex128) else
                      (torch.complex64 if x.is_complex() else torch.float32), device=x.device)

    def call():
        if sparse_indices is None:
            das(x, srcpos, dstpos, offsets, weights, use_fp16=use_fp16, use_bf16=use_bf16, out=out)
        else:
            das_sparse(x, srcpos, dstpos, offsets, weights, sparse_indices, use_fp16=use_fp16, use_bf16=use_bf16,
                       out=out)

    table = []
    cands = candidates(x, dstpos, offsets, sparse_indices)
    if max_candidates:
        cands = cands[:max_candidates]
    for cfg in cands:
        with schedule(cfg, x.device):
            try:
                ms = _time(call, reps)
            except RuntimeError:
                continue
        table.append((ms, cfg))
    table.sort(key=lambda t: t[0])
    best = {"config": table[0][1], "ms": table[0][0], "table": [[m, c] for m, c in table[:8]]}
    if use_cache:
        with _lock:
            path.parent.mkdir(parents=True, exist_ok=True)
            data = {}
            if path.exists():
                try:
                    data = json.loads(path.read_text())
                except Exception:
                    data = {}
            data[key] = best
            tmp = path.with_suffix(".tmp")
            tmp.write_text(json.dumps(data, indent=1))
            os.replace(tmp, path)
    return best
