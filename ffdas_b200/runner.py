"""Graph-captured delay-and-sum for repeated calls with fixed geometry.

    run = DASRunner(x_example, srcpos, dstpos, offsets, weights)          # tunes and captures once
    img = run(x_frame)                                                     # copy-in + graph replay

The runner owns static input and output buffers.  On construction it picks
the schedule with the autotuner (optional), runs one warm-up call, and
captures one das / das_sparse call -- the ingest pass and the delay-and-sum
kernel, with their stream-ordered workspace allocation -- into a CUDA graph
on a private stream.  Each call copies the new channel data into the static
input (or takes it in place with `run.replay()` after writing `run.x`),
replays the graph, and returns the static output (overwritten by the next
call unless `clone=True`).  Geometry tensors must not change after capture
(their device addresses are baked into the graph).
"""
from __future__ import annotations

import torch

from .das import das, das_sparse
from .library import get_library_handle
from .tune import autotune


class DASRunner:
    def __init__(self, x, srcpos, dstpos, offsets, weights, sparse_indices=None, *, srcdir=None,
                 wavenum: float = 0.0, use_fp16: bool = False, use_bf16: bool = False, tune: bool = True,
                 config: dict | None = None):
        if not x.is_cuda:
            raise ValueError("DASRunner needs CUDA tensors")
        self.device = x.device
        self.x = torch.empty_like(x, memory_format=torch.contiguous_format)
        self.x.copy_(x)
        self._geom = dict(srcpos=srcpos.contiguous(), dstpos=dstpos.contiguous(), offsets=offsets.contiguous(),
                          weights=weights.contiguous())
        self._idx = sparse_indices.contiguous() if sparse_indices is not None else None
        self._kw = dict(srcdir=srcdir, wavenum=wavenum, use_fp16=use_fp16, use_bf16=use_bf16)
        if config is None and tune:
            config = autotune(self.x, *self._geom.values(), sparse_indices=self._idx, use_fp16=use_fp16,
                              use_bf16=use_bf16)["config"]
        self.config = config
        self.handle = get_library_handle(self.device)
        self.out = None
        self.stream = torch.cuda.Stream(self.device)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.stream(self.stream):
            self._call()                        # warm-up: first-use attributes, pool growth
        self.stream.synchronize()
        with torch.cuda.graph(self.graph, stream=self.stream):
            self._call()

    def _call(self):
        self.handle.set_config(self.config)
        g = self._geom
        with torch.no_grad():
            if self._idx is None:
                self.out = das(self.x, g["srcpos"], g["dstpos"], g["offsets"], g["weights"], out=self.out,
                               **self._kw)
            else:
                self.out = das_sparse(self.x, g["srcpos"], g["dstpos"], g["offsets"], g["weights"], self._idx,
                                      out=self.out, **self._kw)

    def replay(self) -> torch.Tensor:
        """Re-run the captured call on the current contents of `self.x`."""
        self.graph.replay()
        return self.out

    def __call__(self, x=None, clone: bool = False) -> torch.Tensor:
        if x is not None:
            self.x.copy_(x, non_blocking=True)
        out = self.replay()
        return out.clone() if clone else out
