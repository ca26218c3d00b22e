"""Run one delay-and-sum workload under a fixed schedule, for profilers.

    python profile_call.py ensemble --frames 50 --calls 4 \\
        --schedule '{"variant": 2, "tile_x": 32, "tile_y": 8, "window": 64, "batch_tile": 8}'

Builds the named synthetic workload (ffdas_b200.workloads.CONFIGS), applies the
schedule to the device's library handle, calls das / das_sparse `--calls`
times (the first calls warm the kernel attributes and the memory pool), and
prints the last call's kernel info.  `--backward` runs the forward with
autograd and its backward (output gradient of ones): ffdas_das_backward for
the gradient of x (and, for das_sparse workloads, of the delays and
weights).

    python profile_call.py rank_filter --calls 3

runs truncate_rank(x, 5) on the seeded 200-frame 400x256 FP32 slow-time
ensemble (workloads.slow_time_ensemble) instead, and

    python profile_call.py sparse_select --calls 3

runs sparse_select(w, 32, offsets=o) on 64 events x 400x256 pixels (a seeded
0/1 beam mask plus 1e-3 jitter, as `bench.py` configs.sparse_select).
"""
from __future__ import annotations

import argparse
import json

import torch

from ffdas_b200 import workloads as W
from ffdas_b200.das import das, das_sparse
from ffdas_b200.library import get_library_handle


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=sorted(W.CONFIGS) + ["rank_filter", "sparse_select"])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--frames", type=int, default=None, help="ensemble: number of frames")
    ap.add_argument("--calls", type=int, default=4)
    ap.add_argument("--schedule", default=None, help="JSON ffdas_das_config_t fields")
    ap.add_argument("--backward", action="store_true")
    args = ap.parse_args()
    dev = torch.device("cuda", torch.cuda.current_device())
    if args.workload == "rank_filter":
        from ffdas_b200.truncate_rank import truncate_rank
        x = W.slow_time_ensemble(args.frames or 200, (400, 256), torch.float32, dev)
        for _ in range(args.calls):
            y = truncate_rank(x, 5)
        torch.cuda.synchronize()
        print(json.dumps({"rank_filter": list(x.shape), "max_abs_out": float(y.abs().max())}))
        return 0
    if args.workload == "sparse_select":
        import ffdas_b200
        g = torch.Generator().manual_seed(41)
        shape = (64, 400, 256)
        w = ((torch.rand(shape, generator=g) < 0.3).float() + torch.rand(shape, generator=g) * 1e-3).to(dev)
        o = (torch.rand(shape, generator=g) * 1000).to(dev)
        for _ in range(args.calls):
            idx, _, _ = ffdas_b200.sparse_select(w, 32, offsets=o)
        torch.cuda.synchronize()
        print(json.dumps({"sparse_select": list(w.shape), "first_rank_events": int(idx[0].max())}))
        return 0
    kw = {"frames": args.frames} if args.frames is not None else {}
    wl = W.CONFIGS[args.workload](device=dev, scale=args.scale, **kw)
    h = get_library_handle(dev)
    h.set_config(json.loads(args.schedule) if args.schedule else None)
    geo = (wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
    x = wl["x"]
    for _ in range(args.calls):
        if args.backward:
            xg = x.float().requires_grad_(True)
            if "sparse_indices" in wl:   # adjoint of das_sparse: grads of x, delays and weights
                og = wl["offsets"].clone().requires_grad_(True)
                wg = wl["weights"].clone().requires_grad_(True)
                out = das_sparse(xg, wl["srcpos"], wl["dstpos"], og, wg, wl["sparse_indices"])
            else:
                out = das(xg, *geo)
            out.backward(torch.ones_like(out))
        elif "sparse_indices" in wl:
            das_sparse(x, *geo, wl["sparse_indices"])
        else:
            das(x, *geo)
    torch.cuda.synchronize()
    print(json.dumps(h.last_kernel_info()))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
