"""Generate golden vectors from the reference library itself.

    python tests/golden/make_golden.py [--out tests/golden]

Needs a CUDA GPU and oracle/_ref/libffdas_ref.so (the reference's das path
compiled from its sources by `make -C oracle ref`).  Each case is a small,
seeded input; the reference's output is stored next to the inputs, together
with the tolerance at which the FP64 oracle must reproduce it
(tests/test_oracle.py::test_oracle_matches_reference_outputs).  Every call goes
through oracle/reference.py, which guards the reference's unmasked sample
loads with padding computed from the geometry.
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np
import torch

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from ffdas_b200 import workloads as W  # noqa: E402
from oracle import reference  # noqa: E402


def _case_random(seed, B=3, C=6, S=4, N=160, nz=9, nx=11, complex_=False, dtype=torch.float32):
    g = torch.Generator().manual_seed(seed)
    x = torch.randn((B, C, S, N), generator=g)
    if complex_:
        x = torch.complex(x, torch.randn((B, C, S, N), generator=g))
    x = x.to(dtype)
    src = torch.zeros((C, 3))
    src[:, 0] = torch.linspace(-5, 5, C)
    zz, xx = torch.meshgrid(torch.linspace(25, 60, nz), torch.linspace(-6, 6, nx), indexing="ij")
    dst = torch.stack([xx, torch.zeros_like(xx), zz], -1)
    offs = torch.rand((S, nz, nx), generator=g) * 70 - 5
    w = torch.rand((S, nz, nx), generator=g) + 0.1
    return dict(x=x, srcpos=src, dstpos=dst, offsets=offs, weights=w)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(ROOT / "tests" / "golden"))
    a = ap.parse_args()
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    dev = torch.device("cuda:0")
    cases = {}
    cases["ref_plane2d_f32"] = (W.plane2d(scale=0.5), dict(alg=1), 2e-5)
    cases["ref_diverging3d_f32"] = (W.diverging3d(scale=0.125), dict(alg=1), 2e-5)
    cases["ref_random_batched_f32"] = (_case_random(11), dict(alg=1), 2e-5)
    sp = W.sparse_focus(scale=0.1)
    cases["ref_sparse_focus_f32"] = (sp, dict(alg=1, sparse=True), 2e-5)
    cases["ref_random_f16_alg1"] = (_case_random(12, dtype=torch.float16), dict(alg=1), 3e-3)
    cases["ref_random_f64"] = (_case_random(13, dtype=torch.float64), dict(alg=1), 2e-5)
    for name, (wl, opt, tol) in cases.items():
        x = wl["x"]
        if x.ndim == 3:
            x = x[None]
        xd = x.to(dev).contiguous()
        kw = {}
        if opt.get("sparse"):
            kw["sparse_indices"] = wl["sparse_indices"]
        res = reference.das(xd, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"], alg=opt["alg"], **kw)
        xs = x.cpu()
        if xs.dtype == torch.float16:
            xs = xs.float()
        rec = dict(x=xs.numpy(), srcpos=wl["srcpos"].cpu().numpy(), dstpos=wl["dstpos"].cpu().numpy(),
                   offsets=wl["offsets"].cpu().numpy(), weights=wl["weights"].cpu().numpy(),
                   out=res.cpu().numpy(), tol=np.float64(tol), alg=np.int32(opt["alg"]),
                   x_dtype=np.array(str(x.dtype)))
        if "sparse_indices" in kw:
            rec["sparse_indices"] = kw["sparse_indices"].cpu().numpy()
        np.savez_compressed(out / f"{name}.npz", **rec)
        print(name, tuple(res.shape), f"{(out / f'{name}.npz').stat().st_size / 1e3:.0f} kB")
    return 0


if __name__ == "__main__":
    sys.exit(main())
