"""Generate golden vectors from the reference library itself.

    python tests/golden/make_golden.py [--out tests/golden] [--only name,name]

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

import importlib.util  # noqa: E402

# the seeded generators, loaded from their file so that this script does not
# load the library under test (it only runs the reference)
_spec = importlib.util.spec_from_file_location("_ffdas_workloads", ROOT / "ffdas_b200" / "workloads.py")
W = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(W)
from oracle import reference  # noqa: E402


def _case_random(seed, B=3, C=6, S=4, N=160, nz=9, nx=11, complex_=False, dtype=torch.float32):
    g = torch.Generator().manual_seed(seed)
    x = torch.randn((B, C, S, N), generator=g)
    if complex_:
        x = torch.complex(x, torch.randn((B, C, S, N), generator=g))
    x = x.to(dtype) if dtype != torch.complex32 else x.to(torch.complex64).to(dtype)
    src = torch.zeros((C, 3))
    src[:, 0] = torch.linspace(-5, 5, C)
    zz, xx = torch.meshgrid(torch.linspace(25, 60, nz), torch.linspace(-6, 6, nx), indexing="ij")
    dst = torch.stack([xx, torch.zeros_like(xx), zz], -1)
    offs = torch.rand((S, nz, nx), generator=g) * 70 - 5
    w = torch.rand((S, nz, nx), generator=g) + 0.1
    return dict(x=x, srcpos=src, dstpos=dst, offsets=offs, weights=w)


def _case_in_record(seed, B=64, C=4, S=2, N=96, nz=5, nx=6, dtype=torch.float32):
    """Every tap inside the record (0 <= k < N-1): the only geometry on which
    the reference's ALG2, which reads an internal unguarded copy of x, may run."""
    g = torch.Generator().manual_seed(seed)
    x = torch.randn((B, C, S, N), generator=g).to(dtype)
    src = torch.zeros((C, 3))
    src[:, 0] = torch.linspace(-3, 3, C)
    zz, xx = torch.meshgrid(torch.linspace(25, 40, nz), torch.linspace(-4, 4, nx), indexing="ij")
    dst = torch.stack([xx, torch.zeros_like(xx), zz], -1)
    offs = torch.rand((S, nz, nx), generator=g) * 40
    w = torch.rand((S, nz, nx), generator=g) + 0.1
    return dict(x=x, srcpos=src, dstpos=dst, offsets=offs, weights=w)


def _srcdir(C, seed, cos_min):
    """Unit element normals tilted up to ~35 degrees off +z, acceptance cos_min."""
    g = torch.Generator().manual_seed(seed)
    n = torch.cat([torch.rand((C, 2), generator=g) * 1.4 - 0.7, torch.ones((C, 1))], 1)
    n = n / n.norm(dim=1, keepdim=True)
    return torch.cat([n, torch.full((C, 1), cos_min)], 1)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(ROOT / "tests" / "golden"))
    ap.add_argument("--only", default=None, help="comma-separated case names (default: all)")
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
    # complex IQ data with the phase rotation exp(i wavenum tau) (das_alg1_kernels.cuh:81-86);
    # phases stay below ~40 rad, where __sincosf is accurate to a few 1e-6
    cases["ref_random_c32_wavenum"] = (_case_random(14, complex_=True, dtype=torch.complex64),
                                       dict(alg=1, wavenum=0.3), 5e-5)
    # complex32 data: the reference lerps in half precision (quirk Q3)
    cases["ref_random_c16_wavenum"] = (_case_random(15, complex_=True, dtype=torch.complex32),
                                       dict(alg=1, wavenum=0.3), 3e-3)
    # element directivity: a tap counts only when dot(v - c, n) / r > cos_min (:72-76)
    cases["ref_random_srcdir_f32"] = (_case_random(16), dict(alg=1, srcdir=_srcdir(6, 16, 0.93)), 2e-5)
    # beta != 0: out = beta * out + sum (das_device_utils.cuh:33-39)
    cases["ref_random_beta_f32"] = (_case_random(17), dict(alg=1, beta=0.5), 2e-5)
    # all three together on complex data, complex beta
    cases["ref_random_c32_srcdir_beta"] = (_case_random(18, complex_=True, dtype=torch.complex64),
                                           dict(alg=1, wavenum=-0.2, srcdir=_srcdir(6, 18, 0.9),
                                                beta=complex(0.5, -0.25)), 5e-5)
    # ALG2 at its one correct batch size (64 frames, see bench.reference_alg2_ok): it
    # quantises the fraction t to FP16 (das_alg2_kernels.cuh:129), so it matches the
    # oracle only to ~1e-3
    cases["ref_inrecord_alg2_b64_f32"] = (_case_in_record(19), dict(alg=2), 3e-3)
    cases["ref_inrecord_alg2_b64_f16"] = (_case_in_record(20, dtype=torch.float16), dict(alg=2), 5e-3)
    if a.only:
        keep = set(a.only.split(","))
        cases = {k: v for k, v in cases.items() if k in keep}
    for name, (wl, opt, tol) in cases.items():
        x = wl["x"]
        if x.ndim == 3:
            x = x[None]
        xd = x.to(dev).contiguous()
        kw = {}
        if opt.get("sparse"):
            kw["sparse_indices"] = wl["sparse_indices"]
        spatial = tuple(wl["dstpos"].shape[:-1])
        out_init = None
        if opt.get("beta", 0) != 0:
            g = torch.Generator().manual_seed(100)
            out_init = torch.randn((x.shape[0], *spatial), generator=g)
            if x.is_complex():
                out_init = torch.complex(out_init, torch.randn(out_init.shape, generator=g))
            if x.dtype == torch.float64:
                out_init = out_init.double()
            out_init = out_init.to(dev)
        res = reference.das(xd, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"], alg=opt["alg"],
                            srcdir=opt.get("srcdir"), wavenum=opt.get("wavenum", 0.0), beta=opt.get("beta", 0.0),
                            out_init=out_init, **kw)
        xs = x.cpu()
        if xs.dtype == torch.float16:
            xs = xs.float()
        if xs.dtype == torch.complex32:
            xs = xs.to(torch.complex64)
        rec = dict(x=xs.numpy(), srcpos=wl["srcpos"].cpu().numpy(), dstpos=wl["dstpos"].cpu().numpy(),
                   offsets=wl["offsets"].cpu().numpy(), weights=wl["weights"].cpu().numpy(),
                   out=res.cpu().numpy(), tol=np.float64(tol), alg=np.int32(opt["alg"]),
                   x_dtype=np.array(str(x.dtype)))
        if "sparse_indices" in kw:
            rec["sparse_indices"] = kw["sparse_indices"].cpu().numpy()
        if opt.get("srcdir") is not None:
            rec["srcdir"] = opt["srcdir"].numpy()
        if opt.get("wavenum"):
            rec["wavenum"] = np.float64(opt["wavenum"])
        if out_init is not None:
            rec["beta"] = np.complex128(opt["beta"])
            rec["out_init"] = out_init.cpu().numpy()
        np.savez_compressed(out / f"{name}.npz", **rec)
        print(name, tuple(res.shape), f"{(out / f'{name}.npz').stat().st_size / 1e3:.0f} kB")
    return 0


if __name__ == "__main__":
    sys.exit(main())
