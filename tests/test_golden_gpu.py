"""This library against the reference's own outputs (tests/golden/ref_*.npz).

Each fixture holds seeded inputs and the output of the reference library run
on a B200 (tests/golden/make_golden.py).  Here the same inputs go through
ffdas_das / ffdas_das_sparse of this library (C-ABI, beta and the initial
output included) and the result is compared with the reference's:

* FP32 and FP64 cases, complex64 with phase rotation, directivity and
  beta != 0 included: 1e-5 relative L2 (the parity bar); phases are kept
  below ~40 rad, so both libraries' __sincosf agree to a few 1e-7;
* 16-bit cases (float16, complex32): the reference interpolates in half
  precision (math/vector.cuh:42), this library in FP32, so the two differ by
  the reference's own rounding; this library must be at least as close to the
  FP64 oracle as the reference is, and within the fixture's stated tolerance
  of the reference;
* the reference's ALG2 cases (64 frames, every tap inside the record): ALG2
  quantises the fraction to FP16, so this library is held to the fixture's
  tolerance against it and, like above, must be closer to the oracle.
"""
import ctypes
from pathlib import Path

import numpy as np
import pytest
import torch

import ffdas_b200
from ffdas_b200 import _lib
from ffdas_b200._lib import DataType
from oracle import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
GOLDEN = Path(__file__).resolve().parent / "golden"

_TORCH = {"torch.float32": torch.float32, "torch.float16": torch.float16, "torch.float64": torch.float64,
          "torch.complex64": torch.complex64, "torch.complex32": torch.complex32}
_CODE = {torch.float32: DataType.R_32F, torch.float16: DataType.R_16F, torch.float64: DataType.R_64F,
         torch.complex64: DataType.C_32F, torch.complex32: DataType.C_16F}
_OUT = {torch.float32: torch.float32, torch.float16: torch.float32, torch.float64: torch.float64,
        torch.complex64: torch.complex64, torch.complex32: torch.complex64}


def _run_ours(z):
    xdt = _TORCH[str(z["x_dtype"])]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    x = t(z["x"]).to(xdt).contiguous()
    src, dst = t(z["srcpos"]).float(), t(z["dstpos"]).float()
    offs, w = t(z["offsets"]).float(), t(z["weights"]).float()
    srcdir = t(z["srcdir"]).float() if "srcdir" in z.files else None
    wavenum = float(z["wavenum"]) if "wavenum" in z.files else 0.0
    odt = _OUT[xdt]
    spatial = tuple(dst.shape[:-1])
    out = torch.zeros((x.shape[0], *spatial), dtype=odt, device=DEV)
    beta_v = complex(z["beta"]) if "beta" in z.files else 0.0
    if "out_init" in z.files:
        out.copy_(t(z["out_init"]).to(odt).reshape(out.shape))
    if odt in (torch.float64, torch.complex128):
        beta = (ctypes.c_double * 2)(beta_v.real, beta_v.imag)
    else:
        beta = (ctypes.c_float * 2)(beta_v.real, beta_v.imag)
    xd = _lib.TensorDesc(list(x.shape), list(x.stride()), _CODE[xdt])
    od = _lib.TensorDesc(list(out.shape), None, _CODE[odt])
    h = ffdas_b200.get_library_handle(DEV)
    h.set_stream(torch.cuda.current_stream().cuda_stream)
    L = _lib.load()
    sdp = None if srcdir is None else srcdir.data_ptr()
    if "sparse_indices" in z.files:
        idx = t(z["sparse_indices"]).int()
        rc = L.ffdas_das_sparse(h.h, src.data_ptr(), sdp, wavenum, xd.desc, x.data_ptr(), dst.data_ptr(),
                                offs.data_ptr(), w.data_ptr(), int(idx.shape[0]), idx.data_ptr(),
                                ctypes.cast(beta, ctypes.c_void_p), od.desc, out.data_ptr(), 0, 0)
    else:
        rc = L.ffdas_das(h.h, src.data_ptr(), sdp, wavenum, xd.desc, x.data_ptr(), dst.data_ptr(),
                         offs.data_ptr(), w.data_ptr(), ctypes.cast(beta, ctypes.c_void_p), od.desc,
                         out.data_ptr(), 0, 0)
    _lib.check(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy(), xdt


def _oracle(z):
    kw = {}
    for k in ("srcdir", "sparse_indices"):
        if k in z.files:
            kw[k] = z[k]
    if "beta" in z.files:
        kw["beta"] = complex(z["beta"])
        kw["out"] = z["out_init"]
    return oracle.das_f64(z["x"], z["srcpos"], z["dstpos"], z["offsets"], z["weights"],
                          wavenum=float(z["wavenum"]) if "wavenum" in z.files else 0.0, **kw)


@pytest.mark.parametrize("path", sorted(GOLDEN.glob("ref_*.npz")), ids=lambda p: p.stem)
def test_matches_reference_output(path):
    z = np.load(path, allow_pickle=False)
    if "q1" in z.files and bool(z["q1"]):
        pytest.skip("reproduces the reference's 3-D event-0 indexing, which this library does not")
    ours, xdt = _run_ours(z)
    ref = z["out"]
    alg2 = int(z["alg"]) == 2
    if xdt in (torch.float32, torch.float64, torch.complex64) and not alg2:
        assert oracle.rel_l2(ours, ref) < 1e-5
        return
    exact = _oracle(z)
    e_ours, e_ref = oracle.rel_l2(ours, exact), oracle.rel_l2(ref, exact)
    assert e_ours <= e_ref * 1.01 + 1e-6, (e_ours, e_ref)
    assert oracle.rel_l2(ours, ref) < float(z["tol"])
