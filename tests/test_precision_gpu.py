"""Storage precision on the full 3-D diverging-wave volume against the FP64
CPU oracle.

The volume is the benchmark's (1024 channels, 16 transmits, 4096 samples,
128^3 voxels) with every channel scaled to peak 1; four depth planes spread
over the volume are beamformed and compared, so the oracle finishes in
seconds.

Two questions are asked of each channel-data dtype:

* compute error -- the image against the FP64 oracle run on the SAME channel
  data (for 16-bit data: the 16-bit values, widened exactly).  This is the
  error the kernels add; it is bounded by 2e-4, the FP32 delay rounding the
  reference has too (about 1.0e-4 on these planes; parity with the reference
  itself is held to 1e-5 elsewhere).  The 16-bit pair formats must not add to
  it beyond the 1e-3 target.
* storage error -- the image of the 16-bit data against the FP64 oracle of the
  original FP32 data: quantising the channel data itself.  Measured on B200
  (this library; the FP64 oracle of the quantised data alone in brackets):
  bf16 (8-bit mantissa) 1.04e-3 (1.02e-3) on these four planes and 1.72e-3
  (1.70e-3) on eight; fp16 (11 bits) 1.6e-4 (1.2e-4) and 3.7e-4 (3.2e-4).
  The 1e-3 bar therefore holds for fp16 storage and, for bf16, only against
  the oracle of the same bf16 data (the compute error above): rounding the
  data to 8 bits already costs 1.0-1.7e-3, whatever the kernel does.  The
  bf16 storage check stays at 2e-3 for that reason.
"""
import numpy as np
import pytest
import torch

import ffdas_b200
from ffdas_b200 import workloads as W
from ffdas_b200.tune import schedule
from oracle import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.fixture(scope="module")
def volume():
    wl = W.diverging3d(device=DEV)
    xn = W.normalize_channels(wl["x"])
    sel = torch.tensor(np.linspace(0, wl["dstpos"].shape[0] - 1, 4).astype(np.int64), device=DEV)
    geo = (wl["srcpos"], wl["dstpos"][sel].contiguous(), wl["offsets"][:, sel].contiguous(),
           wl["weights"][:, sel].contiguous())
    geo_np = [t.cpu().numpy() for t in geo]
    refs = {}

    def ref(dtype):
        if dtype not in refs:
            refs[dtype] = oracle.das_f64(xn.to(dtype).double().cpu().numpy(), *geo_np)
        return refs[dtype]
    return xn, geo, ref


CFGS = [None, dict(variant=2, tile_x=16, tile_y=16, window=32), dict(variant=1, tile_x=16, tile_y=16)]


@pytest.mark.parametrize("dtype,tol", [(torch.float32, 2e-4), (torch.float16, 2e-4), (torch.bfloat16, 2e-4)])
@pytest.mark.parametrize("cfg", CFGS, ids=["auto", "staged", "gather"])
def test_compute_error_vs_fp64_oracle_of_same_data(volume, dtype, tol, cfg):
    xn, geo, ref = volume
    with schedule(cfg, DEV):
        img = ffdas_b200.das(xn.to(dtype), *geo)
    assert oracle.rel_l2(img.cpu().numpy(), ref(dtype)) < tol


@pytest.mark.parametrize("dtype,tol", [(torch.float16, 1e-3), (torch.bfloat16, 2e-3)])
def test_storage_error_vs_fp64_oracle_of_fp32_data(volume, dtype, tol):
    xn, geo, ref = volume
    img = ffdas_b200.das(xn.to(dtype), *geo)
    assert oracle.rel_l2(img.cpu().numpy(), ref(torch.float32)) < tol
