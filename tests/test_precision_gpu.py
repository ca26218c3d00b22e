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
  original FP32 data: quantising the channel data itself.  Over the whole
  image it is far inside the 1e-3 bar: the FP64 oracle of the bf16 data
  against that of the FP32 data gives 3.1e-5 relative L2 over all 128 depth
  planes (fp16: 2.6e-6), and 1.4-5.4e-5 over every 2nd, 4th, 8th or 16th
  plane, so the 16 planes 0, 8, ..., 120 stand for the volume here and are
  held to 1e-3.  Planes 66-127 lie past the end of the 4096-sample record
  and image to zero.  Plane by plane the relative error is larger where
  little signal is left: on the four planes below (two of them empty) bf16
  measured 1.04e-3 (the oracle of the bf16 data alone: 1.02e-3) and on eight
  1.72e-3 (1.70e-3); fp16 1.6e-4 and 3.7e-4.  Those four-plane checks stay
  at 2e-3 (bf16) and 1e-3 (fp16).
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


@pytest.fixture(scope="module")
def volume16():
    # depth planes 0, 8, ..., 120 of the same volume
    wl = W.diverging3d(device=DEV)
    xn = W.normalize_channels(wl["x"])
    sel = torch.arange(0, 128, 8, device=DEV)
    geo = (wl["srcpos"], wl["dstpos"][sel].contiguous(), wl["offsets"][:, sel].contiguous(),
           wl["weights"][:, sel].contiguous())
    ref = oracle.das_f64(xn.double().cpu().numpy(), *[t.cpu().numpy() for t in geo])
    return xn, geo, ref


@pytest.mark.parametrize("dtype", [torch.bfloat16, torch.float16])
def test_storage_error_over_the_volume(volume16, dtype):
    # the 16-bit image against the FP64 oracle of the FP32 data over 16
    # planes spread through the volume: the 1e-3 bar
    xn, geo, ref = volume16
    img = ffdas_b200.das(xn.to(dtype), *geo)
    err = oracle.rel_l2(img.cpu().numpy(), ref)
    assert err < 1e-3, err
    # the FP32 / FP16 pair storage of FP32 data on the same planes, same bar
    img_p = ffdas_b200.das(xn, *geo, **({"use_bf16": True} if dtype == torch.bfloat16 else {"use_fp16": True}))
    assert oracle.rel_l2(img_p.cpu().numpy(), ref) < 1e-3
