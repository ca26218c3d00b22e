"""Parity with the reference implementation itself, run live on the GPU.

The reference's das path is compiled from its sources into
oracle/_ref/libffdas_ref.so (`make -C oracle ref`) and driven through its own
C-ABI by oracle/reference.py, which pads x so the reference's unmasked loads
stay inside memory it owns.  Tolerance (relative L2, the parity bar): FP32
1e-5 against the reference's FP32 das on the same inputs.
"""
import numpy as np
import pytest
import torch

import ffdas_b200
from ffdas_b200 import workloads as W
from oracle import oracle, reference

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not reference.available(), reason="reference library not built")]
DEV = "cuda:0"


def _ours(wl, x):
    if "sparse_indices" in wl:
        return ffdas_b200.das_sparse(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"],
                                     wl["sparse_indices"])
    return ffdas_b200.das(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])


CASES = [
    ("plane2d", dict(scale=1.0)),
    ("diverging3d", dict(scale=0.25)),
    ("autofocus", dict(scale=0.5)),
    ("sparse_focus", dict(scale=0.25)),
]


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_fp32_matches_reference_das(name, kw):
    wl = W.CONFIGS[name](device=DEV, **kw)
    x = wl["x"].float().contiguous()
    ours = _ours(wl, x)
    ref = reference.das(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"],
                        sparse_indices=wl.get("sparse_indices"), alg=1)
    err = oracle.rel_l2(ours.cpu().numpy(), ref.cpu().numpy())
    assert err < 1e-5, err


def test_batched_ensemble_matches_reference_alg1():
    # ALG1 with the 16-frame register tile (FFDAS_ALG1_TILE_SIZE=16; the
    # default tile of 32 is rejected for float output, das_alg1.cu:219-239).
    # The reference's ALG2 is not used as a bar: on this case its image
    # differed from its own ALG1 and from the FP64 oracle (rel-L2 ~1.0).
    wl = W.ensemble(device=DEV, scale=0.2, frames=16, dtype=torch.float32)
    x = wl["x"].contiguous()
    ours = ffdas_b200.das(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
    ref1 = reference.das(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"], alg=1, tile=16)
    assert oracle.rel_l2(ours.cpu().numpy(), ref1.cpu().numpy()) < 1e-5


def test_fp16_input_against_reference_and_oracle():
    wl = W.diverging3d(device=DEV, scale=0.25)
    x = W.normalize_channels(wl["x"]).half().contiguous()
    ours = ffdas_b200.das(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
    ref = reference.das(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"], alg=1)
    exact = oracle.das_f64(x.float().cpu().numpy(), wl["srcpos"].cpu().numpy(), wl["dstpos"].cpu().numpy(),
                           wl["offsets"].cpu().numpy(), wl["weights"].cpu().numpy())
    e_ours = oracle.rel_l2(ours.cpu().numpy(), exact)
    e_ref = oracle.rel_l2(ref.cpu().numpy(), exact)
    # our fp16 path interpolates in fp32; the reference interpolates in fp16
    assert e_ours <= e_ref * 1.01 + 1e-6, (e_ours, e_ref)
