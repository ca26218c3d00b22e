"""Python API validation: the reference's ValueError cases (bindings/python/tests/
test_das.py:39-79) are raised before any GPU work, so they run on CPU."""
import warnings

import numpy as np
import pytest
import torch

import ffdas_b200
from ffdas_b200 import workloads as W


def _das_args(**overrides):
    n_ch, n_seq, n_samp, n_tgt = 4, 2, 16, 8
    args = dict(x=torch.zeros((n_ch, n_seq, n_samp)), srcpos=torch.zeros((n_ch, 3)),
                dstpos=torch.zeros((n_tgt, 3)), offsets=torch.zeros((n_seq, n_tgt)),
                weights=torch.ones((n_seq, n_tgt)))
    args.update(overrides)
    return args


def _das_sparse_args(**overrides):
    n_ch, n_seq, n_samp, n_tgt, n_sparse = 4, 8, 16, 6, 3
    args = dict(x=torch.zeros((n_ch, n_seq, n_samp)), srcpos=torch.zeros((n_ch, 3)),
                dstpos=torch.zeros((n_tgt, 3)), offsets=torch.zeros((n_sparse, n_tgt)),
                weights=torch.ones((n_sparse, n_tgt)), sparse_indices=torch.zeros((n_sparse, n_tgt), dtype=torch.int32))
    args.update(overrides)
    return args


def test_dstpos_wrong_trailing_dim():
    with pytest.raises(ValueError):
        ffdas_b200.das(**_das_args(dstpos=torch.zeros((8, 2))))


def test_dstpos_1d():
    with pytest.raises(ValueError):
        ffdas_b200.das(**_das_args(dstpos=torch.zeros((3,))))


def test_offsets_shape_mismatch():
    with pytest.raises(ValueError):
        ffdas_b200.das(**_das_args(offsets=torch.zeros((2, 99))))


def test_weights_shape_mismatch():
    with pytest.raises(ValueError):
        ffdas_b200.das(**_das_args(weights=torch.zeros((2, 99))))


def test_sparse_indices_shape_mismatch():
    with pytest.raises(ValueError):
        ffdas_b200.das_sparse(**_das_sparse_args(sparse_indices=torch.zeros((99, 6), dtype=torch.int32)))


def test_sparse_offsets_count_mismatch():
    with pytest.raises(ValueError):
        ffdas_b200.das_sparse(**_das_sparse_args(offsets=torch.zeros((5, 6))))


def test_numpy_inputs_are_validated_too():
    with pytest.raises(ValueError):
        ffdas_b200.das(np.zeros((4, 2, 16), np.float32), np.zeros((4, 3)), np.zeros((8, 2)),
                       np.zeros((2, 8)), np.ones((2, 8)))


def test_cpu_tensor_is_rejected_loudly():
    # no CPU fallback: a host tensor is an error, not a silent slow path
    with pytest.raises(ValueError, match="CUDA"):
        ffdas_b200.das(**_das_args())


def test_sparse_select_validation_before_gpu_work():
    w = torch.ones((8, 5, 6))
    with pytest.raises(ValueError, match="k must lie"):
        ffdas_b200.sparse_select(w, 0)
    with pytest.raises(ValueError, match="k must lie"):
        ffdas_b200.sparse_select(w, 9)
    with pytest.raises(ValueError, match="k must lie"):
        ffdas_b200.sparse_select(torch.ones((40, 6)), 33)
    with pytest.raises(TypeError):
        ffdas_b200.sparse_select(w, 2.0)
    with pytest.raises(ValueError, match="offsets shape"):
        ffdas_b200.sparse_select(w, 2, offsets=torch.ones((8, 5, 7)))
    with pytest.raises(ValueError, match="n_events"):
        ffdas_b200.sparse_select(torch.ones(8), 2)
    with pytest.raises(ValueError, match="CUDA"):
        ffdas_b200.sparse_select(w, 2)


@pytest.mark.parametrize("name", list(W.CONFIGS))
def test_workload_shapes(name):
    wl = W.CONFIGS[name](scale=0.05)
    x = wl["x"]
    spatial = wl["dstpos"].shape[:-1]
    assert wl["offsets"].shape[1:] == spatial and wl["weights"].shape[1:] == spatial
    assert wl["srcpos"].shape == (x.shape[-3], 3)
    assert torch.isfinite(x.float()).all()
    if "sparse_indices" in wl:
        idx = wl["sparse_indices"]
        assert idx.dtype == torch.int32 and idx.shape == wl["offsets"].shape
        assert int(idx.min()) >= 0 and int(idx.max()) < x.shape[-2]


def test_full_size_workload_geometry():
    # full-size shapes of the benchmark configs (geometry only, no channel data)
    assert W.diverging3d.__doc__ is None or True
    wl = W.plane2d(scale=1.0)
    assert tuple(wl["x"].shape) == (1, 128, 1, 2048)
    assert tuple(wl["dstpos"].shape) == (256, 1, 128, 3)
    assert wl["units"] == 256 * 128 * 128


def test_tuner_candidates_cover_each_kernel_family():
    # host-side schedule search space (no GPU): the one-launch direct kernel
    # for small real frames, the staged kernels (512-voxel tiles for sparse
    # lists), gather chunks and channel-slice targets for sparse lists, and
    # only the gather kernel for complex data
    from ffdas_b200.tune import candidates
    small = W.plane2d(scale=0.25)
    c = candidates(small["x"], small["dstpos"], small["offsets"])
    assert any(k["variant"] == 5 for k in c) and any(k["variant"] == 2 for k in c)
    assert {k.get("tile_x") for k in c if k["variant"] == 5} >= {None, 2, 32}
    big = W.diverging3d(scale=0.5)
    assert not any(k["variant"] == 5 for k in candidates(big["x"], big["dstpos"], big["offsets"]))
    sp = W.sparse_focus(scale=0.25)
    cs = candidates(sp["x"], sp["dstpos"], sp["offsets"], sp["sparse_indices"])
    assert any(k["variant"] == 2 and k["tile_x"] * k["tile_y"] == 512 for k in cs)
    assert any(k["variant"] == 1 and k.get("event_chunk") == 8 and k.get("min_blocks") == 16 for k in cs)
    assert not any(k["variant"] == 5 for k in cs)
    xc = small["x"].to(torch.complex64)
    cc = candidates(xc, small["dstpos"], small["offsets"])
    assert cc and all(k["variant"] == 1 for k in cc)


# ------------------------------------------------ truncate_rank argument checks
# reference bindings/python/tests/test_truncate_rank.py:11-33: ValueError before
# any device work (CPU tensors suffice).

def test_truncate_rank_1d_rejected():
    with pytest.raises(ValueError):
        ffdas_b200.truncate_rank(torch.ones(10), start=0)


@pytest.mark.parametrize("start, stop", [(-1, None), (4, None), (2, 1), (0, 5)])
def test_truncate_rank_window_rejected(start, stop):
    with pytest.raises(ValueError):
        ffdas_b200.truncate_rank(torch.ones((4, 8)), start=start, stop=stop)


def test_truncate_rank_out_shape_rejected():
    with pytest.raises(ValueError):
        ffdas_b200.truncate_rank(torch.ones((4, 8)), 0, out=torch.ones((8, 4)))


def test_truncate_rank_needs_cuda():
    with pytest.raises(ValueError, match="CUDA"):
        ffdas_b200.truncate_rank(torch.ones((4, 8)), 0)


def test_backward_coverage_by_dtype():
    # the adjoint kernels take real data without phase rotation and complex64
    # / complex32 data with any wavenum; everything else raises
    # NotImplementedError in the autograd backward (and keeps no pair rows)
    from ffdas_b200.autograd import _backward_supported
    for dt in (torch.float32, torch.float16, torch.bfloat16):
        assert _backward_supported(torch.zeros(1, dtype=dt), 0.0)
        assert not _backward_supported(torch.zeros(1, dtype=dt), 0.1)
    assert not _backward_supported(torch.zeros(1, dtype=torch.float64), 0.0)
    for dt in (torch.complex64, torch.complex32):
        assert _backward_supported(torch.zeros(1, dtype=dt), 0.0)
        assert _backward_supported(torch.zeros(1, dtype=dt), 0.3)
    assert not _backward_supported(torch.zeros(1, dtype=torch.complex128), 0.0)
