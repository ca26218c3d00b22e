"""ffdas_sparse_select against a numpy statement of the reference's host step
(bindings/python/examples/sparse_compounding.py:141-144: argpartition of the
weights over the event axis, take_along_axis of weights and delays), and the
example's end-to-end check: das_sparse over the selected lists equals das over
all events with the unselected weights set to zero.

Selection is exact integer work: indices must match bit for bit (with the
documented order: descending weight, NaN first, ties to the lower event).
"""
import numpy as np
import pytest
import torch

import ffdas_b200
from oracle import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _expected(w: np.ndarray, k: int):
    """numpy statement: stable sort on (NaN first, -weight, event index)."""
    S = w.shape[0]
    flat = w.reshape(S, -1)
    isn = np.isnan(flat)
    key = np.where(isn, -np.inf, -flat)
    # lexsort: last key is primary
    ev = np.broadcast_to(np.arange(S)[:, None], flat.shape)
    order = np.lexsort((ev, key, ~isn), axis=0)[:k]
    return order.astype(np.int32).reshape((k, *w.shape[1:]))


@pytest.mark.parametrize("S,k,shape", [(25, 8, (40, 33)), (64, 32, (1000,)), (7, 1, (3, 5, 7)), (5, 5, (300,)),
                                       (40, 16, (257,))])
def test_matches_numpy_selection(S, k, shape):
    g = torch.Generator().manual_seed(S * 100 + k)
    w = torch.rand((S, *shape), generator=g)
    offs = torch.rand((S, *shape), generator=g) * 100
    idx, sw, so = ffdas_b200.sparse_select(w.to(DEV), k, offsets=offs.to(DEV))
    exp = _expected(w.numpy(), k)
    assert idx.dtype == torch.int32 and tuple(idx.shape) == (k, *shape)
    np.testing.assert_array_equal(idx.cpu().numpy(), exp)
    np.testing.assert_array_equal(sw.cpu().numpy(), np.take_along_axis(w.numpy(), exp, axis=0))
    np.testing.assert_array_equal(so.cpu().numpy(), np.take_along_axis(offs.numpy(), exp, axis=0))
    # the selected set is the reference's argpartition set (no ties in this data)
    ref_set = np.sort(np.argpartition(w.numpy(), -k, axis=0)[-k:], axis=0)
    np.testing.assert_array_equal(np.sort(idx.cpu().numpy(), axis=0), ref_set)


def test_ties_nan_and_binary_masks():
    # the reference example's weights are a 0/1 beam mask: many ties
    g = torch.Generator().manual_seed(7)
    w = (torch.rand((25, 64, 48), generator=g) < 0.3).float()
    w[3, 0, :] = float("nan")
    w[:, 1, :] = 0.0
    idx, sw, so = ffdas_b200.sparse_select(w.to(DEV), 8)
    assert so is None
    exp = _expected(w.numpy(), 8)
    np.testing.assert_array_equal(idx.cpu().numpy(), exp)
    assert np.isnan(sw.cpu().numpy()[0, 0]).all()          # NaN ranks first
    np.testing.assert_array_equal(idx.cpu().numpy()[:, 1, 0], np.arange(8))   # all ties: lowest events


@pytest.mark.parametrize("S,k", [(64, 32), (33, 32), (100, 32), (200, 7)])
def test_signed_zeros_infinities_and_long_event_axes(S, k):
    # -0 and +0 tie (lower event first), infinities and NaN in both signs,
    # and event axes longer than 64 (the one-thread-per-voxel kernel)
    g = torch.Generator().manual_seed(S + 31 * k)
    w = torch.randn((S, 301), generator=g)
    pick = torch.randint(0, 8, (S, 301), generator=g)
    for code, val in enumerate([0.0, -0.0, float("inf"), -float("inf"), float("nan"), -float("nan"), 1.0]):
        w = torch.where(pick == code, torch.full_like(w, val), w)
    offs = torch.rand((S, 301), generator=g) * 100
    idx, sw, so = ffdas_b200.sparse_select(w.to(DEV), k, offsets=offs.to(DEV))
    exp = _expected(w.numpy(), k)
    np.testing.assert_array_equal(idx.cpu().numpy(), exp)
    got_w = sw.cpu().numpy()
    exp_w = np.take_along_axis(w.numpy(), exp, axis=0)
    np.testing.assert_array_equal(got_w.view(np.uint32), exp_w.view(np.uint32))   # the stored bits, -0 and NaN too
    np.testing.assert_array_equal(so.cpu().numpy(), np.take_along_axis(offs.numpy(), exp, axis=0))


def test_das_sparse_on_selected_lists_equals_masked_das():
    # bindings/python/examples/sparse_compounding.py:146-166: the two images agree
    g = torch.Generator().manual_seed(11)
    B, C, S, N = 1, 16, 12, 512
    x = torch.randn((B, C, S, N), generator=g)
    src = torch.zeros((C, 3))
    src[:, 0] = torch.linspace(-8, 8, C)
    zz, xx = torch.meshgrid(torch.linspace(30, 200, 24), torch.linspace(-10, 10, 20), indexing="ij")
    dst = torch.stack([xx, torch.zeros_like(xx), zz], -1)
    offs = torch.rand((S, 24, 20), generator=g) * 40 + zz[None]
    w = torch.rand((S, 24, 20), generator=g)
    k = 5
    idx, sw, so = ffdas_b200.sparse_select(w.to(DEV), k, offsets=offs.to(DEV))
    sparse = ffdas_b200.das_sparse(x.to(DEV), src.to(DEV), dst.to(DEV), so, sw, idx)
    mask = torch.zeros_like(w)
    mask.scatter_(0, idx.cpu().long(), 1.0)
    dense = ffdas_b200.das(x.to(DEV), src.to(DEV), dst.to(DEV), offs.to(DEV), (w * mask).to(DEV))
    assert oracle.rel_l2(sparse.cpu().numpy(), dense.cpu().numpy()) < 1e-6
