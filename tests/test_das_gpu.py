"""GPU parity of the forward das / das_sparse against the FP64 oracle.

Tolerances (relative L2 against the FP64 oracle on the same inputs):
  fp32 pairs  2e-5   (fp32 delay rounding, as in the reference's own fp32 path)
  fp16 pairs  2e-3   (11-bit storage of channel data)
  bf16 pairs  8e-3   (8-bit storage of channel data)
  fp64 pairs  2e-5   (delays stay fp32, as in the reference, so the delay
                      rounding bounds the error like in the fp32 path)
"""
import numpy as np
import pytest
import torch

import ffdas_b200
from ffdas_b200 import workloads as W
from oracle import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TOL = {torch.float32: 2e-5, torch.float16: 1e-3, torch.bfloat16: 2e-3, torch.float64: 2e-5}


def _np(t):
    return t.detach().cpu().numpy()


def _oracle_of(wl, x=None, **kw):
    x = wl["x"] if x is None else x
    return oracle.das_f64(_np(x.float() if x.dtype in (torch.float16, torch.bfloat16) else x), _np(wl["srcpos"]),
                          _np(wl["dstpos"]), _np(wl["offsets"]), _np(wl["weights"]),
                          sparse_indices=_np(wl["sparse_indices"]) if "sparse_indices" in wl else None, **kw)


def _run(wl, x=None, **kw):
    x = wl["x"] if x is None else x
    if "sparse_indices" in wl:
        return ffdas_b200.das_sparse(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"],
                                     wl["sparse_indices"], **kw)
    return ffdas_b200.das(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"], **kw)


CASES = [
    ("plane2d", dict(scale=0.25)),
    ("diverging3d", dict(scale=0.125)),
    ("ensemble", dict(scale=0.1, dtype=torch.float32)),
    ("sparse_focus", dict(scale=0.2)),
    ("autofocus", dict(scale=0.2)),
]


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_forward_fp32_matches_oracle(name, kw):
    wl = W.CONFIGS[name](device=DEV, **kw)
    x = wl["x"].float()
    got = _run(wl, x)
    ref = _oracle_of(wl, x)
    assert got.shape == ref.shape
    assert oracle.rel_l2(_np(got), ref) < TOL[torch.float32]


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16, torch.float64])
def test_forward_storage_dtypes(dtype):
    wl = W.diverging3d(device=DEV, scale=0.125)
    x = W.normalize_channels(wl["x"].double()).to(dtype)
    got = _run(wl, x)
    ref = _oracle_of(wl, x.double())
    assert got.dtype == (torch.float64 if dtype == torch.float64 else torch.float32)
    assert oracle.rel_l2(_np(got), ref) < TOL[dtype]


@pytest.mark.parametrize("flag", ["use_fp16", "use_bf16"])
def test_reduced_precision_from_fp32_input(flag):
    wl = W.diverging3d(device=DEV, scale=0.125)
    x = W.normalize_channels(wl["x"])
    got = _run(wl, x, **{flag: True})
    ref = _oracle_of(wl, x)
    tol = TOL[torch.float16] if flag == "use_fp16" else TOL[torch.bfloat16]
    assert oracle.rel_l2(_np(got), ref) < tol


def _small(rng, B=1, C=5, S=3, N=96, V=(6, 7), complex_=False, three_d=False):
    x = rng.standard_normal((B, C, S, N)).astype(np.float32)
    if complex_:
        x = (x + 1j * rng.standard_normal((B, C, S, N))).astype(np.complex64)
    src = rng.uniform(-4, 4, (C, 3)).astype(np.float32)
    src[:, 2] = 0
    zz, xx = np.meshgrid(np.linspace(20, 40, V[0]), np.linspace(-3, 3, V[1]), indexing="ij")
    dst = np.stack([xx, np.zeros_like(xx), zz], -1).astype(np.float32)   # (V0, V1, 3)
    offs = rng.uniform(-10, 40, (S, *V)).astype(np.float32)
    w = rng.uniform(0.1, 1, (S, *V)).astype(np.float32)
    if three_d:
        x = x[0]
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    return t(x), t(src), t(dst), t(offs), t(w)


@pytest.mark.parametrize("B", [1, 2, 3, 5, 8, 13])
def test_batch_sizes(rng, B):
    x, src, dst, offs, w = _small(rng, B=B)
    got = ffdas_b200.das(x, src, dst, offs, w)
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(offs), _np(w))
    assert got.shape == (B, *dst.shape[:-1])
    assert oracle.rel_l2(_np(got), ref) < 2e-5


def test_three_d_input_indexes_offsets_per_event(rng):
    x, src, dst, offs, w = _small(rng, three_d=True)
    got = ffdas_b200.das(x, src, dst, offs, w)
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(offs), _np(w))
    assert got.shape == tuple(dst.shape[:-1])
    assert oracle.rel_l2(_np(got), ref) < 2e-5


def test_complex_with_phase_rotation(rng):
    x, src, dst, offs, w = _small(rng, B=2, complex_=True)
    got = ffdas_b200.das(x, src, dst, offs, w, wavenum=-0.9)
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(offs), _np(w), wavenum=-0.9)
    assert got.dtype == torch.complex64
    assert oracle.rel_l2(_np(got), ref) < 1e-4   # __sincosf of large phases


def test_complex128(rng):
    x, src, dst, offs, w = _small(rng, complex_=True)
    x = x.to(torch.complex128)
    got = ffdas_b200.das(x, src, dst, offs, w, wavenum=0.0)
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(offs), _np(w))
    assert got.dtype == torch.complex128
    assert oracle.rel_l2(_np(got), ref) < 2e-5   # fp32 delays


def test_directivity(rng):
    x, src, dst, offs, w = _small(rng, B=2)
    srcdir = torch.zeros((src.shape[0], 4), device=DEV)
    srcdir[:, 2] = 1.0
    srcdir[:, 3] = 0.99
    got = ffdas_b200.das(x, src, dst, offs, w, srcdir=srcdir)
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(offs), _np(w), srcdir=_np(srcdir))
    assert oracle.rel_l2(_np(got), ref) < 2e-5
    assert not np.allclose(ref, oracle.das_f64(_np(x), _np(src), _np(dst), _np(offs), _np(w)))


def test_channels_trailing_and_strided_input(rng):
    x, src, dst, offs, w = _small(rng, B=2)
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(offs), _np(w))
    xt = x.transpose(1, 2).contiguous()            # (B, S, C, N)
    got = ffdas_b200.das(xt, src, dst, offs, w, channels_trailing=True)
    assert oracle.rel_l2(_np(got), ref) < 2e-5
    wide = torch.zeros((2, x.shape[1], x.shape[2], x.shape[3] + 7), device=DEV)
    wide[..., 3:3 + x.shape[3]] = x
    got2 = ffdas_b200.das(wide[..., 3:3 + x.shape[3]], src, dst, offs, w)  # strided rows
    assert oracle.rel_l2(_np(got2), ref) < 2e-5


def test_out_of_record_voxels_are_exact_zeros(rng):
    x, src, dst, offs, w = _small(rng)
    far = torch.full_like(offs, 1e6)
    assert torch.count_nonzero(ffdas_b200.das(x, src, dst, far, w)).item() == 0
    neg = torch.full_like(offs, -1e6)
    assert torch.count_nonzero(ffdas_b200.das(x, src, dst, neg, w)).item() == 0


@pytest.mark.parametrize("N", [1, 2, 3])
def test_tiny_records(rng, N):
    x, src, dst, offs, w = _small(rng, N=N)
    offs = torch.rand_like(offs) * N - 40  # r ~ 20..40 -> tau around 0..N
    got = ffdas_b200.das(x, src, dst, offs, w)
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(offs), _np(w))
    np.testing.assert_allclose(_np(got), ref, rtol=1e-4, atol=1e-5)


def test_single_voxel_and_impulse():
    # reference test_das.py:121
    x = torch.zeros((1, 1, 64), device=DEV)
    x[0, 0, 32] = 1.0
    out = ffdas_b200.das(x, torch.zeros((1, 3), device=DEV), torch.zeros((1, 3), device=DEV),
                         torch.full((1, 1), 32.0, device=DEV), torch.ones((1, 1), device=DEV))
    assert abs(float(out.squeeze()) - (1 - np.sqrt(1e-7))) < 1e-6


def test_zero_inputs(rng):
    x, src, dst, offs, w = _small(rng)
    assert torch.count_nonzero(ffdas_b200.das(torch.zeros_like(x), src, dst, offs, w)).item() == 0
    assert torch.count_nonzero(ffdas_b200.das(x, src, dst, offs, torch.zeros_like(w))).item() == 0


def test_sparse_matches_dense_and_skips_padding(rng):
    x, src, dst, offs, w = _small(rng, B=2, S=6)
    dense = ffdas_b200.das(x, src, dst, offs, w)
    S = offs.shape[0]
    idx = torch.arange(S, device=DEV, dtype=torch.int32).reshape(S, 1, 1).expand_as(offs).contiguous()
    pad = lambda t, v: torch.cat([t, torch.full((3, *t.shape[1:]), v, device=DEV, dtype=t.dtype)])  # noqa: E731
    sp = ffdas_b200.das_sparse(x, src, dst, pad(offs, 0.0), pad(w, 0.0), pad(idx, 0))
    assert oracle.rel_l2(_np(sp), _np(dense)) < 1e-6


def test_sparse_out_of_range_index_contributes_nothing(rng):
    x, src, dst, offs, w = _small(rng, S=4)
    idx = torch.randint(0, 4, offs.shape, device=DEV, dtype=torch.int32)
    base = ffdas_b200.das_sparse(x, src, dst, offs, w, idx)
    bad = idx.clone()
    bad[0] = 99
    w2 = w.clone()
    w2[0] = 0
    got = ffdas_b200.das_sparse(x, src, dst, offs, w, bad)
    ref = ffdas_b200.das_sparse(x, src, dst, offs, w2, idx)
    assert oracle.rel_l2(_np(got), _np(ref)) < 1e-6
    assert not torch.allclose(base, got)


@pytest.mark.parametrize("B", [1, 3])
def test_sparse_uneven_lists_with_holes(rng, B):
    # per-voxel list lengths 0..n, trailing padding, zero-weight holes and
    # out-of-range indices inside the lists: every kind of padding the
    # load-balanced sparse schedule must skip or neutralise
    x, src, dst, offs, w = _small(rng, B=B, S=7, V=(23, 19))
    n = 20
    V = dst.shape[:-1]
    g = torch.Generator().manual_seed(11)
    idx = torch.randint(0, 7, (n, *V), generator=g).int()
    length = torch.randint(0, n + 1, V, generator=g)
    ofs_s = (torch.rand((n, *V), generator=g) * 50 - 10).float()
    w_s = (torch.rand((n, *V), generator=g) + 0.1).float()
    w_s[torch.arange(n)[:, None, None] >= length[None]] = 0.0          # trailing padding
    w_s[torch.rand((n, *V), generator=g) < 0.1] = 0.0                    # holes
    idx[torch.rand((n, *V), generator=g) < 0.05] = 1000                  # out-of-range entries
    idx, ofs_s, w_s = idx.to(DEV), ofs_s.to(DEV), w_s.to(DEV)
    got = ffdas_b200.das_sparse(x, src, dst, ofs_s, w_s, idx)
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(ofs_s), _np(w_s), sparse_indices=_np(idx))
    assert oracle.rel_l2(_np(got), ref) < 2e-5


SCHEDULES = [
    dict(variant=1, tile_x=16, tile_y=16, batch_tile=1, event_chunk=16),
    dict(variant=1, tile_x=32, tile_y=8, batch_tile=2, event_chunk=4),
    dict(variant=1, tile_x=8, tile_y=8, tile_z=4, batch_tile=4, event_chunk=16),
    dict(variant=1, tile_x=64, tile_y=4, batch_tile=8, event_chunk=4),
]


@pytest.mark.parametrize("cfg", SCHEDULES, ids=lambda c: "x".join(str(c.get(k, 1)) for k in
                                                                   ("tile_x", "tile_y", "tile_z", "batch_tile",
                                                                    "event_chunk")))
def test_every_schedule_gives_the_same_image(rng, cfg):
    wl = W.diverging3d(device=DEV, scale=0.125)
    x = wl["x"].expand(3, *wl["x"].shape[1:]).contiguous()
    h = ffdas_b200.get_library_handle(DEV)
    ref = oracle.das_f64(_np(x), _np(wl["srcpos"]), _np(wl["dstpos"]), _np(wl["offsets"]), _np(wl["weights"]))
    try:
        h.set_config(cfg)
        got = ffdas_b200.das(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
        info = h.last_kernel_info()
    finally:
        h.set_config(None)
    assert info["tile_x"] == cfg["tile_x"] and info["batch_tile"] == cfg["batch_tile"]
    assert oracle.rel_l2(_np(got), ref) < 2e-5


def test_out_argument_and_no_grad_path(rng):
    x, src, dst, offs, w = _small(rng, B=2)
    out = torch.full((2, *dst.shape[:-1]), 7.0, device=DEV)
    res = ffdas_b200.das(x, src, dst, offs, w, out=out)
    assert res is out
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(offs), _np(w))
    assert oracle.rel_l2(_np(out), ref) < 2e-5


def test_runs_on_current_stream(rng):
    x, src, dst, offs, w = _small(rng, B=2)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        got = ffdas_b200.das(x, src, dst, offs, w)
    s.synchronize()
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(offs), _np(w))
    assert oracle.rel_l2(_np(got), ref) < 2e-5


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16, torch.bfloat16])
@pytest.mark.parametrize("B,bt", [(1, 1), (3, 2), (5, 4), (2, 4)])
def test_direct_kernel(dtype, B, bt):
    # one launch straight from x (no pair workspace): same taps as the f32
    # pairs of the other kernels, so the FP32 bound holds for all three inputs
    from ffdas_b200.tune import schedule
    wl = W.diverging3d(device=DEV, scale=0.125)
    x = (wl["x"].expand(B, *wl["x"].shape[1:]) * torch.arange(1, B + 1, device=DEV).view(B, 1, 1, 1)).to(dtype)
    h = ffdas_b200.get_library_handle(DEV)
    with schedule(dict(variant=5, batch_tile=bt), DEV):
        got = ffdas_b200.das(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
        info = h.last_kernel_info()
    assert info["variant"] == 5 and info["kernels"] == 1 and info["batch_tile"] == min(bt, 4 if B >= 4 else (2 if B >= 2 else 1))
    ref = oracle.das_f64(_np(x.float()), _np(wl["srcpos"]), _np(wl["dstpos"]), _np(wl["offsets"]), _np(wl["weights"]))
    assert oracle.rel_l2(_np(got), ref) < TOL[torch.float32]
    with schedule(dict(variant=2, tile_x=32, tile_y=8, window=32), DEV):
        staged = ffdas_b200.das(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
    if dtype == torch.float32:
        assert oracle.rel_l2(_np(got), _np(staged)) < 1e-6


def test_planner_takes_the_direct_kernel_for_small_frames():
    h = ffdas_b200.get_library_handle(DEV)
    h.set_config(None)
    small = W.plane2d(device=DEV, scale=0.5)
    out = ffdas_b200.das(small["x"], small["srcpos"], small["dstpos"], small["offsets"], small["weights"])
    info = h.last_kernel_info()
    assert info["variant"] == 5 and info["kernels"] == 1
    assert oracle.rel_l2(_np(out), _oracle_of(small)) < TOL[torch.float32]
    # complex data, sparse lists and 16-bit pair storage keep the other kernels
    sp = W.sparse_focus(device=DEV, scale=0.2)
    _run(sp)
    assert h.last_kernel_info()["variant"] != 5
    _run(small, small["x"].float(), use_fp16=True)
    assert h.last_kernel_info()["variant"] != 5


@pytest.mark.parametrize("lanes", [1, 2, 8, 32])
def test_direct_kernel_lanes_per_voxel(lanes):
    # lanes share a voxel's channels (ragged: 37 channels over 4-channel
    # unrolled steps); every split gives the same image up to summation order
    from ffdas_b200.tune import schedule
    g = torch.Generator().manual_seed(lanes)
    C, S, N = 37, 3, 300
    x = torch.randn((2, C, S, N), generator=g)
    src = torch.zeros((C, 3))
    src[:, 0] = torch.linspace(-6, 6, C)
    zz, xx = torch.meshgrid(torch.linspace(20, 120, 50), torch.linspace(-8, 8, 30), indexing="ij")
    dst = torch.stack([xx, torch.zeros_like(xx), zz], -1)
    offs = zz[None].expand(S, -1, -1) + torch.rand((S, 50, 30), generator=g) * 5
    w = torch.rand((S, 50, 30), generator=g)
    h = ffdas_b200.get_library_handle(DEV)
    with schedule(dict(variant=5, tile_x=lanes, batch_tile=2), DEV):
        got = ffdas_b200.das(x.to(DEV), src.to(DEV), dst.to(DEV), offs.to(DEV), w.to(DEV))
        info = h.last_kernel_info()
    assert info["variant"] == 5 and info["tile_x"] == lanes
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(offs), _np(w))
    assert oracle.rel_l2(_np(got), ref) < TOL[torch.float32]


@pytest.mark.parametrize("B", [1, 2])
def test_sparse_on_the_staged_kernel(rng, B):
    # lists over x's events run on the 512-voxel staged kernel (each pass takes
    # the entry naming its event); same image as the gather kernel and the oracle
    from ffdas_b200.tune import schedule
    x, src, dst, offs, w = _small(rng, B=B, C=9, S=8, N=200, V=(40, 30))
    g = torch.Generator().manual_seed(21)
    n = 5
    V = dst.shape[:-1]
    perm = torch.argsort(torch.rand((8, *V), generator=g), dim=0)[:n].int()   # distinct events per voxel
    ofs_s = (torch.rand((n, *V), generator=g) * 60 - 10).float()
    w_s = (torch.rand((n, *V), generator=g) + 0.1).float()
    w_s[-1, ::3] = 0.0                                                     # zero-weight padding
    perm[-1, ::3] = perm[0, ::3]                                           # ... repeating an index
    idx, ofs_s, w_s = perm.to(DEV), ofs_s.to(DEV), w_s.to(DEV)
    h = ffdas_b200.get_library_handle(DEV)
    with schedule(dict(variant=2), DEV):
        got = ffdas_b200.das_sparse(x, src, dst, ofs_s, w_s, idx)
        info = h.last_kernel_info()
    assert info["variant"] == 2 and info["kernels"] == 4 and info["tile_x"] * info["tile_y"] == 512
    with schedule(dict(variant=1), DEV):
        gat = ffdas_b200.das_sparse(x, src, dst, ofs_s, w_s, idx)
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(ofs_s), _np(w_s), sparse_indices=_np(idx))
    assert oracle.rel_l2(_np(got), ref) < TOL[torch.float32]
    assert oracle.rel_l2(_np(got), _np(gat)) < 1e-6


def test_sparse_list_naming_an_event_twice_falls_back_on_the_device(rng):
    # the staged pass holds one entry per voxel and event: a doubly named event
    # (both weights nonzero) sets the device gate and the gather kernel
    # computes the call; the result is the oracle's either way
    x, src, dst, offs, w = _small(rng, C=6, S=4, N=150, V=(20, 16))
    V = dst.shape[:-1]
    g = torch.Generator().manual_seed(5)
    idx = torch.stack([torch.full(V, e, dtype=torch.int32) for e in (0, 1, 2, 3)])
    idx[3, 4, 5] = 1                                                       # voxel (4, 5) names event 1 twice
    ofs_s = (torch.rand((4, *V), generator=g) * 40).float()
    w_s = (torch.rand((4, *V), generator=g) + 0.1).float()
    idx, ofs_s, w_s = idx.to(DEV), ofs_s.to(DEV), w_s.to(DEV)
    from ffdas_b200.tune import schedule
    h = ffdas_b200.get_library_handle(DEV)
    with schedule(dict(variant=2), DEV):
        got = ffdas_b200.das_sparse(x, src, dst, ofs_s, w_s, idx)
        assert h.last_kernel_info()["kernels"] == 4
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(ofs_s), _np(w_s), sparse_indices=_np(idx))
    assert oracle.rel_l2(_np(got), ref) < TOL[torch.float32]


@pytest.mark.parametrize("dup", [False, True], ids=["staged", "fallback"])
def test_sparse_channel_slices_with_beta(dup):
    # 96 channels over a small grid: the staged sparse call (asked for with
    # variant 2) splits the channels
    # over CTAs that add into a prepared image (beta * out); with a doubly
    # listed event the preparation is skipped and the gather kernel applies
    # beta instead -- out = beta * out + das_sparse either way
    import ctypes
    from ffdas_b200 import _lib
    from ffdas_b200._lib import DataType
    rng = np.random.default_rng(3)
    x, src, dst, offs, w = _small(rng, C=96, S=6, N=160, V=(24, 20))
    V = dst.shape[:-1]
    g = torch.Generator().manual_seed(9)
    idx = torch.argsort(torch.rand((6, *V), generator=g), dim=0)[:4].int()
    if dup:
        idx[2, 3, 3] = idx[0, 3, 3]
    ofs_s = (torch.rand((4, *V), generator=g) * 50).float()
    w_s = (torch.rand((4, *V), generator=g) + 0.1).float()
    idx, ofs_s, w_s = idx.to(DEV), ofs_s.to(DEV), w_s.to(DEV)
    h = ffdas_b200.get_library_handle(DEV)
    h.set_config(dict(variant=2))
    L = _lib.load()
    prev = torch.randn((1, *V), device=DEV)
    out = prev.clone()
    xd = _lib.TensorDesc(list(x.shape), None, DataType.R_32F)
    od = _lib.TensorDesc(list(out.shape), None, DataType.R_32F)
    beta = (ctypes.c_float * 2)(0.5, 0.0)
    h.set_stream(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.ffdas_das_sparse(h.h, src.data_ptr(), None, 0.0, xd.desc, x.data_ptr(), dst.data_ptr(),
                                  ofs_s.data_ptr(), w_s.data_ptr(), 4, idx.data_ptr(),
                                  ctypes.cast(beta, ctypes.c_void_p), od.desc, out.data_ptr(), 0, 0))
    info = h.last_kernel_info()
    h.set_config(None)
    torch.cuda.synchronize()
    assert info["variant"] == 2 and info["kernels"] == 5
    ref = 0.5 * _np(prev) + oracle.das_f64(_np(x), _np(src), _np(dst), _np(ofs_s), _np(w_s),
                                          sparse_indices=_np(idx))
    assert oracle.rel_l2(_np(out), ref) < TOL[torch.float32]


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex32])
@pytest.mark.parametrize("B", [1, 2])
def test_complex_on_the_staged_kernel(dtype, B):
    # IQ data with phase rotation and directivity on 64x80 pixels: the staged
    # complex kernel (schedule variant 2) sums in the gather kernel's order, so the two agree to
    # rounding of exact zeros; both match the FP64 oracle
    from ffdas_b200.tune import schedule
    rng = np.random.default_rng(17 + B)
    C, S, N = 24, 5, 400
    x = (rng.standard_normal((B, C, S, N)) + 1j * rng.standard_normal((B, C, S, N))).astype(np.complex64)
    src = np.zeros((C, 3), np.float32)
    src[:, 0] = np.linspace(-10, 10, C)
    zz, xx = np.meshgrid(np.linspace(30, 160, 64), np.linspace(-12, 12, 80), indexing="ij")
    dst = np.stack([xx, np.zeros_like(xx), zz], -1).astype(np.float32)
    offs = (zz[None] + rng.uniform(-5, 5, (S, 64, 80))).astype(np.float32)
    w = rng.uniform(0.2, 1.0, (S, 64, 80)).astype(np.float32)
    srcdir = np.zeros((C, 4), np.float32)
    srcdir[:, 2] = 1.0
    srcdir[:, 3] = 0.3
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    xt = t(x).to(dtype)
    wn = -2 * np.pi * 0.23
    h = ffdas_b200.get_library_handle(DEV)
    with schedule(dict(variant=2), DEV):
        got = ffdas_b200.das(xt, t(src), t(dst), t(offs), t(w), srcdir=t(srcdir), wavenum=wn)
        info = h.last_kernel_info()
    assert info["variant"] == 2 and got.dtype == torch.complex64
    with schedule(dict(variant=1), DEV):
        gat = ffdas_b200.das(xt, t(src), t(dst), t(offs), t(w), srcdir=t(srcdir), wavenum=wn)
    assert oracle.rel_l2(_np(got), _np(gat)) < 1e-7
    xr = xt.to(torch.complex64).cpu().numpy()
    ref = oracle.das_f64(xr, src, dst, offs, w, srcdir=srcdir, wavenum=wn)
    assert oracle.rel_l2(_np(got), ref) < 1e-3   # __sincosf of phases up to ~500 rad, as the reference


def test_sparse_gather_channel_slices_with_beta():
    # the gather kernel splits a small sparse call's channels over CTAs that
    # add into a prepared image: out = beta * out + das_sparse
    import ctypes
    from ffdas_b200 import _lib
    from ffdas_b200._lib import DataType
    rng = np.random.default_rng(8)
    x, src, dst, offs, w = _small(rng, C=96, S=6, N=160, V=(24, 20))
    V = dst.shape[:-1]
    g = torch.Generator().manual_seed(10)
    idx = torch.randint(0, 6, (5, *V), generator=g).int()
    ofs_s = (torch.rand((5, *V), generator=g) * 50).float()
    w_s = (torch.rand((5, *V), generator=g) + 0.1).float()
    idx, ofs_s, w_s = idx.to(DEV), ofs_s.to(DEV), w_s.to(DEV)
    h = ffdas_b200.get_library_handle(DEV)
    L = _lib.load()
    prev = torch.randn((1, *V), device=DEV)
    xd = _lib.TensorDesc(list(x.shape), None, DataType.R_32F)
    outs = []
    for cfg in (dict(variant=1, event_chunk=8), dict(variant=1, event_chunk=4, min_blocks=16)):
        out = prev.clone()
        od = _lib.TensorDesc(list(out.shape), None, DataType.R_32F)
        beta = (ctypes.c_float * 2)(-0.25, 0.0)
        h.set_config(cfg)
        h.set_stream(torch.cuda.current_stream().cuda_stream)
        _lib.check(L.ffdas_das_sparse(h.h, src.data_ptr(), None, 0.0, xd.desc, x.data_ptr(), dst.data_ptr(),
                                      ofs_s.data_ptr(), w_s.data_ptr(), 5, idx.data_ptr(),
                                      ctypes.cast(beta, ctypes.c_void_p), od.desc, out.data_ptr(), 0, 0))
        info = h.last_kernel_info()
        h.set_config(None)
        assert info["variant"] == 1 and info["kernels"] == 3, info
        outs.append(out)
    torch.cuda.synchronize()
    ref = -0.25 * _np(prev) + oracle.das_f64(_np(x), _np(src), _np(dst), _np(ofs_s), _np(w_s),
                                            sparse_indices=_np(idx))
    for out in outs:
        assert oracle.rel_l2(_np(out), ref) < TOL[torch.float32]


@pytest.mark.parametrize("cfg", [None, dict(variant=1), dict(variant=2, tile_x=16, tile_y=16, window=32),
                                 dict(variant=5)], ids=["planner", "gather", "staged", "direct"])
def test_int16_channel_data(cfg):
    # raw ADC samples: int16 x is interpolated in FP32 (FP32 pairs hold every
    # int16 exactly), so every kernel matches the oracle of the same integers
    from ffdas_b200.tune import schedule
    wl = W.diverging3d(device=DEV, scale=0.125)
    g = torch.Generator().manual_seed(3)
    x16 = (wl["x"].cpu() * 8000 + torch.randn(wl["x"].shape, generator=g) * 30).round().clamp(-32768, 32767)
    x16 = x16.to(torch.int16).to(DEV)
    h = ffdas_b200.get_library_handle(DEV)
    with schedule(cfg, DEV):
        got = ffdas_b200.das(x16, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
        info = h.last_kernel_info()
    assert got.dtype == torch.float32 and info["storage"] == 0
    if cfg is not None:
        assert info["variant"] == cfg["variant"]
    ref = oracle.das_f64(_np(x16).astype(np.float64), _np(wl["srcpos"]), _np(wl["dstpos"]), _np(wl["offsets"]),
                         _np(wl["weights"]))
    assert oracle.rel_l2(_np(got), ref) < TOL[torch.float32]


def test_int16_channel_data_gradients():
    # the adjoint runs on the same FP32 pairs; an int16 tensor carries no gradient
    # itself, the geometry does
    wl = W.autofocus(device=DEV, scale=0.2)
    x16 = (wl["x"] * 3000).round().to(torch.int16)
    xf = x16.float()
    leaves16 = [t.clone().requires_grad_(True) for t in (wl["offsets"], wl["weights"])]
    leavesf = [t.clone().requires_grad_(True) for t in (wl["offsets"], wl["weights"])]
    ffdas_b200.das(x16, wl["srcpos"], wl["dstpos"], *leaves16).square().sum().backward()
    ffdas_b200.das(xf, wl["srcpos"], wl["dstpos"], *leavesf).square().sum().backward()
    for a, b in zip(leaves16, leavesf):
        assert oracle.rel_l2(_np(a.grad), _np(b.grad)) < 1e-6


# ----------------------------------------------------------- channel scale ---
# ffdas_set_channel_scale: the ingest multiplies channel c (of item b) by its
# scale before storing the pairs, so the image is that of scale * x.

@pytest.mark.parametrize("cfg", [None, dict(variant=1), dict(variant=2, tile_x=16, tile_y=16, window=32)],
                         ids=["planner", "gather", "staged"])
@pytest.mark.parametrize("per_item", [False, True])
def test_channel_scale_fp32(cfg, per_item):
    from ffdas_b200.tune import schedule
    rng = np.random.default_rng(21)
    x, src, dst, offs, w = _small(rng, B=3, C=40, S=4, N=128, V=(24, 30))
    B, C = x.shape[0], x.shape[1]
    scale = torch.from_numpy(rng.uniform(0.2, 3.0, (B, C) if per_item else (C,)).astype(np.float32)).to(DEV)
    with schedule(cfg, DEV):
        got = ffdas_b200.das(x, src, dst, offs, w, channel_scale=scale)
    xs = _np(x).astype(np.float64) * (_np(scale).astype(np.float64).reshape(B if per_item else 1, C, 1, 1))
    ref = oracle.das_f64(xs, _np(src), _np(dst), _np(offs), _np(w))
    assert oracle.rel_l2(_np(got), ref) < TOL[torch.float32]
    # the setting does not outlive the call
    plain = ffdas_b200.das(x, src, dst, offs, w)
    assert oracle.rel_l2(_np(plain), oracle.das_f64(_np(x), _np(src), _np(dst), _np(offs), _np(w))) < 2e-5


def test_channel_scale_int16_gains_and_sparse():
    # raw ADC samples with per-channel gains, dense and das_sparse
    wl = W.diverging3d(device=DEV, scale=0.125)
    g = torch.Generator().manual_seed(5)
    x16 = (wl["x"].cpu() * 8000).round().clamp(-32768, 32767).to(torch.int16).to(DEV)
    C = x16.shape[1]
    gains = (torch.rand(C, generator=g) * 2 + 0.5).float().to(DEV)
    got = ffdas_b200.das(x16, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"], channel_scale=gains)
    xs = _np(x16).astype(np.float64) * _np(gains).astype(np.float64).reshape(1, C, 1, 1)
    geo = [_np(t) for t in (wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])]
    assert oracle.rel_l2(_np(got), oracle.das_f64(xs, *geo)) < TOL[torch.float32]
    S = x16.shape[2]
    V = wl["dstpos"].shape[:-1]
    idx = torch.argsort(torch.rand((S, *V), generator=g), dim=0)[: max(1, S // 2)].int().to(DEV)
    ofs_s = torch.gather(wl["offsets"], 0, idx.long())
    w_s = torch.gather(wl["weights"], 0, idx.long())
    got_s = ffdas_b200.das_sparse(x16, wl["srcpos"], wl["dstpos"], ofs_s, w_s, idx, channel_scale=gains)
    ref_s = oracle.das_f64(xs, geo[0], geo[1], _np(ofs_s), _np(w_s), sparse_indices=_np(idx))
    assert oracle.rel_l2(_np(got_s), ref_s) < TOL[torch.float32]


@pytest.mark.parametrize("flag,tol", [("use_bf16", TOL[torch.bfloat16]), ("use_fp16", TOL[torch.float16])])
def test_channel_scale_normalises_before_16bit_storage(flag, tol):
    # FP32 data normalised per channel (scale = 1 / peak) inside the ingest and
    # stored as 16-bit pairs: the image of the normalised data, as if the
    # caller had normalised it
    wl = W.diverging3d(device=DEV, scale=0.125)
    x = wl["x"] * 1e4   # far outside FP16's comfortable range before scaling
    peak = x.abs().amax(dim=(0, 2, 3)).clamp_min(1e-30)
    got = ffdas_b200.das(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"], channel_scale=1.0 / peak,
                         **{flag: True})
    xn = _np(x).astype(np.float64) / _np(peak).astype(np.float64).reshape(1, -1, 1, 1)
    ref = oracle.das_f64(xn, *[_np(t) for t in (wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])])
    assert oracle.rel_l2(_np(got), ref) < tol


def test_channel_scale_is_checked():
    rng = np.random.default_rng(2)
    x, src, dst, offs, w = _small(rng, B=2, C=6)
    with pytest.raises(ValueError):
        ffdas_b200.das(x, src, dst, offs, w, channel_scale=torch.ones(5, device=DEV))
    xg = x.clone().requires_grad_(True)
    with pytest.raises(NotImplementedError):
        ffdas_b200.das(xg, src, dst, offs, w, channel_scale=torch.ones(6, device=DEV))
    # through the C-ABI a wrong length is INVALID_ARGUMENT, and the backward refuses
    h = ffdas_b200.get_library_handle(DEV)
    bad = torch.ones(7, device=DEV)
    h.set_channel_scale(bad.data_ptr(), 7)
    try:
        with pytest.raises(RuntimeError):
            ffdas_b200.das(x, src, dst, offs, w)
    finally:
        h.set_channel_scale(None, 0)


# --------------------------------------------- das_sparse, persistent items ---
# das_sparse schedule variant 6: lists bucketed by event, tiles pulled from a
# queue longest first by a persistent grid, voxels of a pass ordered by their
# entry count, windows staged by TMA.

def _distinct_lists(g, S, n, V, p_zero=0.0):
    """Per voxel a list of up to n distinct events of S (random order), uneven
    lengths 0..n padded with zero weight and a repeated index."""
    perm = torch.argsort(torch.rand((S, *V), generator=g), dim=0)[:n].int()
    length = torch.randint(0, n + 1, V, generator=g)
    ofs_s = (torch.rand((n, *V), generator=g) * 60 - 10).float()
    w_s = (torch.rand((n, *V), generator=g) + 0.1).float()
    pad = torch.arange(n).reshape(n, *([1] * len(V))) >= length[None]
    w_s[pad] = 0.0
    perm[pad] = perm[0:1].expand_as(perm)[pad]
    if p_zero:
        w_s[torch.rand((n, *V), generator=g) < p_zero] = 0.0
    return perm, ofs_s, w_s


@pytest.mark.parametrize("cfg", [dict(variant=6), dict(variant=6, event_chunk=4), dict(variant=6, window=32)],
                         ids=["default", "chunk4", "window32"])
@pytest.mark.parametrize("B", [1, 3])
def test_sparse_items_uneven_lists(rng, cfg, B):
    from ffdas_b200.tune import schedule
    x, src, dst, offs, w = _small(rng, B=B, C=12, S=13, N=180, V=(37, 29))
    g = torch.Generator().manual_seed(31 + B)
    V = dst.shape[:-1]
    idx, ofs_s, w_s = _distinct_lists(g, 13, 9, V, p_zero=0.1)
    idx, ofs_s, w_s = idx.to(DEV), ofs_s.to(DEV), w_s.to(DEV)
    h = ffdas_b200.get_library_handle(DEV)
    with schedule(cfg, DEV):
        got = ffdas_b200.das_sparse(x, src, dst, ofs_s, w_s, idx)
        info = h.last_kernel_info()
    assert info["variant"] == 6
    with schedule(dict(variant=1), DEV):
        gat = ffdas_b200.das_sparse(x, src, dst, ofs_s, w_s, idx)
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(ofs_s), _np(w_s), sparse_indices=_np(idx))
    assert oracle.rel_l2(_np(got), ref) < TOL[torch.float32]
    assert oracle.rel_l2(_np(got), _np(gat)) < 1e-6


@pytest.mark.parametrize("dup", [False, True], ids=["items", "fallback"])
def test_sparse_items_channel_slices_with_beta(dup):
    # 128 channels over a small grid: the work items split the channels, each
    # slice adding into an image prepared with beta; a doubly named event
    # falls back to the gated gather kernel, which applies beta itself
    import ctypes
    from ffdas_b200 import _lib
    from ffdas_b200._lib import DataType
    rng = np.random.default_rng(8)
    x, src, dst, offs, w = _small(rng, C=128, S=10, N=160, V=(24, 20))
    V = dst.shape[:-1]
    g = torch.Generator().manual_seed(12)
    idx, ofs_s, w_s = _distinct_lists(g, 10, 6, V)
    if dup:
        idx[1, 3, 3] = idx[0, 3, 3]
        w_s[0, 3, 3] = w_s[1, 3, 3] = 0.7
    idx, ofs_s, w_s = idx.to(DEV), ofs_s.to(DEV), w_s.to(DEV)
    h = ffdas_b200.get_library_handle(DEV)
    h.set_config(dict(variant=6))
    L = _lib.load()
    prev = torch.randn((1, *V), device=DEV)
    out = prev.clone()
    xd = _lib.TensorDesc(list(x.shape), None, DataType.R_32F)
    od = _lib.TensorDesc(list(out.shape), None, DataType.R_32F)
    beta = (ctypes.c_float * 2)(0.5, 0.0)
    h.set_stream(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.ffdas_das_sparse(h.h, src.data_ptr(), None, 0.0, xd.desc, x.data_ptr(), dst.data_ptr(),
                                  ofs_s.data_ptr(), w_s.data_ptr(), idx.shape[0], idx.data_ptr(),
                                  ctypes.cast(beta, ctypes.c_void_p), od.desc, out.data_ptr(), 0, 0))
    info = h.last_kernel_info()
    h.set_config(None)
    torch.cuda.synchronize()
    assert info["variant"] == 6 and info["kernels"] == 6   # ingest, buckets, order, image prep, items, gather
    ref = 0.5 * _np(prev) + oracle.das_f64(_np(x), _np(src), _np(dst), _np(ofs_s), _np(w_s),
                                          sparse_indices=_np(idx))
    assert oracle.rel_l2(_np(out), ref) < TOL[torch.float32]


def test_sparse_items_3d_volume_and_16bit_storage():
    # a 3-D volume with half its transmits per voxel, FP32 and BF16 pair storage
    wl = W.diverging3d(device=DEV, scale=0.25)
    S = wl["x"].shape[2]
    V = wl["dstpos"].shape[:-1]
    g = torch.Generator().manual_seed(40)
    idx, _, w_s = _distinct_lists(g, S, max(1, S // 2), V)
    idx = idx.to(DEV)
    ofs_s = torch.gather(wl["offsets"], 0, idx.long())
    w_s = w_s.to(DEV) * torch.gather(wl["weights"], 0, idx.long())
    h = ffdas_b200.get_library_handle(DEV)
    geo = [_np(t) for t in (wl["srcpos"], wl["dstpos"])]
    ref = oracle.das_f64(_np(wl["x"]), *geo, _np(ofs_s), _np(w_s), sparse_indices=_np(idx))
    from ffdas_b200.tune import schedule
    with schedule(dict(variant=6), DEV):
        got = ffdas_b200.das_sparse(wl["x"], wl["srcpos"], wl["dstpos"], ofs_s, w_s, idx)
        assert h.last_kernel_info()["variant"] == 6
        xb = wl["x"].to(torch.bfloat16)
        gotb = ffdas_b200.das_sparse(xb, wl["srcpos"], wl["dstpos"], ofs_s, w_s, idx, use_bf16=True)
    assert oracle.rel_l2(_np(got), ref) < TOL[torch.float32]
    refb = oracle.das_f64(_np(xb.float()), *geo, _np(ofs_s), _np(w_s), sparse_indices=_np(idx))
    assert oracle.rel_l2(_np(gotb), refb) < TOL[torch.bfloat16]


# -------------------------------------------- host-resident channel data ---
# ffdas_das_from_host: x in host memory, uploaded in channel runs on the
# handle's upload stream while earlier runs are beamformed.

@pytest.mark.parametrize("B, chunks", [(1, 0), (1, 3), (2, 4), (3, 1), (1, 16)])
def test_das_from_host_matches_das(rng, B, chunks):
    x, src, dst, offs, w = _small(rng, B=B, C=40, S=3, N=200, V=(33, 27))
    xh = x.cpu().pin_memory()
    got = ffdas_b200.das_from_host(xh, src, dst, offs, w, chunks=chunks)
    assert got.is_cuda and got.shape == (B, 33, 27)
    dev = ffdas_b200.das(x, src, dst, offs, w)
    assert oracle.rel_l2(_np(got), _np(dev)) < 1e-6
    ref = oracle.das_f64(_np(x), _np(src), _np(dst), _np(offs), _np(w))
    assert oracle.rel_l2(_np(got), ref) < TOL[torch.float32]


def test_das_from_host_staged_volume_beta_and_pageable_memory():
    # a volume large enough for the staged kernel, run in 8 channel runs:
    # beta applies once (the first run), the later runs add; pageable host
    # memory gives the same image
    import ctypes
    from ffdas_b200 import _lib
    from ffdas_b200._lib import DataType
    wl = W.diverging3d(device=DEV, scale=0.5)          # 256 channels, 64^3 voxels: the staged kernel
    x = wl["x"]
    geo = (wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
    xh = x.cpu().pin_memory()
    h = ffdas_b200.get_library_handle(DEV)
    L = _lib.load()
    prev = torch.randn((x.shape[0], *wl["dstpos"].shape[:-1]), device=DEV)
    out = prev.clone()
    xd = _lib.TensorDesc(list(x.shape), None, DataType.R_32F)
    od = _lib.TensorDesc(list(out.shape), None, DataType.R_32F)
    beta = (ctypes.c_float * 2)(0.25, 0.0)
    h.set_stream(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.ffdas_das_from_host(h.h, geo[0].data_ptr(), None, 0.0, xd.desc, xh.data_ptr(), geo[1].data_ptr(),
                                     geo[2].data_ptr(), geo[3].data_ptr(), ctypes.cast(beta, ctypes.c_void_p),
                                     od.desc, out.data_ptr(), 0, 0, 8))
    torch.cuda.synchronize()
    assert h.last_kernel_info()["kernels"] >= 16          # ingest + kernel per run
    dev = ffdas_b200.das(x, *geo)
    assert oracle.rel_l2(_np(out), _np(0.25 * prev + dev)) < 1e-6
    got_pageable = ffdas_b200.das_from_host(x.cpu(), *geo)
    assert oracle.rel_l2(_np(got_pageable), _np(dev)) < 1e-6


def test_das_from_host_channel_scale_and_16bit():
    # per-channel scale is offset to each run; FP16 host data
    rng = np.random.default_rng(17)
    x, src, dst, offs, w = _small(rng, C=48, S=2, N=160, V=(20, 18))
    scale = torch.linspace(0.5, 2.0, 48, device=DEV)
    got = ffdas_b200.das_from_host(x.cpu().pin_memory(), src, dst, offs, w, chunks=3, channel_scale=scale)
    dev = ffdas_b200.das(x, src, dst, offs, w, channel_scale=scale)
    assert oracle.rel_l2(_np(got), _np(dev)) < 1e-6
    xh16 = x.half().cpu().pin_memory()
    got16 = ffdas_b200.das_from_host(xh16, src, dst, offs, w, chunks=3)
    dev16 = ffdas_b200.das(x.half(), src, dst, offs, w)
    assert oracle.rel_l2(_np(got16), _np(dev16)) < 1e-6


def test_das_from_host_rejections():
    import ctypes
    from ffdas_b200 import _lib
    from ffdas_b200._lib import DataType, Error
    rng = np.random.default_rng(18)
    x, src, dst, offs, w = _small(rng, C=8, S=2, N=64, V=(6, 5))
    with pytest.raises(ValueError, match="host memory"):
        ffdas_b200.das_from_host(x, src, dst, offs, w)                   # x already on the GPU
    with pytest.raises(ValueError, match="on the GPU"):
        ffdas_b200.das_from_host(x.cpu(), src.cpu(), dst, offs, w)       # geometry on the host
    with pytest.raises(ValueError):
        ffdas_b200.das_from_host(x.cpu(), src, dst, offs, w, chunks=-1)
    h = ffdas_b200.get_library_handle(DEV)
    L = _lib.load()
    xh = x.cpu()
    out = torch.empty((1, 6, 5), device=DEV)
    od = _lib.TensorDesc(list(out.shape), None, DataType.R_32F)
    beta = (ctypes.c_float * 2)()
    strided = _lib.TensorDesc([1, 8, 2, 32], [1024, 128, 64, 2], DataType.R_32F)   # every other sample
    rc = L.ffdas_das_from_host(h.h, src.data_ptr(), None, 0.0, strided.desc, xh.data_ptr(), dst.data_ptr(),
                               offs.data_ptr(), w.data_ptr(), ctypes.cast(beta, ctypes.c_void_p), od.desc,
                               out.data_ptr(), 0, 0, 0)
    assert rc == Error.NON_CONTIGUOUS
    xdsc = _lib.TensorDesc(list(xh.shape), None, DataType.R_32F)
    rc = L.ffdas_das_from_host(h.h, src.data_ptr(), None, 0.0, xdsc.desc, None, dst.data_ptr(), offs.data_ptr(),
                               w.data_ptr(), ctypes.cast(beta, ctypes.c_void_p), od.desc, out.data_ptr(), 0, 0, 0)
    assert rc == Error.NULL_POINTER
