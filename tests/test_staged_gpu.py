"""GPU tests of the TMA-staged forward kernel (variant 2).

* parity with the FP64 oracle (same tolerances as the gather kernel);
* bitwise identity with the L1-gather kernel when both use the same event
  chunk (same FFMA sequence per voxel);
* windows wider than a slot fall back to global reads and stay correct;
* the bounded-wait path: a test hook leaves the first pipeline stage unfilled,
  the kernel's waits expire (about 2 s), it returns without writing and the
  handle reports device status 1; the next call is normal again.
"""
import numpy as np
import pytest
import torch

import ffdas_b200
from ffdas_b200 import workloads as W, _lib
from ffdas_b200.tune import schedule, autotune
from oracle import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _np(t):
    return t.detach().cpu().numpy()


def _ref(wl, x):
    return oracle.das_f64(_np(x.float()), _np(wl["srcpos"]), _np(wl["dstpos"]), _np(wl["offsets"]),
                          _np(wl["weights"]))


def _run(wl, x, cfg, **kw):
    h = ffdas_b200.get_library_handle(DEV)
    with schedule(cfg, DEV):
        out = ffdas_b200.das(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"], **kw)
        info = h.last_kernel_info()
    return out, info


CASES = [
    ("diverging3d", dict(scale=0.25), dict(variant=2, tile_x=16, tile_y=16, window=32)),
    ("diverging3d", dict(scale=0.25), dict(variant=2, tile_x=32, tile_y=8, window=64, event_chunk=8)),
    # full-size 2-D grid: delays up to ~2000 samples, fp32 delay rounding (as in
    # the reference) puts FP32 vs FP64 at ~3e-5 here
    ("plane2d", dict(scale=1.0), dict(variant=2, tile_x=128, tile_y=2, window=64, tol=5e-5)),
    ("ensemble", dict(scale=0.1, dtype=torch.float32), dict(variant=2, tile_x=64, tile_y=4, window=64)),
    ("autofocus", dict(scale=0.25), dict(variant=2, tile_x=32, tile_y=8, window=32)),
    # 512-voxel tiles: two voxels per consumer thread
    ("diverging3d", dict(scale=0.25), dict(variant=2, tile_x=32, tile_y=16, window=32)),
    ("diverging3d", dict(scale=0.25), dict(variant=2, tile_x=16, tile_y=32, window=64, event_chunk=1)),
    ("plane2d", dict(scale=1.0), dict(variant=2, tile_x=128, tile_y=4, window=64, tol=5e-5)),
    ("ensemble", dict(scale=0.1, dtype=torch.float32), dict(variant=2, tile_x=64, tile_y=8, window=64)),
    ("autofocus", dict(scale=0.25), dict(variant=2, tile_x=32, tile_y=16, window=32)),
]


@pytest.mark.parametrize("copy", [1, 2], ids=["tma", "cp_async"])
@pytest.mark.parametrize("name,kw,cfg", CASES,
                         ids=[f"{c[0]}-{c[2]['tile_x']}x{c[2]['tile_y']}-w{c[2]['window']}" for c in CASES])
def test_staged_matches_oracle(name, kw, cfg, copy):
    wl = W.CONFIGS[name](device=DEV, **kw)
    x = wl["x"].float()
    cfg = dict(cfg, copy_engine=copy)
    tol = cfg.pop("tol", 2e-5)
    out, info = _run(wl, x, cfg)
    assert info["variant"] == 2 and info["copy_engine"] == copy
    assert info["tile_x"] * info["tile_y"] == cfg["tile_x"] * cfg["tile_y"]
    assert oracle.rel_l2(_np(out), _ref(wl, x)) < tol
    assert ffdas_b200.get_library_handle(DEV).device_status() == 0


@pytest.mark.parametrize("tile", [(16, 16), (32, 16)], ids=["256", "512"])
@pytest.mark.parametrize("dtype,flag", [(torch.float16, "use_fp16"), (torch.bfloat16, "use_bf16")])
def test_staged_16bit_pairs(dtype, flag, tile):
    # FP32 data stored as 16-bit pairs (the fp16 / bf16 compute types): the
    # image interpolates the rounded samples exactly
    wl = W.diverging3d(device=DEV, scale=0.25)
    x = W.normalize_channels(wl["x"])
    out, info = _run(wl, x, dict(variant=2, tile_x=tile[0], tile_y=tile[1], window=32), **{flag: True})
    assert info["variant"] == 2 and info["storage"] == (1 if dtype == torch.float16 else 2)
    assert oracle.rel_l2(_np(out), _ref(wl, x.to(dtype))) < 2e-5


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
def test_16bit_input_widens_to_fp32_pairs(dtype):
    wl = W.diverging3d(device=DEV, scale=0.25)
    x = W.normalize_channels(wl["x"]).to(dtype)
    out, info = _run(wl, x, dict(variant=2, tile_x=32, tile_y=16, window=32))
    assert info["storage"] == 0
    assert oracle.rel_l2(_np(out), _ref(wl, x)) < 2e-5


def test_staged_agrees_with_gather():
    # same taps; the staged kernel sums even and odd events in two packed
    # partial sums, so only the summation order differs
    wl = W.diverging3d(device=DEV, scale=0.25)
    x = wl["x"].float()
    a, _ = _run(wl, x, dict(variant=2, tile_x=16, tile_y=16, window=32, event_chunk=16))
    b, _ = _run(wl, x, dict(variant=1, tile_x=16, tile_y=16, batch_tile=1, event_chunk=16))
    c, _ = _run(wl, x, dict(variant=2, tile_x=32, tile_y=16, window=32, event_chunk=4))
    assert oracle.rel_l2(_np(a), _np(b)) < 1e-6
    assert oracle.rel_l2(_np(c), _np(b)) < 1e-6


def test_copy_engines_stage_identical_windows():
    # TMA tile loads and cp.async copies fill the same slots: bitwise equal images
    wl = W.diverging3d(device=DEV, scale=0.25)
    x = wl["x"].float()
    for wb in (32, 64):
        a, _ = _run(wl, x, dict(variant=2, tile_x=32, tile_y=8, window=wb, copy_engine=1))
        b, _ = _run(wl, x, dict(variant=2, tile_x=32, tile_y=8, window=wb, copy_engine=2))
        assert torch.equal(a, b)
    for dt in (torch.float16, torch.bfloat16):
        xs = W.normalize_channels(x).to(dt)
        a, _ = _run(wl, xs, dict(variant=2, tile_x=16, tile_y=16, window=64, copy_engine=1))
        b, _ = _run(wl, xs, dict(variant=2, tile_x=16, tile_y=16, window=64, copy_engine=2))
        assert torch.equal(a, b)


def test_overflowing_windows_fall_back_and_stay_correct():
    # 16x16 tiles on the 2-D grid (7 samples per voxel in depth) overflow every window
    wl = W.plane2d(device=DEV, scale=0.5)
    x = wl["x"]
    out, info = _run(wl, x, dict(variant=2, tile_x=16, tile_y=16, window=32))
    assert info["variant"] == 2
    assert oracle.rel_l2(_np(out), _ref(wl, x)) < 2e-5
    out, info = _run(wl, x, dict(variant=2, tile_x=32, tile_y=16, window=32))
    assert oracle.rel_l2(_np(out), _ref(wl, x)) < 2e-5


@pytest.mark.parametrize("tile", [(32, 8), (32, 16)], ids=["256", "512"])
def test_directivity_through_staged(rng, tile):
    wl = W.autofocus(device=DEV, scale=0.25)
    x = wl["x"].float()
    srcdir = torch.zeros((x.shape[-3], 4), device=DEV)
    srcdir[:, 2] = 1.0
    # an acceptance cosine that no (voxel, channel) pair of this lattice sits
    # on: at exactly 0.8 the 3-4-5 triangles of the grid make FP32 and FP64
    # disagree about which channels are inside
    srcdir[:, 3] = 0.8137
    out, info = _run(wl, x, dict(variant=2, tile_x=tile[0], tile_y=tile[1], window=32), srcdir=srcdir)
    ref = oracle.das_f64(_np(x), _np(wl["srcpos"]), _np(wl["dstpos"]), _np(wl["offsets"]), _np(wl["weights"]),
                         srcdir=_np(srcdir))
    assert info["variant"] == 2
    assert oracle.rel_l2(_np(out), ref) < 2e-5


@pytest.mark.parametrize("copy", [1, 2], ids=["tma", "cp_async"])
def test_bounded_wait_expires_into_a_status_not_a_hang(copy):
    wl = W.diverging3d(device=DEV, scale=0.125)
    x = wl["x"].float()
    h = ffdas_b200.get_library_handle(DEV)
    assert h.device_status() == 0
    sentinel = torch.full((1, *wl["dstpos"].shape[:-1]), 123.0, device=DEV)
    _lib.load().ffdas_debug_staged_drop_stage(1)
    with schedule(dict(variant=2, tile_x=16, tile_y=16, window=32, copy_engine=copy), DEV):
        ffdas_b200.das(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"], out=sentinel)
    torch.cuda.synchronize()
    assert h.device_status() == 1              # the kernel gave up and said so
    assert torch.all(sentinel == 123.0)        # and wrote nothing
    out, _ = _run(wl, x, dict(variant=2, tile_x=16, tile_y=16, window=32))
    assert h.device_status() == 0
    assert oracle.rel_l2(_np(out), _ref(wl, x)) < 2e-5


def test_autotune_picks_a_correct_schedule(tmp_path, monkeypatch):
    monkeypatch.setenv("FFDAS_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    wl = W.diverging3d(device=DEV, scale=0.25)
    x = wl["x"].float()
    best = autotune(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"], reps=1)
    assert best["ms"] > 0 and (tmp_path / "tune.json").exists()
    out, _ = _run(wl, x, best["config"])
    assert oracle.rel_l2(_np(out), _ref(wl, x)) < 2e-5
    again = autotune(x, wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"], reps=1)
    assert again["config"] == best["config"]


@pytest.mark.parametrize("cfg", [dict(variant=1, tile_x=32, tile_y=8), dict(variant=2, tile_x=32, tile_y=8, window=32),
                                 dict(variant=2, tile_x=32, tile_y=16, window=32), dict(variant=5, batch_tile=4)],
                         ids=["gather", "staged256", "staged512", "direct"])
def test_beta_accumulates_into_out(cfg):
    # out = beta * out + das(...), through the C-ABI (the Python API has no beta)
    import ctypes
    from ffdas_b200._lib import DataType
    wl = W.autofocus(device=DEV, scale=0.25)
    x = wl["x"].float().contiguous()
    h = ffdas_b200.get_library_handle(DEV)
    L = _lib.load()
    prev = torch.randn((x.shape[0], *wl["dstpos"].shape[:-1]), device=DEV)
    out = prev.clone()
    xd = _lib.TensorDesc(list(x.shape), None, DataType.R_32F)
    od = _lib.TensorDesc(list(out.shape), None, DataType.R_32F)
    beta = (ctypes.c_float * 2)(0.75, 0.0)
    with schedule(cfg, DEV):
        h.set_stream(torch.cuda.current_stream().cuda_stream)
        _lib.check(L.ffdas_das(h.h, wl["srcpos"].data_ptr(), None, 0.0, xd.desc, x.data_ptr(),
                               wl["dstpos"].data_ptr(), wl["offsets"].data_ptr(), wl["weights"].data_ptr(),
                               ctypes.cast(beta, ctypes.c_void_p), od.desc, out.data_ptr(), 0, 0))
        assert h.last_kernel_info()["variant"] == cfg["variant"]
    torch.cuda.synchronize()
    ref = 0.75 * _np(prev) + _ref(wl, x)
    assert oracle.rel_l2(_np(out), ref) < 2e-5


@pytest.mark.parametrize("B,bt,ec,wb", [(4, 2, 8, 32), (4, 4, 4, 32), (5, 4, 8, 64), (11, 8, 4, 64), (3, 2, 4, 64)],
                         ids=lambda v: str(v))
def test_batch_tiles_match_oracle(B, bt, ec, wb):
    # several batch items per CTA share each window's delays; B not a multiple
    # of the batch tile leaves items past B with zero windows
    wl = W.ensemble(device=DEV, scale=0.1, frames=B, dtype=torch.float32)
    x = wl["x"]
    out, info = _run(wl, x, dict(variant=2, tile_x=32, tile_y=8, window=wb, event_chunk=ec, batch_tile=bt))
    assert info["variant"] == 2 and info["batch_tile"] == bt
    assert oracle.rel_l2(_np(out), _ref(wl, x)) < 2e-5


@pytest.mark.parametrize("dtype,flag", [(torch.float16, "use_fp16"), (torch.bfloat16, "use_bf16")])
def test_batch_tiles_16bit(dtype, flag):
    wl = W.ensemble(device=DEV, scale=0.1, frames=6, dtype=torch.float32)
    x = wl["x"]
    out, info = _run(wl, x, dict(variant=2, tile_x=64, tile_y=4, window=64, batch_tile=4), **{flag: True})
    assert info["batch_tile"] == 4 and info["storage"] in (1, 2)
    assert oracle.rel_l2(_np(out), _ref(wl, x.to(dtype))) < 2e-5
    x16 = x.to(dtype)   # 16-bit data, default compute: FP32 pairs
    out, info = _run(wl, x16, dict(variant=2, tile_x=64, tile_y=4, window=64, batch_tile=4))
    assert info["storage"] == 0
    assert oracle.rel_l2(_np(out), _ref(wl, x16)) < 2e-5


def test_default_planner_picks_staged_for_dense_volumes():
    h = ffdas_b200.get_library_handle(DEV)
    h.set_config(None)
    wl = W.diverging3d(device=DEV, scale=0.4)   # 1.3e8 units: above the direct kernel's range
    out = ffdas_b200.das(wl["x"], wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
    info = h.last_kernel_info()
    assert info["variant"] == 2 and info["tile_x"] * info["tile_y"] * info["tile_z"] == 512
    # 1638 samples: delays up to ~1.6e3, so the fp32 delay rounding bound is wider
    assert oracle.rel_l2(_np(out), _ref(wl, wl["x"])) < 5e-5
    af = W.autofocus(device=DEV, scale=0.25)
    out = ffdas_b200.das(af["x"], af["srcpos"], af["dstpos"], af["offsets"], af["weights"])
    info = h.last_kernel_info()
    assert info["variant"] == 2 and info["batch_tile"] == 4
    assert oracle.rel_l2(_np(out), _ref(af, af["x"])) < 2e-5


@pytest.mark.parametrize("dtype,kind", [(torch.float16, 1), (torch.bfloat16, 2)])
def test_large_16bit_batches_keep_16bit_pairs(dtype, kind):
    # eight or more items: the 16-bit data stays in 16-bit pairs (bytes count
    # once the per-tap arithmetic is shared); the image is the same
    wl = W.ensemble(device=DEV, scale=0.1, frames=9, dtype=dtype)
    x = wl["x"]
    out, info = _run(wl, x, dict(variant=2, tile_x=32, tile_y=8, window=64, batch_tile=8))
    assert info["storage"] == kind and info["batch_tile"] == 8
    assert oracle.rel_l2(_np(out), _ref(wl, x)) < 2e-5


@pytest.mark.parametrize("tile", [(32, 8), (32, 16)], ids=["256", "512"])
def test_channel_split_for_small_problems(tile):
    # a small image splits each tile's channels over several CTAs that add
    # into it; a lower CTA target (min_blocks=1) splits less: same image
    wl = W.plane2d(device=DEV, scale=1.0)
    x = wl["x"]
    cfg = dict(variant=2, tile_x=tile[0], tile_y=tile[1], window=64)
    a, ia = _run(wl, x, cfg)
    b, ib = _run(wl, x, dict(cfg, min_blocks=1))
    assert ia["grid"] > ib["grid"] and ia["kernels"] == 3
    assert oracle.rel_l2(_np(a), _np(b)) < 1e-6
    assert oracle.rel_l2(_np(a), _ref(wl, x)) < 5e-5
