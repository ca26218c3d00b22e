"""CUDA-graph runner: captured ingest + kernel replays give the eager result."""
import pytest
import torch

import ffdas_b200
from ffdas_b200 import workloads as W
from ffdas_b200.runner import DASRunner
from oracle import oracle

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def test_runner_replays_match_eager_for_new_frames():
    wl = W.ensemble(device=DEV, scale=0.1, frames=6, dtype=torch.float16)
    geo = (wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
    run = DASRunner(wl["x"], *geo, tune=False, config=dict(variant=1, batch_tile=2))
    for k in range(3):
        xk = (wl["x"].float() * (1 + 0.1 * k)).roll(k, dims=-1).half()
        got = run(xk, clone=True)
        ref = ffdas_b200.das(xk, *geo)
        assert torch.equal(got, ref)


def test_runner_with_staged_schedule_and_sparse():
    wl = W.diverging3d(device=DEV, scale=0.25)
    geo = (wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
    run = DASRunner(wl["x"], *geo, tune=False, config=dict(variant=2, tile_x=16, tile_y=16, window=32))
    got = run(wl["x"] * 2, clone=True)
    assert oracle.rel_l2(got.cpu().numpy(), (ffdas_b200.das(wl["x"], *geo) * 2).cpu().numpy()) < 1e-6
    sp = W.sparse_focus(device=DEV, scale=0.2)
    geo_s = (sp["srcpos"], sp["dstpos"], sp["offsets"], sp["weights"])
    run_s = DASRunner(sp["x"], *geo_s, sparse_indices=sp["sparse_indices"], tune=True)
    ref = ffdas_b200.das_sparse(sp["x"], *geo_s, sp["sparse_indices"])
    assert torch.equal(run_s(sp["x"], clone=True), ref)


@pytest.mark.parametrize("depth", [1, 2, 3])
def test_stream_pipeline_matches_per_frame_calls(depth):
    from ffdas_b200.runner import DASStream
    wl = W.diverging3d(device=DEV, scale=0.25)
    geo = (wl["srcpos"], wl["dstpos"], wl["offsets"], wl["weights"])
    cfg = dict(variant=2, tile_x=32, tile_y=16, window=32)
    frames = [((wl["x"] * (1 + 0.25 * k)).roll(3 * k, dims=-1)).cpu().pin_memory() for k in range(5)]
    st = DASStream(wl["x"], *geo, depth=depth, tune=False, config=cfg)
    images = st.run(frames)
    assert len(images) == 5 and not images[0].is_cuda
    outs = [torch.empty_like(images[0]).pin_memory() for _ in frames]
    again = st.run(frames, outputs=outs)
    assert again[2] is outs[2]
    h = ffdas_b200.get_library_handle(DEV)
    h.set_config(cfg)
    for k, xh in enumerate(frames):
        ref = ffdas_b200.das(xh.to(DEV), *geo).cpu()
        assert oracle.rel_l2(images[k].numpy(), ref.numpy()) < 1e-6
        assert oracle.rel_l2(outs[k].numpy(), ref.numpy()) < 1e-6
