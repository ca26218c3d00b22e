"""CPU checks of the oracle (FP64 restatement) and of the pure-torch reference.

The known-answer cases are the reference's own das tests
(bindings/python/tests/test_das.py:83-132) re-expressed on numpy; the
reference-output fixtures under tests/golden/ pin the oracle to outputs of the
reference library itself (see tests/golden/make_golden.py).
"""
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import oracle
from tests.torch_ref import das_ref

GOLDEN = Path(__file__).resolve().parent / "golden"


def _args(n_ch=4, n_seq=2, n_samp=16, n_tgt=8):
    # reference test_das.py:8-19
    return dict(
        x=np.zeros((n_ch, n_seq, n_samp), np.float32),
        srcpos=np.zeros((n_ch, 3), np.float32),
        dstpos=np.zeros((n_tgt, 3), np.float32),
        offsets=np.zeros((n_seq, n_tgt), np.float32),
        weights=np.ones((n_seq, n_tgt), np.float32),
    )


def test_zero_input_zero_output():
    out = oracle.das_f64(**_args())
    np.testing.assert_allclose(out, 0.0, atol=1e-12)


def test_zero_weights_zero_output(rng):
    a = _args()
    a["x"] = rng.standard_normal(a["x"].shape).astype(np.float32)
    a["weights"] = np.zeros_like(a["weights"])
    np.testing.assert_allclose(oracle.das_f64(**a), 0.0, atol=1e-12)


def test_output_shapes():
    a = _args()
    a["dstpos"] = np.zeros((8, 6, 3), np.float32)
    a["offsets"] = np.zeros((2, 8, 6), np.float32)
    a["weights"] = np.ones((2, 8, 6), np.float32)
    assert oracle.das_f64(**a).shape == (8, 6)
    a["x"] = np.zeros((3, 4, 2, 32), np.float32)
    assert oracle.das_f64(**a).shape == (3, 8, 6)


def test_single_sample_impulse():
    # reference test_das.py:121: |out| > 0.5; exact value 1 - sqrt(1e-7)
    x = np.zeros((1, 1, 64), np.float32)
    x[0, 0, 32] = 1.0
    out = oracle.das_f64(x, np.zeros((1, 3)), np.zeros((1, 3)), np.full((1, 1), 32.0), np.ones((1, 1)))
    assert abs(out[0] - (1.0 - np.sqrt(1e-7))) < 1e-12


def test_linear_interpolation_and_bounds():
    N = 10
    x = np.arange(N, dtype=np.float32)[None, None] ** 2  # x[k] = k^2
    src = np.zeros((1, 3), np.float32)
    dst = np.array([[0.0, 0.0, 2.25]], np.float32)       # r = 2.25
    for ofs, want in [(0.0, 4 + 0.25 * 5), (-3.0, 0.0), (N - 2 - 2.25 + 0.5, 64 + 0.5 * 17),
                      (N - 1 - 2.25, 0.0), (N - 1 - 2.25 - 1e-3, None)]:
        out = oracle.das_f64(x, src, dst, np.array([[ofs]], np.float32), np.ones((1, 1), np.float32))
        if want is None:
            assert out[0] != 0.0          # k = N-2 is the last valid cell
        else:
            assert abs(out[0] - want) < 1e-4, (ofs, out[0], want)


def test_sparse_with_all_events_equals_dense(rng):
    C, S, N, V = 3, 5, 64, 7
    x = rng.standard_normal((2, C, S, N)).astype(np.float32)
    src = rng.uniform(-3, 3, (C, 3)).astype(np.float32)
    dst = rng.uniform(-3, 3, (V, 3)).astype(np.float32) + [0, 0, 10]
    offs = rng.uniform(0, 30, (S, V)).astype(np.float32)
    w = rng.uniform(0, 1, (S, V)).astype(np.float32)
    dense = oracle.das_f64(x, src, dst, offs, w)
    idx = np.repeat(np.arange(S, dtype=np.int32)[:, None], V, 1)
    sparse = oracle.das_f64(x, src, dst, offs, w, sparse_indices=idx)
    np.testing.assert_allclose(sparse, dense, rtol=1e-12, atol=1e-12)
    # padding entries with weight 0 change nothing (uneven subsets)
    idx2 = np.concatenate([idx, np.zeros((2, V), np.int32)])
    offs2 = np.concatenate([offs, np.zeros((2, V), np.float32)])
    w2 = np.concatenate([w, np.zeros((2, V), np.float32)])
    np.testing.assert_allclose(oracle.das_f64(x, src, dst, offs2, w2, sparse_indices=idx2), dense,
                               rtol=1e-12, atol=1e-12)


def test_directivity_excludes_channels(rng):
    C, N = 4, 64
    x = rng.standard_normal((C, 1, N)).astype(np.float32)
    src = np.zeros((C, 3), np.float32)
    dst = np.array([[0, 0, 10.0]], np.float32)
    offs = np.full((1, 1), 5.0, np.float32)
    w = np.ones((1, 1), np.float32)
    dirs = np.zeros((C, 4), np.float32)
    dirs[:, 2] = 1.0
    dirs[:, 3] = 0.5
    base = oracle.das_f64(x, src, dst, offs, w)
    assert abs(oracle.das_f64(x, src, dst, offs, w, srcdir=dirs)[0] - base[0]) < 1e-12
    dirs[:, 2] = -1.0  # pointing away: every channel excluded
    assert oracle.das_f64(x, src, dst, offs, w, srcdir=dirs)[0] == 0.0


def test_complex_phase_rotation(rng):
    C, N = 2, 64
    x = (rng.standard_normal((C, 1, N)) + 1j * rng.standard_normal((C, 1, N))).astype(np.complex64)
    src = np.zeros((C, 3), np.float32)
    dst = np.array([[0, 0, 7.0]], np.float32)
    offs = np.full((1, 1), 3.0, np.float32)
    w = np.ones((1, 1), np.float32)
    k0 = oracle.das_f64(x, src, dst, offs, w, wavenum=0.0)
    kw = oracle.das_f64(x, src, dst, offs, w, wavenum=0.75)
    np.testing.assert_allclose(kw, k0 * np.exp(1j * 0.75 * 10.0), rtol=1e-9)


def test_beta_accumulates(rng):
    a = _args()
    a["x"] = rng.standard_normal(a["x"].shape).astype(np.float32)
    a["offsets"] = rng.uniform(0, 8, a["offsets"].shape).astype(np.float32)
    base = oracle.das_f64(**a)
    prev = rng.standard_normal(base.shape)
    out = oracle.das_f64(**a, beta=0.5, out=prev.copy())
    np.testing.assert_allclose(out, 0.5 * prev + base, rtol=1e-12)


def test_q1_event0_indexing(rng):
    # reference quirk: 3-D x reuses event 0's offsets/weights for every event
    C, S, N, V = 2, 3, 32, 4
    x = rng.standard_normal((C, S, N)).astype(np.float32)
    src = np.zeros((C, 3), np.float32)
    dst = rng.uniform(0, 2, (V, 3)).astype(np.float32)
    offs = rng.uniform(0, 20, (S, V)).astype(np.float32)
    w = rng.uniform(0, 1, (S, V)).astype(np.float32)
    q1 = oracle.das_f64(x, src, dst, offs, w, q1=True)
    same = oracle.das_f64(x, src, dst, np.repeat(offs[:1], S, 0), np.repeat(w[:1], S, 0))
    np.testing.assert_allclose(q1, same, rtol=1e-12)
    # with a batch dim the quirk does not apply
    q1b = oracle.das_f64(x[None], src, dst, offs, w, q1=True)
    np.testing.assert_allclose(q1b[0], oracle.das_f64(x, src, dst, offs, w), rtol=1e-12)


def test_f32_loop_matches_f64(rng):
    C, S, N, V = 8, 3, 256, 50
    x = rng.standard_normal((1, C, S, N)).astype(np.float32)
    src = rng.uniform(-4, 4, (C, 3)).astype(np.float32)
    dst = (rng.uniform(-4, 4, (V, 3)) + [0, 0, 60]).astype(np.float32)
    offs = rng.uniform(0, 100, (S, V)).astype(np.float32)
    w = rng.uniform(0, 1, (S, V)).astype(np.float32)
    ref = oracle.das_f64(x, src, dst, offs, w)
    f32 = oracle.das_f32(x, src, dst, offs, w)
    assert oracle.rel_l2(f32, ref) < 1e-4


def test_torch_reference_matches_oracle(rng):
    C, S, N = 3, 4, 40
    x = rng.standard_normal((2, C, S, N)).astype(np.float32)
    src = rng.uniform(-2, 2, (C, 3)).astype(np.float32)
    dst = (rng.uniform(-2, 2, (5, 3)) + [0, 0, 9]).astype(np.float32)
    offs = rng.uniform(-5, 30, (S, 5)).astype(np.float32)
    w = rng.uniform(0, 1, (S, 5)).astype(np.float32)
    ref = oracle.das_f64(x, src, dst, offs, w)
    got = das_ref(*(torch.from_numpy(a) for a in (x, src, dst, offs, w))).numpy()
    np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-9)
    idx = rng.integers(0, S, (3, 5)).astype(np.int32)
    ref_s = oracle.das_f64(x, src, dst, offs[:3], w[:3], sparse_indices=idx)
    got_s = das_ref(*(torch.from_numpy(a) for a in (x, src, dst, offs[:3], w[:3])),
                    sparse_indices=torch.from_numpy(idx)).numpy()
    np.testing.assert_allclose(got_s, ref_s, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("path", sorted(GOLDEN.glob("ref_*.npz")), ids=lambda p: p.stem)
def test_oracle_matches_reference_outputs(path):
    """Outputs of the reference library (run on a B200) against the oracle."""
    z = np.load(path, allow_pickle=False)
    kw = {}
    for k in ("srcdir", "sparse_indices"):
        if k in z.files:
            kw[k] = z[k]
    wavenum = float(z["wavenum"]) if "wavenum" in z.files else 0.0
    q1 = bool(z["q1"]) if "q1" in z.files else False
    if "beta" in z.files:   # out = beta * out_init + sum
        kw["beta"] = complex(z["beta"])
        kw["out"] = z["out_init"]
    ref_out = z["out"]
    got = oracle.das_f64(z["x"], z["srcpos"], z["dstpos"], z["offsets"], z["weights"], wavenum=wavenum,
                         q1=q1, **kw)
    tol = float(z["tol"])
    assert oracle.rel_l2(ref_out, got) < tol


# ---------------------------------------------------------------- rank filter

from oracle import truncate_rank as tro  # noqa: E402


@pytest.mark.parametrize("shape", [(16, 64), (64, 16), (32, 32), (8, 4, 16)])
@pytest.mark.parametrize("cplx", [False, True])
def test_rank_filter_oracle_matches_svd(shape, cplx):
    # the eigen route of the reference equals the SVD reconstruction its tests
    # use (test_truncate_rank.py:38-43) on spectra with a gap at the cut
    m = shape[0]
    n = int(np.prod(shape[1:]))
    x = tro.clutter_ensemble(m, n, rank=3, complex_=cplx, seed=1).reshape(shape)
    for start, stop in [(0, 3), (3, None), (1, 3), (0, min(m, n))]:
        a = tro.truncate_rank_f64(x, start, stop)
        b = tro.svd_filter_f64(x, start, stop)
        assert a.shape == x.shape
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-9 * np.abs(x).max())


def test_rank_filter_oracle_keep_all_is_identity(rng):
    # reference test_truncate_rank.py:46-50
    x = rng.standard_normal((8, 32))
    np.testing.assert_allclose(tro.truncate_rank_f64(x, 0, 8), x, atol=1e-12)


def test_rank_filter_oracle_projection_properties(rng):
    # idempotent, and the kept and dropped parts add up to x
    x = rng.standard_normal((12, 40)) + 1j * rng.standard_normal((12, 40))
    a = tro.truncate_rank_f64(x, 2, 7)
    np.testing.assert_allclose(tro.truncate_rank_f64(a, 0, 5), a, atol=1e-10)
    parts = tro.truncate_rank_f64(x, 0, 2) + a + tro.truncate_rank_f64(x, 7, 12)
    np.testing.assert_allclose(parts, x, atol=1e-10)
