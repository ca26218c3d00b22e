"""Test-only checker for the rank filter (ffdas_truncate_rank).

This module is test infrastructure.  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline and reference legs use it, and only as the checker;
no product code path imports it.

truncate_rank_f64 restates the reference's algorithm in numpy float64 /
complex128 (src/truncate_rank/truncate_rank_impl.cuh):
  * x (m, n) is read as A = x when m <= n, else as A = x^T (the Gram matrix
    of the smaller side, :451-453);
  * G = A A^H / q (the reference's GEMM with alpha = 1/nrows, :51-64);
  * eigenvectors of G, eigenvalues ascending (syevd, :68-90), so singular
    rank s is eigenvector p-1-s;
  * out = V_k V_k^H A with V_k the eigenvectors of ranks start..stop-1
    (the SYRK + SYMM projection, :104-140).
svd_filter_f64 is the checker of the reference's own tests
(bindings/python/tests/test_truncate_rank.py:38-43): the thin SVD of x,
reconstructed from components start..stop-1.  The two agree wherever the
singular values of the kept window are separated from the dropped ones,
which pins the restatement (tests/test_oracle.py).
"""
from __future__ import annotations

import numpy as np


def _as_matrix(x):
    x = np.asarray(x)
    m = x.shape[0]
    return x.reshape(m, -1), m, int(np.prod(x.shape[1:]))


def truncate_rank_f64(x, start: int, stop: int | None = None) -> np.ndarray:
    """Eigen-route rank filter in float64/complex128; returns x's shape."""
    xm, m, n = _as_matrix(x)
    cplx = np.iscomplexobj(xm)
    xm = xm.astype(np.complex128 if cplx else np.float64)
    p = min(m, n)
    stop = p if stop is None else stop
    if not (0 <= start < stop <= p):
        raise ValueError("need 0 <= start < stop <= min(m, n)")
    rows = m <= n
    A = xm if rows else xm.T
    q = A.shape[1]
    G = (A @ A.conj().T) / q
    _, V = np.linalg.eigh(G)            # ascending
    Vk = V[:, p - stop:p - start]
    out_a = Vk @ (Vk.conj().T @ A)
    out = out_a if rows else out_a.T
    return out.reshape(np.asarray(x).shape)


def svd_filter_f64(x, start: int, stop: int | None = None) -> np.ndarray:
    """Thin-SVD reconstruction from components start..stop-1 (float64/complex128)."""
    xm, m, n = _as_matrix(x)
    cplx = np.iscomplexobj(xm)
    xm = xm.astype(np.complex128 if cplx else np.float64)
    stop = min(m, n) if stop is None else stop
    U, S, Vh = np.linalg.svd(xm, full_matrices=False)
    out = (U[:, start:stop] * S[start:stop]) @ Vh[start:stop, :]
    return out.reshape(np.asarray(x).shape)


def clutter_ensemble(m: int, n: int, *, rank: int = 3, blood: float = 1e-2, complex_: bool = False,
                     seed: int = 0, decay: float = 4.0) -> np.ndarray:
    """Synthetic slow-time ensemble (m frames, n voxels): a strong low-rank
    'tissue' part with well separated singular values plus weak full-rank
    'blood' noise (singular values of the tissue part fall by `decay` per
    rank).  Used to give the filter a spectrum with clear gaps: cuts at or
    below `rank` are well conditioned in FP32, cuts inside the noise are not."""
    rng = np.random.default_rng(seed)

    def draw(*shape):
        a = rng.standard_normal(shape)
        if complex_:
            a = a + 1j * rng.standard_normal(shape)
        return a

    U, _ = np.linalg.qr(draw(m, rank))
    V, _ = np.linalg.qr(draw(n, rank))
    s = np.sqrt(n) * (float(decay) ** -np.arange(rank)) * 10.0
    tissue = (U * s) @ V.conj().T
    return tissue + blood * draw(m, n)
