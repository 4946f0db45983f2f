"""The eigensolver's Cholesky-QR kernel (chol.cu, one cluster launch: the
factor G = R^H R and its inverse R^-1) through the C-ABI, against LAPACK's
potrf and a triangular inverse in FP64.

Sizes cover one tile, tile edges (31/32/33 real, 15/16/17 complex), ragged
last tiles and every cluster size up to 16 CTAs, including the 540-column
subspace blocks of the Si64 solve.  Bars: the inverse factor within 1e-11
relative of LAPACK's (the Gram matrices here have condition numbers near
1e3), R^-H G R^-1 = I to 1e-11, exact zeros below the diagonal.  A matrix
whose leading minor of order p + 1 is not positive definite returns
info = p + 1, as potrf counts."""

import numpy as np
import pytest
import scipy.linalg as sla

from pwgpu.lib import dense_cholesky_inverse

pytestmark = pytest.mark.gpu


def gram(q, cpx, seed):
    rng = np.random.default_rng(seed)
    n = 3 * q + 8
    y = rng.standard_normal((n, q))
    if cpx:
        y = y + 1j * rng.standard_normal((n, q))
    y *= np.logspace(0, 1.5, q)[None, :]  # column scales 1 .. 30
    g = y.conj().T @ y
    return 0.5 * (g + g.conj().T)


def check(q, cpx, seed=7):
    g = gram(q, cpx, seed + q)
    ri, rd, info, ctas = dense_cholesky_inverse(g)
    assert info == 0
    r_ref = sla.cholesky(g, lower=False)
    ri_ref = sla.solve_triangular(r_ref, np.eye(q), lower=False)
    assert np.max(np.abs(ri - ri_ref)) <= 1e-11 * np.max(np.abs(ri_ref))
    assert np.max(np.abs(rd - np.real(np.diag(r_ref)))) <= 1e-12 * np.max(np.abs(rd))
    assert np.all(ri[np.tril_indices(q, -1)] == 0)
    eye = ri.conj().T @ g @ ri
    assert np.max(np.abs(eye - np.eye(q))) < 1e-11
    return ctas


@pytest.mark.parametrize("q", [1, 5, 31, 32, 33, 64, 80, 100, 180, 181, 255, 360, 540])
def test_real(q):
    check(q, False)


@pytest.mark.parametrize("q", [1, 7, 15, 16, 17, 48, 100, 180, 361])
def test_complex(q):
    check(q, True)


def test_cluster_sizes_reach_sixteen():
    assert check(540, False) == 16
    assert check(64, False) in (2, 4)


@pytest.mark.parametrize("cpx", [False, True])
@pytest.mark.parametrize("q,p", [(1, 0), (40, 0), (40, 17), (100, 31), (100, 32), (200, 150), (300, 299)])
def test_failed_pivot_reports_potrf_info(q, p, cpx):
    g = gram(q, cpx, 11 + q + p)
    # make the Schur complement of the leading p x p block negative at row p
    r = sla.cholesky(g, lower=False)
    g[p, p] -= (r[p, p] ** 2) * 1.5
    _, _, info, _ = dense_cholesky_inverse(g)
    fn = sla.lapack.zpotrf if cpx else sla.lapack.dpotrf
    _, ref_info = fn(g, lower=0)
    assert ref_info == p + 1
    assert info == p + 1


def test_identity_and_diagonal():
    for q in (3, 64, 97):
        d = np.linspace(0.5, 4.0, q)
        ri, rd, info, _ = dense_cholesky_inverse(np.diag(d))
        assert info == 0
        assert np.allclose(rd, np.sqrt(d), rtol=1e-15, atol=0)
        assert np.allclose(ri, np.diag(1.0 / np.sqrt(d)), rtol=1e-15, atol=0)
