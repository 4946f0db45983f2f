"""The cluster eigensolver of the Rayleigh-Ritz step (pwgpu_dense_eigh)
against LAPACK (numpy.linalg.eigh), as the reference's own dense solver
tests do (eigensolver/dense.rs:272-358: eigenvalues exact, vectors through
their residuals and orthonormality, since signs and phases are arbitrary).

Bars, relative to ||A||: eigenvalues 1e-12, residual ||A z - w z|| 1e-12,
orthonormality |Z^H Z - I| 1e-12.  Cases: random real symmetric and
complex Hermitian matrices over every cluster size the solver picks
(m = 1 .. 544), spectra with exactly repeated and nearly repeated
eigenvalues, already-diagonal and block-diagonal matrices (every reflector
the identity), and the block structure of a LOBPCG subspace matrix
[[diag(lambda), Z^H], [Z, G]].
"""

import numpy as np
import pytest

from conftest import rng
from pwgpu.lib import dense_eigh

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _sym(g, m, cpx):
    a = g.standard_normal((m, m))
    if cpx:
        a = a + 1j * g.standard_normal((m, m))
    return 0.5 * (a + a.conj().T)


def _with_spectrum(g, lam, cpx):
    m = len(lam)
    a = g.standard_normal((m, m)) + (1j * g.standard_normal((m, m)) if cpx else 0.0)
    q, _ = np.linalg.qr(a)
    return (q * lam) @ q.conj().T


def _check(a, nev):
    w, z, nc = dense_eigh(a, nev)
    ref = np.linalg.eigvalsh(a)[:nev]
    scale = max(np.max(np.abs(ref)), np.linalg.norm(a, 2), 1e-300)
    assert np.max(np.abs(w - ref)) <= TOL * scale, f"eigenvalues: {np.max(np.abs(w - ref)) / scale:.2e}"
    res = np.linalg.norm(a @ z - z * w, axis=0)
    assert np.max(res) <= TOL * scale * 10, f"residual: {np.max(res) / scale:.2e}"
    orth = np.max(np.abs(z.conj().T @ z - np.eye(nev)))
    assert orth <= TOL * 10, f"orthonormality: {orth:.2e}"
    return nc


@pytest.mark.parametrize("m", [1, 2, 3, 17, 64, 100, 160, 161, 180, 270, 360, 451, 540, 544])
def test_random_real_symmetric(m):
    g = rng(m)
    a = _sym(g, m, False)
    _check(a, m)
    if m > 3:
        _check(a, m // 3)


@pytest.mark.parametrize("m", [2, 5, 81, 113, 200, 300, 400])
def test_random_complex_hermitian(m):
    g = rng(1000 + m)
    a = _sym(g, m, True)
    _check(a, m)
    _check(a, max(1, m // 3))


@pytest.mark.parametrize("cpx", [False, True])
def test_repeated_and_close_eigenvalues(cpx):
    g = rng(7)
    m = 240
    lam = np.sort(g.uniform(-10.0, 300.0, m))
    lam[10:14] = lam[10]               # four-fold degenerate
    lam[40:43] = lam[40] + np.array([0.0, 1e-9, 2e-9])   # nearly degenerate triple
    lam[80:82] = lam[80] + np.array([0.0, 1e-13])
    lam = np.sort(lam)
    a = _with_spectrum(g, lam, cpx)
    _check(a, m)
    _check(a, 90)


@pytest.mark.parametrize("m", [1, 50, 200, 540])
def test_diagonal_and_block_diagonal(m):
    g = rng(11)
    d = np.diag(g.uniform(-5, 5, m))
    _check(d, m)
    if m >= 50:
        b = d.copy()
        h = m // 2
        b[:h, :h] = _sym(g, h, False)
        _check(b, m // 2)


@pytest.mark.parametrize("m,nd", [(540, 180), (180, 60), (300, 180)])
def test_lobpcg_block_structure(m, nd):
    """[[diag(lambda), Z^T], [Z, G]] with small couplings, as a late LOBPCG step produces."""
    g = rng(m + nd)
    q = m - nd
    a = np.zeros((m, m))
    a[:nd, :nd] = np.diag(np.sort(g.uniform(-6.0, 8.0, nd)))
    zc = 1e-3 * g.standard_normal((q, nd))
    a[nd:, :nd] = zc
    a[:nd, nd:] = zc.T
    a[nd:, nd:] = _sym(g, q, False) * 5.0 + np.diag(g.uniform(0.0, 400.0, q))
    _check(a, nd)
