"""The reference's mixer unit tests restated on the oracle's mixers, which the
device mixers (pwgpu_mix, the SCF loop) are checked against step by step on
the GPU:

* scf/mixing/anderson.rs:416-572 (linear first step, Kerker suppression of
  G = 0, multi-step Anderson + Kerker, the small and large q_TF limits, plain
  mixing independent of the FFT);
* scf/mixing/broyden.rs:279-390 (linear first step, finite multi-step with
  and without Kerker, convergence on a fixed-point problem, history
  trimming);
* scf/mixing/kerker.rs:56-100 (q_TF range, real preconditioned residual,
  high-G pass-through) and scf/mixing/linalg.rs:59-64 (the 2x2 solve).

As in the reference, the "|G|^2" arrays of these tests are synthetic values
indexed by grid point, and the Kerker weights are P = G^2 / (G^2 + q_TF^2)
with P = 0 at G = 0 (kerker.rs:18-35).
"""

import numpy as np
import pytest

from oracle import pwdft_oracle as O

# the singular-pivot fallback of the small solve is exercised on purpose
pytestmark = pytest.mark.filterwarnings("ignore::scipy.linalg.LinAlgWarning")


def kerker_weights(g2, q_tf):
    g2 = np.asarray(g2, dtype=float)
    return np.where(g2 == 0.0, 0.0, g2 / (g2 + q_tf * q_tf))


def g2_line(n, step=1.0):
    return np.array([0.0 if i == 0 else 1.0 + step * i for i in range(n)])


def sin_density(n, amp, freq=1.0):
    return 1.0 + amp * np.sin(freq * np.arange(n, dtype=float))


# --- anderson.rs ------------------------------------------------------------

def test_anderson_first_step_is_linear():
    m = O.AndersonMixer(0.3, 4, (2, 2, 2))
    out = m.mix(np.ones(8), np.full(8, 2.0))
    assert np.max(np.abs(out - 1.3)) < 1e-10


def test_kerker_suppresses_uniform_residual():
    dims = (4, 4, 4)
    m = O.AndersonMixer(0.3, 4, dims, kerker_weights(g2_line(64), 1.0))
    out = m.mix(np.ones(64), np.full(64, 2.0))
    assert np.max(np.abs(out - 1.0)) < 0.1


def test_anderson_kerker_three_steps_finite():
    dims = (4, 4, 4)
    m = O.AndersonMixer(0.3, 4, dims, kerker_weights(g2_line(64, 0.5), 1.0))
    rho = sin_density(64, 0.01)
    target = 1.0 + 0.02 * np.cos(np.arange(64, dtype=float))
    for _ in range(3):
        rho = m.mix(rho, target)
        assert np.all(np.isfinite(rho))


def test_kerker_small_q_tf_approaches_plain():
    dims = (4, 4, 4)
    rho_in = sin_density(64, 0.1, 0.3)
    rho_out = sin_density(64, 0.2, 0.3)
    plain = O.AndersonMixer(0.3, 4, dims).mix(rho_in, rho_out)
    kerk = O.AndersonMixer(0.3, 4, dims, kerker_weights(g2_line(64), 0.001)).mix(rho_in, rho_out)
    assert np.max(np.abs(plain - kerk)) < 0.01


def test_kerker_large_q_tf_suppresses_mixing():
    dims = (4, 4, 4)
    m = O.AndersonMixer(0.3, 4, dims, kerker_weights(g2_line(64), 1000.0))
    out = m.mix(np.ones(64), np.full(64, 2.0))
    assert np.max(np.abs(out - 1.0)) < 0.01


def test_plain_mixing_is_deterministic():
    a = O.AndersonMixer(0.3, 4, (2, 2, 2)).mix(np.ones(8), np.full(8, 2.0))
    b = O.AndersonMixer(0.3, 4, (2, 2, 2)).mix(np.ones(8), np.full(8, 2.0))
    assert np.max(np.abs(a - b)) < 1e-15


# --- broyden.rs -------------------------------------------------------------

def test_broyden_first_step_is_linear():
    out = O.BroydenMixer(0.3, 4, (2, 2, 2)).mix(np.ones(8), np.full(8, 2.0))
    assert np.max(np.abs(out - 1.3)) < 1e-10


def test_broyden_five_steps_finite_with_and_without_kerker():
    dims = (4, 4, 4)
    target = 1.0 + 0.02 * np.cos(np.arange(64, dtype=float))
    for kw in (None, kerker_weights(g2_line(64), 1.0)):
        m = O.BroydenMixer(0.3, 4, dims, kw)
        rho = sin_density(64, 0.01)
        for _ in range(5):
            rho = m.mix(rho, target)
            assert np.all(np.isfinite(rho))


def test_broyden_converges_on_fixed_point():
    dims = (4, 4, 4)
    m = O.BroydenMixer(0.5, 8, dims)
    target = sin_density(64, 0.1, 0.3)
    rho = np.ones(64)
    err0 = np.linalg.norm(rho - target)
    for _ in range(20):
        rho = m.mix(rho, target)
    assert np.linalg.norm(rho - target) < 0.01 * err0


def test_broyden_history_is_trimmed():
    m = O.BroydenMixer(0.3, 2, (2, 2, 2))
    rho = np.ones(8)
    for it in range(10):
        rho = m.mix(rho, rho + 0.1 * it)
        assert len(m.df) <= 2 and len(m.dv) <= 2


# --- kerker.rs, linalg.rs ---------------------------------------------------

def test_auto_q_tf_in_range():
    q = np.sqrt(O.auto_q_tf_squared(8.0, 40.0))
    assert 0.5 < q < 5.0


def test_preconditioned_residual_is_real_and_finite():
    dims = (4, 4, 4)
    w = np.where(np.arange(64) == 0, 0.0, 0.5)
    res = np.sin(0.1 * np.arange(64, dtype=float))
    rg = O.fft3(res.astype(np.complex128), dims) * w
    back = O.ifft3(rg, dims) / res.size
    assert np.all(np.isfinite(back.real))
    # a real residual filtered by weights that depend on the grid index only
    # through |G| stays real only when w(G) = w(-G); this synthetic w does
    assert np.max(np.abs(back.imag)) < 1e-12


def test_kerker_weights_near_one_at_high_g():
    w = kerker_weights(100.0 + np.arange(64, dtype=float), 1.0)
    assert np.all(w > 0.99)


def test_solve_small_two_by_two():
    x = O.solve_small(np.array([[2.0, 1.0], [1.0, 3.0]]), np.array([5.0, 7.0]))
    assert abs(x[0] - 1.6) < 1e-10 and abs(x[1] - 1.8) < 1e-10


def test_solve_small_singular_fallback():
    """linalg.rs:24-50: a pivot below 1e-15 returns the uniform 1/(n+1)."""
    x = O.solve_small(np.zeros((3, 3)), np.ones(3))
    assert np.allclose(x, 0.25)
