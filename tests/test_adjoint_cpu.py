"""Host pieces of the differentiation form that need no GPU: eigen-perturbation tangents
and the eigenvector-rotation gradient, against finite differences."""
import numpy as np

from taco_b200.adjoint import eig_tangent, grad_U_from_rotated
from taco_b200.inputs import SX, SZ, System


def test_eig_tangent_matches_fd():
    rng = np.random.default_rng(1)
    X = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
    H = X + X.conj().T
    dH = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
    dH = dH + dH.conj().T
    s = System(H, [])
    dlam, dU = eig_tangent(s.U, s.eps, dH)
    h = 1e-6
    sp, sm = System(H + h * dH, []), System(H - h * dH, [])
    assert np.allclose((sp.eps - sm.eps) / (2 * h), dlam, atol=1e-8)
    # a phase-invariant function of U: |U|^2 and U diag(lam) U^H
    f = lambda S: np.abs(S.U) ** 2
    fd = (f(sp) - f(sm)) / (2 * h)
    an = 2 * np.real(np.conj(s.U) * dU)
    assert np.allclose(fd, an, atol=1e-7)


def test_rotation_gradient_matches_fd():
    rng = np.random.default_rng(2)
    U = np.linalg.qr(rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3)))[0]
    A = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
    W = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
    loss = lambda V: float(np.real(np.sum(np.conj(W) * (V.conj().T @ A @ V))))
    GU = grad_U_from_rotated(A, W, U)
    dU = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
    h = 1e-6
    fd = (loss(U + h * dU) - loss(U - h * dU)) / (2 * h)
    assert abs(float(np.real(np.sum(np.conj(GU) * dU))) - fd) <= 1e-7


def test_spin_boson_buckets_record_representative_pairs():
    s = System(0.5 * SZ + 0.3 * SX, [SZ])
    for b, (m, n) in enumerate(s.rep_pairs):
        assert abs(s.eps[m] - s.eps[n] - s.omegas[b]) <= 1e-12
