"""The general (non-symmetric) eigen-solve of the Davidson step against
LAPACK's dgeev (numpy.linalg.eig), which the reference calls on the Ritz
matrix (src/lib_cc/mod_davidson.f90:185-219): the same eigenvalues, and
eigenvectors of unit norm with their largest component real (equal to
dgeev's up to a sign for simple eigenvalues)."""
import numpy as np
import pytest

from cpsd_b200 import api

pytestmark = pytest.mark.gpu


def _check(A, simple=True):
    n = A.shape[0]
    wr, wi, V, sweeps = api.geev(A)
    assert sweeps >= 0
    scale = max(np.abs(A).max(), 1e-300)
    lam = np.linalg.eig(A).eigenvalues
    mine = np.sort_complex(wr + 1j * wi)
    ref = np.sort_complex(lam)
    np.testing.assert_allclose(mine, ref, rtol=0, atol=1e-11 * scale * max(1, n))
    # pairs in dgeev order: positive imaginary part first, equal real parts
    k = 0
    while k < n:
        if wi[k] != 0.0:
            assert wi[k] > 0 and wi[k + 1] == -wi[k] and wr[k + 1] == wr[k]
            # the real and imaginary parts (each of unit norm, as the
            # reference keeps them) span an invariant plane of A whose
            # eigenvalues are the pair
            P = V[:, k:k + 2]
            assert abs(np.linalg.norm(P[:, 0]) - 1) < 1e-12 and abs(np.linalg.norm(P[:, 1]) - 1) < 1e-12
            M = np.linalg.lstsq(P, A @ P, rcond=None)[0]
            np.testing.assert_allclose(A @ P, P @ M, rtol=0, atol=1e-10 * scale * n)
            mu = np.sort_complex(np.linalg.eigvals(M))
            np.testing.assert_allclose(mu, np.sort_complex([wr[k] - 1j * wi[k], wr[k] + 1j * wi[k]]), atol=1e-9 * scale)
            k += 2
        else:
            v = V[:, k]
            assert abs(np.linalg.norm(v) - 1.0) < 1e-12
            np.testing.assert_allclose(A @ v, wr[k] * v, rtol=0, atol=1e-11 * scale * n)
            k += 1
    if simple:
        # every eigenvector equals dgeev's up to a sign (the reference then
        # normalises the real and imaginary parts it keeps separately)
        w, VL = np.linalg.eig(A)
        for k in range(n):
            if wi[k] < 0:
                continue
            j = int(np.argmin(np.abs(w - (wr[k] + 1j * wi[k]))))
            v = VL[:, j]
            if wi[k] > 0:
                # "largest component real" fixes the phase only when one
                # component is clearly the largest
                m2 = np.sort(np.abs(v) ** 2)
                if n > 1 and m2[-1] - m2[-2] < 1e-8 * m2[-1]:
                    continue
                ref = v / np.linalg.norm(v)
                c_re = ref.real / np.linalg.norm(ref.real)
                c_im = ref.imag / np.linalg.norm(ref.imag)
                for got, want in ((V[:, k], c_re), (V[:, k + 1], c_im)):
                    s = np.sign(np.dot(got, want))
                    np.testing.assert_allclose(s * got, want, rtol=0, atol=1e-9)
            else:
                v = v.real
                s = np.sign(np.dot(V[:, k], v))
                np.testing.assert_allclose(s * V[:, k], v, rtol=0, atol=1e-9)


@pytest.mark.parametrize("n", [1, 2, 3, 4, 7, 12, 20, 32])
def test_random_general(n):
    rng = np.random.default_rng(100 + n)
    _check(rng.standard_normal((n, n)))


@pytest.mark.parametrize("n", [2, 5, 20, 32])
def test_random_symmetric(n):
    rng = np.random.default_rng(200 + n)
    A = rng.standard_normal((n, n))
    A = A + A.T
    wr, wi, V, _ = api.geev(A)
    assert np.all(wi == 0.0)
    np.testing.assert_allclose(np.sort(wr), np.linalg.eigvalsh(A), rtol=0, atol=1e-12 * n)
    _check(A)


def test_near_symmetric_ritz_like():
    """A Ritz matrix of a slightly non-symmetric operator: real, close
    eigenvalues, the shape the Davidson step sees."""
    rng = np.random.default_rng(7)
    n = 20
    Q = np.linalg.qr(rng.standard_normal((n, n)))[0]
    A = Q @ np.diag(np.linspace(0.3, 2.0, n)) @ Q.T + 1e-3 * rng.standard_normal((n, n))
    _check(A)


def test_structured():
    # upper triangular (already Schur), rotation blocks (complex pairs),
    # an unreduced Hessenberg companion matrix, a block-diagonal matrix
    rng = np.random.default_rng(3)
    T = np.triu(rng.standard_normal((9, 9)))
    _check(T)
    R = np.zeros((6, 6))
    for k, (a, b) in enumerate([(0.5, 1.0), (-0.2, 0.3), (1.5, 2.0)]):
        R[2 * k:2 * k + 2, 2 * k:2 * k + 2] = [[a, -b], [b, a]]
    R += np.triu(0.1 * rng.standard_normal((6, 6)), 2)
    _check(R)
    c = rng.standard_normal(8)
    C = np.diag(np.ones(7), -1)
    C[:, -1] = -c
    _check(C)
    B = np.zeros((10, 10))
    B[:5, :5] = rng.standard_normal((5, 5))
    B[5:, 5:] = rng.standard_normal((5, 5))
    _check(B)


def test_repeated_eigenvalues():
    # a diagonal matrix with repeated values and the zero matrix: the
    # eigenvalues, with eigenvectors checked through the residual only
    D = np.diag([1.0, 2.0, 2.0, 3.0, 1.0])
    _check(D, simple=False)
    _check(np.zeros((4, 4)), simple=False)
