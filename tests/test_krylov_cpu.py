"""The MG solver's outer loop restated in numpy: flexible (Polak-Ribiere) CG
in the Chronopoulos-Gear form, as k_pcg_mg runs it.

Each iteration forms w = A z, gamma = (r, z), delta = (z, w) and
zeta = (z, s_old) in one pass, then beta = -alpha_old zeta / gamma_old,
(p, A p) = delta + 2 beta zeta + beta^2 (p, A p)_old, alpha = gamma / (p, A p),
p = z + beta p, s = w + beta s, x += alpha p, r -= alpha s.  The tests check
that the recurrences for (p, A p) and s = A p hold at every iteration, that a
non-symmetric preconditioner (one forward Gauss-Seidel sweep; the
over-relaxed V-cycle is slightly non-symmetric too) still converges where
the textbook Fletcher-Reeves PCG stalls, and that with a symmetric one the
iterates follow the textbook PCG.
"""
import numpy as np


def _poisson(n):
    """5-point Dirichlet Laplacian on an n x n grid (SPD)."""
    m = n * n
    A = np.zeros((m, m))
    for j in range(n):
        for i in range(n):
            c = i + j * n
            A[c, c] = 4.0
            for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1)):
                a, b = i + di, j + dj
                if 0 <= a < n and 0 <= b < n:
                    A[c, a + b * n] = -1.0
    return A


def _flexible_cg(A, b, apply_m, tol=1e-10, maxit=500, check=True):
    x = np.zeros_like(b)
    r = b.copy()
    p = np.zeros_like(b)
    s = np.zeros_like(b)
    gam_old = alpha_old = den_old = 1.0
    it = 0
    while np.linalg.norm(r) > tol * np.linalg.norm(b) and it < maxit:
        z = apply_m(r)
        w = A @ z
        gam, delta, zeta = r @ z, z @ w, z @ s
        beta = -alpha_old * zeta / gam_old if it > 0 else 0.0
        den = delta + beta * (2.0 * zeta + beta * den_old) if it > 0 else delta
        alpha = gam / den
        p = z + beta * p if it > 0 else z
        s = w + beta * s if it > 0 else w
        if check:
            assert np.allclose(s, A @ p, rtol=1e-9, atol=1e-12)
            assert abs(den - p @ (A @ p)) <= 1e-9 * abs(den)
        x += alpha * p
        r -= alpha * s
        gam_old, alpha_old, den_old = gam, alpha, den
        it += 1
    return x, it


def _textbook_pcg(A, b, apply_m, tol=1e-10, maxit=500):
    x = np.zeros_like(b)
    r = b.copy()
    z = apply_m(r)
    p = z.copy()
    rz = r @ z
    it = 0
    while np.linalg.norm(r) > tol * np.linalg.norm(b) and it < maxit:
        q = A @ p
        alpha = rz / (p @ q)
        x += alpha * p
        r -= alpha * q
        z = apply_m(r)
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
        it += 1
    return x, it


def test_recurrences_hold_and_a_nonsymmetric_preconditioner_converges():
    """With one forward Gauss-Seidel sweep as the preconditioner (M^-1 = L^-1,
    not symmetric) the flexible loop converges (118 iterations here), where the
    textbook Fletcher-Reeves PCG stalls (relative residual 0.2 after 2000)."""
    A = _poisson(12)
    b = np.random.default_rng(0).standard_normal(A.shape[0])
    L = np.tril(A)
    m = lambda r: np.linalg.solve(L, r)
    x, it = _flexible_cg(A, b, m)
    assert np.linalg.norm(b - A @ x) <= 1e-10 * np.linalg.norm(b) and it < 200
    xt, itt = _textbook_pcg(A, b, m, maxit=400)
    assert itt == 400 and np.linalg.norm(b - A @ xt) > 1e-3 * np.linalg.norm(b)


def test_symmetric_preconditioner_matches_textbook_pcg():
    A = _poisson(10)
    b = np.random.default_rng(1).standard_normal(A.shape[0])
    m = lambda r: r / np.diag(A)
    x1, it1 = _flexible_cg(A, b, m)
    x2, it2 = _textbook_pcg(A, b, m)
    assert abs(it1 - it2) <= 1
    assert np.allclose(x1, x2, rtol=1e-8, atol=1e-10)
