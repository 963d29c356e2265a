"""The row interchanges of the integrator's LU, on the CPU.

LINPACK's dgefa/dgesl (dgefa.f90:60-117, dgesl.f90:71-131) apply each row
interchange to the right-hand side between the columns of the forward sweep.
The device code (chem_bdf.cuh, dgefa/dgesl) instead swaps the multipliers of
earlier columns along with their rows, as LAPACK's getrf stores them, and
permutes the right-hand side once before an interchange-free sweep.  Both
perform the same floating-point operations on the same values in the same
order, so the solutions agree bit for bit; this restates both forms in plain
Python floats and checks that on random, badly scaled and nearly diagonal
systems of the sizes the kernels use."""
import numpy as np
import pytest


def _factor(A, lapack_rows):
    n = A.shape[0]
    a = [list(map(float, A[:, j])) for j in range(n)]  # a[j][i] = A[i, j]
    ipvt, perm = [0] * n, list(range(n))
    for k in range(n - 1):
        l, dmax = k, abs(a[k][k])
        for i in range(k + 1, n):
            if abs(a[k][i]) > dmax:
                l, dmax = i, abs(a[k][i])
        ipvt[k] = l
        if a[k][l] == 0.0:
            continue
        if l != k:
            a[k][l], a[k][k] = a[k][k], a[k][l]
            if lapack_rows:
                for j in range(k):
                    a[j][l], a[j][k] = a[j][k], a[j][l]
                perm[k], perm[l] = perm[l], perm[k]
        t = -1.0 / a[k][k]
        for i in range(k + 1, n):
            a[k][i] = t * a[k][i]
        for j in range(k + 1, n):
            tj = a[j][l]
            if l != k:
                a[j][l], a[j][k] = a[j][k], tj
            if tj != 0.0:
                for i in range(k + 1, n):
                    a[j][i] = a[j][i] + tj * a[k][i]
    ipvt[n - 1] = n - 1
    return a, ipvt, perm


def _back(a, b):
    n = len(b)
    for k in range(n - 1, -1, -1):
        b[k] = b[k] / a[k][k]
        t = -b[k]
        if t != 0.0:
            for i in range(k):
                b[i] = b[i] + t * a[k][i]
    return b


def solve_linpack(A, rhs):
    a, ipvt, _ = _factor(A, lapack_rows=False)
    b = list(map(float, rhs))
    n = len(b)
    for k in range(n - 1):
        l = ipvt[k]
        t = b[l]
        if l != k:
            b[l], b[k] = b[k], t
        if t != 0.0:
            for i in range(k + 1, n):
                b[i] = b[i] + t * a[k][i]
    return _back(a, b)


def solve_permuted(A, rhs):
    a, _, perm = _factor(A, lapack_rows=True)
    b = [float(rhs[perm[i]]) for i in range(len(rhs))]
    n = len(b)
    for k in range(n - 1):
        t = b[k]
        if t != 0.0:
            for i in range(k + 1, n):
                b[i] = b[i] + t * a[k][i]
    return _back(a, b)


@pytest.mark.parametrize("n", [8, 9, 13, 15, 17])
def test_permuted_solve_gives_linpack_bits(n):
    rng = np.random.default_rng(n)
    for trial in range(150):
        if trial % 3 == 0:  # an iteration matrix I - h l0 J with a small h
            A = np.eye(n) + 1e-3 * rng.standard_normal((n, n)) * (rng.random((n, n)) < 0.3)
        else:  # entries over six decades: many interchanges
            A = rng.standard_normal((n, n)) * 10.0 ** rng.uniform(-3, 3, (n, n))
        rhs = rng.standard_normal(n)
        x1, x2 = solve_linpack(A, rhs), solve_permuted(A, rhs)
        assert x1 == x2, (n, trial)
        assert np.allclose(A @ np.array(x1), rhs, rtol=1e-6, atol=1e-6 * np.abs(rhs).max())
