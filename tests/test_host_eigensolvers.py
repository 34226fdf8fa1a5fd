"""The library's host eigensolvers on the CPU, against numpy's dense eigensolver.

The Lanczos loops diagonalise their tridiagonal (or, for block Lanczos, band) matrices on the host,
in FP64, as RealTriDiagonalSymmetricMatrix::Diagonalize (RealTriDiagonalSymmetricMatrix.cc:687-760)
and RealBandDiagonalSymmetricMatrix::Tridiagonalize (RealBandDiagonalSymmetricMatrix.cc:847) do in
the reference.  These solvers are internal C++ functions of libdiagham_b200 (namespace dh), reached
here by their exported Itanium C++ ABI symbol names; no GPU is involved.

- tridiagonal_eigen: implicit QL, all eigenvalues and eigenvectors.
- tridiagonal_lowest: the m lowest eigenvalues by Sturm bisection.
- tridiagonal_lowest_below: the lowest eigenvalue of T_k given that of its leading block T_{k-1}
  (an upper bound by interlacing), by safeguarded Newton steps; the batched engine's per-step
  convergence test at block size 1.
- symmetric_eigen: Householder tridiagonalisation then QL, the dense fallback of the refinement.
- band_eigenvalues / band_inverse_iteration: the block Lanczos band matrix's eigenvalues and the
  Ritz vector of the lowest one.
"""
import ctypes

import numpy as np
import pytest

D = ctypes.POINTER(ctypes.c_double)

SYMBOLS = {
    "tridiagonal_eigen": ("_ZN2dh17tridiagonal_eigenEiPKdS1_PdS2_", [ctypes.c_int, D, D, D, D]),
    "tridiagonal_lowest": ("_ZN2dh18tridiagonal_lowestEiPKdS1_iPd", [ctypes.c_int, D, D, ctypes.c_int, D]),
    "tridiagonal_lowest_below": ("_ZN2dh24tridiagonal_lowest_belowEiPKdS1_dPd",
                                 [ctypes.c_int, D, D, ctypes.c_double, D]),
    "symmetric_eigen": ("_ZN2dh15symmetric_eigenEiPdS0_S0_", [ctypes.c_int, D, D, D]),
    "band_eigenvalues": ("_ZN2dh16band_eigenvaluesEiiPdS0_", [ctypes.c_int, ctypes.c_int, D, D]),
    "band_inverse_iteration": ("_ZN2dh22band_inverse_iterationEiiPKddPd",
                               [ctypes.c_int, ctypes.c_int, D, ctypes.c_double, D]),
}


@pytest.fixture(scope="module")
def solvers(dh):
    lib = ctypes.CDLL(dh.library_path())
    out = {}
    for name, (sym, argtypes) in SYMBOLS.items():
        fn = getattr(lib, sym)
        fn.argtypes = argtypes
        fn.restype = ctypes.c_int
        out[name] = fn
    return out


def ptr(a):
    return a.ctypes.data_as(D)


def dense(d, e):
    return np.diag(d) + np.diag(e, 1) + np.diag(e, -1)


def tridiagonals():
    """Seeded tridiagonal matrices, including the forms that trouble eigensolvers."""
    rng = np.random.default_rng(7)
    cases = []
    for n in (1, 2, 3, 5, 17, 64, 150):
        cases.append(("random%d" % n, rng.normal(size=n), rng.uniform(0.1, 1.0, max(n - 1, 0))))
    # a Lanczos-like matrix: alphas near a value, betas decaying (converging Ritz values)
    n = 120
    cases.append(("lanczos", 25.0 + 0.3 * rng.normal(size=n), 2.0 * np.exp(-np.arange(n - 1) / 30.0)))
    # decoupled blocks: a zero coupling, the lowest eigenvalue in the later block
    d = np.concatenate([np.full(10, 2.0), np.full(10, -3.0)])
    e = np.full(19, 0.5)
    e[9] = 0.0
    cases.append(("decoupled", d, e))
    # the lowest eigenvector localised at the end (the last diagonal entry far below the rest)
    d = np.full(40, 1.0)
    d[-1] = -50.0
    cases.append(("localised_end", d, np.full(39, 1e-3)))
    # Wilkinson's W21+: pairs of nearly equal eigenvalues
    cases.append(("wilkinson21", np.abs(np.arange(-10, 11)).astype(float), np.ones(20)))
    # equal diagonal, tiny couplings: a near-degenerate cluster
    cases.append(("cluster", np.full(30, 4.0), np.full(29, 1e-9)))
    # large scale
    cases.append(("scaled", 1e6 * rng.normal(size=50), 1e6 * rng.uniform(0.1, 1.0, 49)))
    return cases


CASES = tridiagonals()


@pytest.mark.parametrize("name,d,e", CASES, ids=[c[0] for c in CASES])
def test_tridiagonal_eigen(solvers, name, d, e):
    n = d.size
    d, e = np.ascontiguousarray(d), np.ascontiguousarray(e if e.size else np.zeros(1))
    eig = np.zeros(n)
    z = np.zeros((n, n))
    assert solvers["tridiagonal_eigen"](n, ptr(d), ptr(e), ptr(eig), ptr(z)) == 0
    T = dense(d, e[:n - 1])
    ref = np.linalg.eigvalsh(T)
    scale = np.max(np.abs(ref)) + 1.0
    assert np.max(np.abs(eig - ref)) < 1e-12 * scale
    # rows of z (as stored: eigenvector i at z[i]) are orthonormal eigenvectors
    assert np.max(np.abs(z @ z.T - np.eye(n))) < 1e-11
    assert np.max(np.abs(T @ z.T - z.T * eig)) < 1e-11 * scale


@pytest.mark.parametrize("name,d,e", CASES, ids=[c[0] for c in CASES])
def test_tridiagonal_lowest(solvers, name, d, e):
    n = d.size
    d, e = np.ascontiguousarray(d), np.ascontiguousarray(e if e.size else np.zeros(1))
    m = min(n, 4)
    eig = np.zeros(m)
    assert solvers["tridiagonal_lowest"](n, ptr(d), ptr(e), m, ptr(eig)) == 0
    ref = np.linalg.eigvalsh(dense(d, e[:n - 1]))[:m]
    scale = np.max(np.abs(d)) + 2 * np.max(np.abs(e)) + 1.0
    assert np.max(np.abs(eig - ref)) < 1e-12 * scale


@pytest.mark.parametrize("name,d,e", CASES, ids=[c[0] for c in CASES])
def test_tridiagonal_lowest_below_along_a_growing_matrix(solvers, name, d, e):
    """Each leading block T_k from T_{k-1}'s lowest eigenvalue, as the engine calls it step by step."""
    n = d.size
    d, e = np.ascontiguousarray(d), np.ascontiguousarray(e if e.size else np.zeros(1))
    scale = np.max(np.abs(d)) + 2 * np.max(np.abs(e)) + 1.0
    above = d[0]
    for k in range(1, n + 1):
        out = np.zeros(1)
        assert solvers["tridiagonal_lowest_below"](k, ptr(d), ptr(e), float(above), ptr(out)) == 0
        ref = np.linalg.eigvalsh(dense(d[:k], e[:k - 1]))[0]
        assert abs(out[0] - ref) < 1e-12 * scale, (k, out[0], ref)
        above = out[0]


def test_tridiagonal_lowest_below_with_a_loose_bound(solvers):
    """A bound well above the lowest eigenvalue (every eigenvalue below it) still gives the lowest."""
    rng = np.random.default_rng(11)
    d = rng.normal(size=60)
    e = rng.uniform(0.1, 1.0, 59)
    ref = np.linalg.eigvalsh(dense(d, e))
    out = np.zeros(1)
    assert solvers["tridiagonal_lowest_below"](60, ptr(d), ptr(e), float(ref[-1] + 1.0), ptr(out)) == 0
    assert abs(out[0] - ref[0]) < 1e-12 * (np.max(np.abs(ref)) + 1.0)


@pytest.mark.parametrize("n,b", [(1, 1), (6, 2), (40, 3), (64, 4), (90, 8)])
def test_band_eigenvalues_and_ritz_vector(solvers, n, b):
    rng = np.random.default_rng(100 + n * b)
    a = np.zeros((n, n))
    for k in range(b + 1):
        v = rng.normal(size=n - k)
        a += np.diag(v, k) + (np.diag(v, -k) if k else 0)
    ref_vals, ref_vecs = np.linalg.eigh(a)
    work = np.ascontiguousarray(a.copy())
    eig = np.zeros(n)
    assert solvers["band_eigenvalues"](n, b, ptr(work), ptr(eig)) == 0
    scale = np.max(np.abs(ref_vals)) + 1.0
    assert np.max(np.abs(eig - ref_vals)) < 1e-11 * scale
    # inverse iteration at the lowest eigenvalue: the Ritz vector of the block Lanczos refinement
    a_in = np.ascontiguousarray(a)
    vec = np.zeros(n)
    assert solvers["band_inverse_iteration"](n, b, ptr(a_in), float(ref_vals[0]), ptr(vec)) == 0
    assert np.array_equal(a_in, a)  # not modified
    assert abs(np.linalg.norm(vec) - 1.0) < 1e-12
    assert np.linalg.norm(a @ vec - ref_vals[0] * vec) < 1e-9 * scale
    if n > 1 and ref_vals[1] - ref_vals[0] > 1e-6 * scale:
        assert abs(abs(vec @ ref_vecs[:, 0]) - 1.0) < 1e-9


@pytest.mark.parametrize("n", [1, 2, 3, 8, 33, 100])
def test_symmetric_eigen(solvers, n):
    rng = np.random.default_rng(300 + n)
    m = rng.normal(size=(n, n))
    a = m + m.T
    if n >= 8:
        a[:, 3] = a[3, :] = 0.0  # a zero column: a Householder step with nothing to reflect
        a[3, 3] = 0.5
    ref = np.linalg.eigvalsh(a)
    work = np.ascontiguousarray(a.copy())
    eig = np.zeros(n)
    z = np.zeros((n, n))
    assert solvers["symmetric_eigen"](n, ptr(work), ptr(eig), ptr(z)) == 0
    scale = np.max(np.abs(ref)) + 1.0
    assert np.max(np.abs(eig - ref)) < 1e-11 * scale
    # z row-major with the eigenvectors in its columns
    assert np.max(np.abs(z.T @ z - np.eye(n))) < 1e-11
    assert np.max(np.abs(a @ z - z * eig)) < 1e-10 * scale
