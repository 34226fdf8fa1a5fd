"""The single-vector Lanczos solve's host logic on the CPU: graph-batch sizes and Ritz values.

dh_lanczos_solve issues up to 16 iterations per CUDA-graph batch, then replays the reference's
convergence test (BasicLanczosAlgorithm.cc:200-224: |E_r - E_{r-1}| < precision |E_r|) row by row on
the host; iterations past the converged row are discarded.  The next batch's size comes from
dh::lanczos_batch_prediction (an internal C++ function of libdiagham_b200, reached by its exported
Itanium C++ ABI name) over the test's ratio to its threshold, sampled at each batch's end and six
rows before it.  Here the loop is replayed on the ratio sequences of Lanczos runs of the oracle's
FQHE sectors (seeded start vectors, as the GPU tests use), and the products it issues are compared
with fixed batches of 16.  Each replayed row's lowest Ritz value comes from dh::lanczos_lowest_ritz
(Newton steps from the previous row's value, QL where Newton returns that bound unchanged): the
reference's test must stop at the same row as with QL values.  No GPU is involved.
"""
import ctypes
import math

import numpy as np
import pytest

from conftest import golden

SPAN = 6      # kLanczosRateSpan
BATCH = 16    # the solve's graph batch
FIRST = 3     # rows of the driver loop's first RunLanczosAlgorithm(nev + 2) call at nev = 1


@pytest.fixture(scope="module")
def predict(dh):
    lib = ctypes.CDLL(dh.library_path())
    fn = lib._ZN2dh24lanczos_batch_predictionEiPKiPKdi
    fn.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    fn.restype = ctypes.c_int

    def call(rows, logs, graph_batch=BATCH):
        r = np.ascontiguousarray(rows, np.int32)
        g = np.ascontiguousarray(logs, np.float64)
        return fn(len(r), r.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                  g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), graph_batch)
    return call


def test_prediction_edge_cases(predict):
    assert predict([], []) == BATCH
    assert predict([20], [math.log(1e6)]) == BATCH                        # one sample: no rate
    assert predict([14, 20], [math.log(1e3), math.log(1e6)]) == BATCH     # rising ratio
    assert predict([14, 20], [math.log(1e6), math.log(0.5)]) == BATCH     # passing already
    assert predict([14, 20], [math.log(1e6), float("nan")]) == BATCH
    # one decade per row, two decades left: 0.85 * 2 rows, rounded up
    assert predict([10, 16], [math.log(1e8), math.log(1e2)]) == 2
    # slow decay: capped at the graph batch; fast decay: at least two iterations
    assert predict([10, 16], [math.log(1e7), math.log(1e6)]) == BATCH
    assert predict([10, 16], [math.log(1e60), math.log(1e1)]) == 2
    assert predict([10, 16], [math.log(1e7), math.log(1e6)], graph_batch=8) == 8
    # the rate runs from the newest sample at least six rows back (row 14: a third of a decade per
    # row, two decades left, 0.85 * 6 rows); rows 10 or 4 would give 3 or 4
    assert predict([4, 10, 14, 20], [math.log(1e9), math.log(1e9), math.log(1e4), math.log(1e2)]) == 6


def lanczos_tridiagonal(matvec, dim, v0, steps):
    v = v0 / np.linalg.norm(v0)
    v_prev = np.zeros(dim)
    b = 0.0
    alpha, beta = [], []
    for _ in range(steps):
        w = matvec(v) - b * v_prev
        a = v @ w
        w -= a * v
        alpha.append(a)
        b = np.linalg.norm(w)
        beta.append(b)
        v_prev, v = v, w / b
    return np.array(alpha), np.array(beta)


def convergence_ratios(alpha, beta, precision):
    """ratio[r] = |E_r - E_{r-1}| / (precision |E_r|), E_r the lowest eigenvalue of T_r (the first
    call compares with twice its value, as BasicLanczosAlgorithm does)."""
    out, prev = {}, None
    for r in range(2, len(alpha) + 1):
        t = np.diag(alpha[:r]) + np.diag(beta[:r - 1], 1) + np.diag(beta[:r - 1], -1)
        e = np.linalg.eigvalsh(t)[0]
        out[r] = abs(e - (2 * e if prev is None else prev)) / (precision * abs(e))
        prev = e
    return out


def replay(ratio, predict=None):
    """The solve loop's batches: (converged row, rows issued)."""
    conv = next(r for r in sorted(ratio) if r > FIRST and ratio[r] < 1.0)
    rows, batch = FIRST, BATCH
    s_rows, s_logs = [], []
    while True:
        start, end = rows, rows + batch
        if end >= conv:
            return conv, end
        rows = end
        if predict is None:
            continue
        for r in (end - SPAN, end):
            if r > start and ratio[r] > 0:
                s_rows.append(r)
                s_logs.append(math.log(ratio[r]))
        batch = predict(s_rows, s_logs) if s_rows and s_rows[-1] == end else BATCH


SECTORS = [("n8_2s21_lz0_coulomb", (8, 21, 0)), ("n7_2s18_lz2_coulomb", (7, 18, 2))]


def test_batches_against_fixed_batches(orc, predict):
    wasted = {"fixed": 0, "predicted": 0}
    for tag, (n, s, lz) in SECTORS:
        system = orc.FQHE(n, s, lz, golden("lanczos_%s_basic.npz" % tag)["v"])
        alpha, beta = lanczos_tridiagonal(system.pull, system.dim, orc.random_vector(0, system.dim), 110)
        for precision in (1e-8, 1e-10, 1e-12, 1e-13):
            ratio = convergence_ratios(alpha, beta, precision)
            conv, fixed_end = replay(ratio)
            conv2, end = replay(ratio, predict)
            assert conv2 == conv
            # never more than fixed batches; a plateau of the ratio just before a steep fall (the
            # N=7 run at 1e-13) can leave as many extra rows as fixed batches do
            assert conv <= end <= fixed_end, (tag, precision, conv, end, fixed_end)
            wasted["fixed"] += fixed_end - conv
            wasted["predicted"] += end - conv
    # 26 rows past convergence against 75 for batches of 16 over these eight runs
    assert wasted["predicted"] * 5 <= wasted["fixed"] * 2, wasted


@pytest.fixture(scope="module")
def lowest_ritz(dh):
    lib = ctypes.CDLL(dh.library_path())
    fn = lib._ZN2dh19lanczos_lowest_ritzEiPKdS1_S1_Pd
    d = ctypes.POINTER(ctypes.c_double)
    fn.argtypes = [ctypes.c_int, d, d, d, d]
    fn.restype = ctypes.c_int

    def call(alpha, beta, rows, previous=None):
        out = np.zeros(1)
        prev = None if previous is None else ctypes.pointer(ctypes.c_double(previous))
        assert fn(rows, alpha.ctypes.data_as(d), beta.ctypes.data_as(d), prev, out.ctypes.data_as(d)) == 0
        return out[0]
    return call


def converged_row(values, precision, first=FIRST + 1):
    """BasicLanczosAlgorithm's test over (row, lowest value) pairs: the first passing row or None."""
    prev = None
    for r, e in values:
        last = 2 * e if prev is None else prev
        if r >= first and abs(e - last) < precision * abs(e):
            return r
        prev = e
    return None


@pytest.mark.parametrize("tag,nsl", [("n8_2s21_lz0_coulomb", (8, 21, 0)), ("n7_2s18_lz2_coulomb", (7, 18, 2)),
                                     ("n8_2s21_lz0_v1", (8, 21, 0))])
def test_lowest_ritz_stops_where_ql_stops(orc, lowest_ritz, tag, nsl):
    """Same converged row as with QL values at every precision; on the V1 sector (E0 = 0, which the
    reference runs to max_iter) neither converges."""
    n, s, lz = nsl
    z = golden("lanczos_%s_basic.npz" % tag)
    system = orc.FQHE(n, s, lz, z["v"])
    alpha, beta = lanczos_tridiagonal(system.pull, system.dim, orc.random_vector(0, system.dim), 200)
    ql_values, values, prev = [], [], None
    for rows in range(FIRST, 201):
        t = np.diag(alpha[:rows]) + np.diag(beta[:rows - 1], 1) + np.diag(beta[:rows - 1], -1)
        ql_values.append((rows, np.linalg.eigvalsh(t)[0]))
        prev = lowest_ritz(alpha, beta, rows, prev)
        values.append((rows, prev))
    scale = np.max(np.abs(alpha)) + 2 * np.max(np.abs(beta))
    assert max(abs(a[1] - b[1]) for a, b in zip(ql_values, values)) < 1e-13 * scale
    for precision in (1e-14, 1e-13, 1e-12, 1e-10):
        assert converged_row(values, precision) == converged_row(ql_values, precision)
    if not bool(z["converged"]):
        assert converged_row(values, 1e-14) is None


def test_lowest_ritz_without_or_at_the_bound(lowest_ritz):
    rng = np.random.default_rng(5)
    alpha = rng.normal(size=40)
    beta = rng.uniform(0.1, 1.0, 40)
    t = np.diag(alpha) + np.diag(beta[:39], 1) + np.diag(beta[:39], -1)
    ref = np.linalg.eigvalsh(t)[0]
    assert abs(lowest_ritz(alpha, beta, 40) - ref) < 1e-13
    # the bound equal to the value: Newton cannot improve on it, and the value comes from QL
    assert abs(lowest_ritz(alpha, beta, 40, ref) - ref) < 1e-13
    # the leading block's value as the bound
    lead = np.linalg.eigvalsh(t[:30, :30])[0]
    assert abs(lowest_ritz(alpha, beta, 40, lead) - ref) < 1e-13
