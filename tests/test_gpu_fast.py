"""Stored-element ("fast multiplication") products: the sliced-ELL elements built on the device
against the oracle's products (FP64 1e-13, FP32 2e-6 of max|y|), single vectors and row-interleaved
blocks, with a shift; the memory budget (not built when too small, products unchanged); new
pseudopotentials after the build (only the diagonal is recomputed); partial column ranges (on the
fly); and a Lanczos run against the reference's energy (1e-10 relative)."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _setup(gpu, n=8, s=21, lz=0, v=None):
    z = golden("lanczos_n8_2s21_lz0_coulomb_basic.npz")
    v = z["v"] if v is None else v
    sp = gpu.FermionOnSphere(n, lz, s)
    return z, sp, gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
def test_stored_products_match_oracle(gpu, orc, prec, tol):
    z, sp, H = _setup(gpu)
    on, nbytes = H.EnableFastMultiplication()
    assert on and nbytes > 0
    H.set_precision(prec)
    H.ShiftHamiltonian(0.25)
    O = orc.FQHE(8, 21, 0, z["v"])
    x = orc.random_vector(9, sp.dim)
    ref = O.pull(x) + 0.25 * x
    y = H.LowLevelMultiply(x)
    assert np.max(np.abs(y - ref)) <= tol * np.max(np.abs(ref))
    for k in (2, 3, 4):
        X = np.random.default_rng(k).uniform(-1.0, 1.0, (sp.dim, k))
        Y = H.block_multiply(X)
        for j in range(k):
            r = O.pull(np.ascontiguousarray(X[:, j])) + 0.25 * X[:, j]
            assert np.max(np.abs(Y[:, j] - r)) <= tol * np.max(np.abs(r)), (k, j)


def test_budget_too_small_keeps_on_the_fly(gpu, orc):
    z, sp, H = _setup(gpu)
    on, nbytes = H.EnableFastMultiplication(1000)
    assert not on and nbytes > 1000
    x = orc.random_vector(4, sp.dim)
    ref = orc.FQHE(8, 21, 0, z["v"]).pull(x)
    assert np.max(np.abs(H.LowLevelMultiply(x) - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_new_pseudopotentials_after_build(gpu, orc):
    z, sp, H = _setup(gpu)
    assert H.EnableFastMultiplication()[0]
    v2 = np.array(z["v"]) * 0.7
    v2[3] += 0.11
    H.set_pseudopotentials(v2)
    x = orc.random_vector(6, sp.dim)
    ref = orc.FQHE(8, 21, 0, v2).pull(x)
    assert np.max(np.abs(H.LowLevelMultiply(x) - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_partial_range_and_disable(gpu, orc):
    z, sp, H = _setup(gpu)
    assert H.EnableFastMultiplication()[0]
    O = orc.FQHE(8, 21, 0, z["v"])
    x = orc.random_vector(7, sp.dim)
    first, nbr = 100, 3000
    y = np.zeros(sp.dim)
    H.LowLevelAddMultiply(x, y, first, nbr)
    xm = np.zeros(sp.dim)
    xm[first:first + nbr] = x[first:first + nbr]
    ref = O.pull(xm)
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))
    H.DisableFastMultiplication()
    ref = O.pull(x)
    assert np.max(np.abs(H.LowLevelMultiply(x) - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_lanczos_with_stored_elements(gpu, orc):
    z, sp, H = _setup(gpu)
    assert H.EnableFastMultiplication()[0]
    lz = gpu.BasicLanczosAlgorithm(H, 1, 300)
    lz.InitializeLanczosAlgorithm(orc.random_vector(0, sp.dim))
    r = lz.solve(200)
    e_ref = float(z["eigenvalues"][0])
    assert abs(r["eigenvalues"][0] - e_ref) < 1e-10 * abs(e_ref)
    assert abs(r["iterations"] - int(z["iterations"])) <= 2


def test_stored_matches_on_the_fly_large_sector(gpu):
    import torch
    v = gpu.coulomb_pseudopotentials(27)
    v[0::2] = 0.0
    sp = gpu.FermionOnSphere(10, 0, 27)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 10, 27, v)
    x = torch.rand(sp.dim, 4, dtype=torch.float64, device="cuda") - 0.5
    y0 = H.block_multiply(x)
    assert H.EnableFastMultiplication()[0]
    y1 = H.block_multiply(x)
    assert float((y1 - y0).abs().max()) <= 1e-13 * float(y0.abs().max())


def test_autotune_chooses_between_stored_and_on_the_fly(gpu, orc):
    z, sp, H = _setup(gpu)
    assert H.EnableFastMultiplication()[0]
    r = H.autotune(block_size=2, repeats=2)
    assert r["stored_ms"] > 0 and r["best_ms"] <= r["stored_ms"] + 1e-9
    assert r["stored_in_use"] == (r["best_ms"] == r["stored_ms"])
    x = orc.random_vector(3, sp.dim)
    ref = orc.FQHE(8, 21, 0, z["v"]).pull(x)
    assert np.max(np.abs(H.LowLevelMultiply(x) - ref)) <= 1e-13 * np.max(np.abs(ref))
