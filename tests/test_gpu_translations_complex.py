"""SpinChainJ1J2HamiltonianWithTranslations (complex phases, any momentum K) on the GPU against the
reference's fixtures (chains of 8 to 20 sites) and the oracle:

- the product on complex vectors ((Re, Im) pairs, the reference's ComplexVector storage): FP64 within
  1e-13 and FP32 within 2e-6 of max|y|, with a shift, several vectors one after the other, and a
  column range against the oracle's push form;
- Lanczos on the (Re, Im) form: E0 equal to the lowest eigenvalue of the reference's own dense matrix
  (1e-10), the ground state an eigenvector of H, E0(K) = E0(L - K), the complex and real Hamiltonians
  agreeing at K = 0 and L/2, and the lowest E0 over all L momenta equal to the plain chain's (L = 16
  and 20, the sector dimensions adding up to C(L, N_up));
- what the complex form does not offer is refused with an error."""
import glob
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, golden

pytestmark = pytest.mark.gpu

NAMES = sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "translations_complex_*.npz")))


def _sector(name):
    return tuple(int(v) for v in re.search(r"L(\d+)_sz(-?\d+)_k(\d+)", name).groups())


def _setup(gpu, name):
    z = golden(name)
    L, sz, k = _sector(name)
    sp = gpu.Spin1_2ChainWithTranslations(L, k, sz)
    return z, sp, gpu.SpinChainJ1J2HamiltonianWithTranslations(sp, L, float(z["j1"]), float(z["j2"]))


def _x(orc, z, dim):
    return orc.random_vector(int(z["seed_re"]), dim) + 1j * orc.random_vector(int(z["seed_im"]), dim)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
@pytest.mark.parametrize("name", NAMES)
def test_complex_product_matches_reference(gpu, orc, name, prec, tol):
    z, sp, H = _setup(gpu, name)
    H.set_precision(prec)
    assert H.dim == 2 * sp.dim
    x = _x(orc, z, sp.dim)
    ref = z["y"]
    scale = np.max(np.abs(ref))
    y = H.LowLevelMultiply(x)
    assert y.dtype == np.complex128 and np.max(np.abs(y - ref)) <= tol * scale
    H.ShiftHamiltonian(0.37)
    assert np.max(np.abs(H.LowLevelMultiply(x) - ref - 0.37 * x)) <= tol * scale
    H.ShiftHamiltonian(0.0)
    X = np.stack([x, (0.5 - 2j) * x])
    D = np.zeros_like(X)
    H.LowLevelMultipleAddMultiply(X, D)
    assert np.max(np.abs(D[0] - ref)) <= tol * scale
    assert np.max(np.abs(D[1] - (0.5 - 2j) * ref)) <= tol * abs(0.5 - 2j) * scale


@pytest.mark.parametrize("name", ["translations_complex_L12_sz2_k5_j2_0.4.npz",
                                  "translations_complex_L16_sz0_k3_j2_0.2.npz"])
def test_complex_column_range_matches_oracle(gpu, orc, name):
    z, sp, H = _setup(gpu, name)
    L, sz, k = _sector(name)
    x = _x(orc, z, sp.dim)
    first, nbr = sp.dim // 5, sp.dim // 3
    xs = np.zeros_like(x)
    xs[first:first + nbr] = x[first:first + nbr]
    ref = orc.translation_j1j2_push_complex(L, sz, k, float(z["j1"]), float(z["j2"]), xs)
    y = np.zeros(sp.dim, np.complex128)
    H.LowLevelAddMultiply(x, y, first, nbr)
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))


def _e0(gpu, H, seed=3, max_iter=800):
    lz = gpu.BasicLanczosAlgorithm(H, 1, max_iter)
    lz.InitializeLanczosAlgorithm(seed=seed)
    r = lz.solve(max_iter)
    assert r["converged"]
    return float(r["eigenvalues"][0])


@pytest.mark.parametrize("name", [n for n in NAMES if "eigenvalues" in golden(n).files and _sector(n)[0] >= 12])
def test_complex_lanczos_matches_reference_dense(gpu, name):
    z, sp, H = _setup(gpu, name)
    e_ref = float(z["eigenvalues"][0])
    assert abs(_e0(gpu, H) - e_ref) <= 1e-10 * abs(e_ref)
    g = gpu.BasicLanczosAlgorithmWithGroundState(H, 1, 800)
    g.InitializeLanczosAlgorithm(seed=4)
    g.solve(800)
    psi = H.as_complex(g.GetGroundState())
    r = H.LowLevelMultiply(psi) - e_ref * psi
    assert np.linalg.norm(r) <= 1e-6 * np.linalg.norm(psi)


def test_complex_and_real_hamiltonians_agree_at_real_momenta(gpu, orc):
    for L, k in ((12, 0), (12, 6), (14, 7)):
        sp = gpu.Spin1_2ChainWithTranslations(L, k, 0)
        Hc = gpu.SpinChainJ1J2HamiltonianWithTranslations(sp, L, 1.0, 0.4)
        Hr = gpu.SpinChainJ1J2RealHamiltonianWithTranslations(sp, L, 1.0, 0.4)
        x = orc.random_vector(5, sp.dim)
        yc = Hc.LowLevelMultiply(x.astype(np.complex128))
        assert np.max(np.abs(yc.imag)) <= 1e-14 * np.max(np.abs(yc.real))
        assert np.max(np.abs(yc.real - Hr.LowLevelMultiply(x))) <= 1e-13 * np.max(np.abs(yc.real))


@pytest.mark.parametrize("L,j2", [(16, 0.3), (20, 0.2)])
def test_all_momenta_hold_the_chain_spectrum_bottom(gpu, L, j2):
    e, total = [], 0
    for k in range(L):
        sp = gpu.Spin1_2ChainWithTranslations(L, k, 0)
        total += sp.dim
        e.append(_e0(gpu, gpu.SpinChainJ1J2HamiltonianWithTranslations(sp, L, 1.0, j2)))
    from math import comb
    assert total == comb(L, L // 2)
    for k in range(1, L):
        assert abs(e[k] - e[L - k]) <= 1e-10 * abs(e[k])
    e_chain = _e0(gpu, gpu.SpinChainJ1J2Hamiltonian(gpu.Spin1_2Chain(L, 0), 1.0, j2))
    assert abs(min(e) - e_chain) <= 1e-10 * abs(e_chain)


def test_complex_refusals(gpu, tmp_path):
    sp = gpu.Spin1_2ChainWithTranslations(12, 1, 0)
    H = gpu.SpinChainJ1J2HamiltonianWithTranslations(sp, 12, 1.0, 0.5)
    with pytest.raises(gpu.DiagHamError, match="error -4"):
        gpu.BasicLanczosAlgorithmWithDiskStorage(H, 1, 100, directory=str(tmp_path))
    with pytest.raises(gpu.DiagHamError, match="error -4"):
        H.block_multiply(np.ones((H.dim, 2)))
    with pytest.raises(gpu.DiagHamError, match="error -4"):
        gpu.BasicBlockLanczosAlgorithm(H, 1, 100, block_size=2)
    with pytest.raises(gpu.DiagHamError, match="error -1"):
        gpu._Hamiltonian.LowLevelMultiply(H, np.ones(H.dim), None, 1, 4)
    with pytest.raises(gpu.DiagHamError):
        gpu.SpinChainJ1J2HamiltonianWithTranslations(gpu.Spin1_2Chain(12, 0), 12, 1.0, 0.5)
