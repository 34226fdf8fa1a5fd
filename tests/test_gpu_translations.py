"""Spin1_2ChainWithTranslations with SpinChainJ1J2RealHamiltonianWithTranslations on the GPU against the
reference's fixtures (chains of 8 to 20 sites, Sz 0 to 2, momenta 0 and L/2) and the oracle:

- the basis: the representatives equal the reference's in order, FindStateIndex returns every
  representative's own index, and a word that is not a representative is not found;
- the product: FP64 within 1e-13 and FP32 within 2e-6 of max|y|, with a shift, in blocks of 2 and 4
  vectors (both layouts) and over a column range;
- Lanczos: the reference's E0 (1e-10 relative, iteration counter within 2) on every sector of 300
  states or more, and for chains of 18 to 24 sites the lower of the K = 0 and K = L/2 ground energies
  equals the ground energy of the whole Sz sector (plain Spin1_2Chain), -3L/8 at the Majumdar-Ghosh
  point J2 = J1/2;
- the element count equals the oracle's, and momenta other than 0 and L/2 are refused by the real
  Hamiltonian."""
import glob
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, golden

pytestmark = pytest.mark.gpu

NAMES = sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "translations_L*.npz")))


def _sector(name):
    L, sz, k = (int(v) for v in re.search(r"L(\d+)_sz(-?\d+)_k(\d+)", name).groups())
    return L, sz, k


def _setup(gpu, name):
    z = golden(name)
    L, sz, k = _sector(name)
    sp = gpu.Spin1_2ChainWithTranslations(L, k, sz)
    return z, sp, gpu.SpinChainJ1J2RealHamiltonianWithTranslations(sp, L, float(z["j1"]), float(z["j2"]))


@pytest.mark.parametrize("name", NAMES)
def test_translation_basis_matches_reference(gpu, name):
    z, sp, _ = _setup(gpu, name)
    words, _ = sp.states()
    assert sp.dim == len(z["words"])
    assert np.array_equal(words, z["words"])
    assert np.array_equal(sp.FindStateIndex(words), np.arange(sp.dim))
    # the rotations of a representative that differ from it are not in the basis
    L = _sector(name)[0]
    mask = (1 << L) - 1
    rot = np.array([((int(w) >> 1) | ((int(w) & 1) << (L - 1))) & mask for w in words[:64]], np.uint64)
    moved = rot != words[:64]
    assert np.all(sp.FindStateIndex(rot[moved]) == -1)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
@pytest.mark.parametrize("name", NAMES)
def test_translation_product_matches_reference(gpu, orc, name, prec, tol):
    z, sp, H = _setup(gpu, name)
    H.set_precision(prec)
    x = orc.random_vector(int(z["seed"]), sp.dim)
    ref = z["y"]
    scale = np.max(np.abs(ref))
    y = H.LowLevelMultiply(x)
    assert np.max(np.abs(y - ref)) <= tol * scale
    H.ShiftHamiltonian(0.37)
    y = H.LowLevelMultiply(x)
    assert np.max(np.abs(y - ref - 0.37 * x)) <= tol * scale
    H.ShiftHamiltonian(0.0)
    for kb in (2, 4):
        X = np.stack([x * c for c in (1.0, -0.5, 2.0, 0.25)[:kb]], axis=1)
        Y = H.block_multiply(X)
        srcs = np.ascontiguousarray(X.T)
        dsts = np.zeros_like(srcs)
        H.LowLevelMultipleAddMultiply(srcs, dsts)
        for j in range(kb):
            c = X[0, j] / x[0]
            assert np.max(np.abs(Y[:, j] - c * ref)) <= tol * abs(c) * scale, (kb, j)
            assert np.max(np.abs(dsts[j] - c * ref)) <= tol * abs(c) * scale, (kb, j)


@pytest.mark.parametrize("name", ["translations_L12_sz2_k6_j2_0.5.npz", "translations_L16_sz0_k8_j2_0.2.npz"])
def test_translation_column_range_matches_oracle(gpu, orc, name):
    z, sp, H = _setup(gpu, name)
    L, sz, k = _sector(name)
    x = orc.random_vector(5, sp.dim)
    first, nbr = sp.dim // 5, sp.dim // 3
    xs = np.zeros(sp.dim)
    xs[first:first + nbr] = x[first:first + nbr]
    ref = orc.translation_j1j2_push(L, sz, k, float(z["j1"]), float(z["j2"]), xs)
    y = np.zeros(sp.dim)
    H.LowLevelAddMultiply(x, y, first, nbr)
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.parametrize("name", [n for n in NAMES if "eigenvalues" in golden(n).files])
def test_translation_lanczos_matches_reference(gpu, orc, name):
    z, sp, H = _setup(gpu, name)
    lz = gpu.BasicLanczosAlgorithm(H, 1, 400)
    lz.InitializeLanczosAlgorithm(orc.random_vector(int(z["seed"]), sp.dim))
    r = lz.solve(400)
    e_ref = float(z["eigenvalues"][0])
    assert abs(r["eigenvalues"][0] - e_ref) <= 1e-10 * abs(e_ref)
    assert abs(r["iterations"] - int(z["iterations"])) <= 2


def _ground(gpu, H):
    lz = gpu.BasicLanczosAlgorithm(H, 1, 600)
    lz.InitializeLanczosAlgorithm(seed=3)
    return lz.solve(600)["eigenvalues"][0]


@pytest.mark.parametrize("L,j2", [(18, 0.3), (20, 0.2), (24, 0.5)])
def test_momentum_sectors_hold_the_chain_ground_state(gpu, L, j2):
    e = [_ground(gpu, gpu.SpinChainJ1J2RealHamiltonianWithTranslations(
        gpu.Spin1_2ChainWithTranslations(L, k, 0), L, 1.0, j2)) for k in (0, L // 2)]
    e_chain = _ground(gpu, gpu.SpinChainJ1J2Hamiltonian(gpu.Spin1_2Chain(L, 0), 1.0, j2))
    assert abs(min(e) - e_chain) <= 1e-10 * abs(e_chain)
    if j2 == 0.5:
        assert abs(e[0] + 3.0 * L / 8.0) <= 1e-10 and abs(e[1] + 3.0 * L / 8.0) <= 1e-10


def test_translation_counts_and_refusals(gpu, orc):
    for L, sz, k in ((12, 0, 0), (13, 1, 0), (16, 0, 8)):
        sp = gpu.Spin1_2ChainWithTranslations(L, k, sz)
        H = gpu.SpinChainJ1J2RealHamiltonianWithTranslations(sp, L, 1.0, 0.5)
        assert H.count_elements() == orc.translation_flip_count(L, sz, k)
        assert H.count_diagonal_elements() == 0
    sp = gpu.Spin1_2ChainWithTranslations(12, 1, 0)
    assert sp.dim == len(orc.translation_basis(12, 0, 1)[0])
    with pytest.raises(gpu.DiagHamError, match="error -4"):
        gpu.SpinChainJ1J2RealHamiltonianWithTranslations(sp, 12, 1.0, 0.5)
    with pytest.raises(gpu.DiagHamError):
        gpu.Spin1_2ChainWithTranslations(12, 12, 0)
    with pytest.raises(gpu.DiagHamError):
        gpu.Spin1_2ChainWithTranslations(12, 0, 1)
