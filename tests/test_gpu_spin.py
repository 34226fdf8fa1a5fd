"""Spin1_2Chain + the periodic J1-J2 chain on the GPU against the reference fixtures.
Indices bit-exact; FP64 products to rounding (1e-12); FP32 within 2e-6 max|y|."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden

pytestmark = pytest.mark.gpu


def _parse(name):
    parts = name[:-4].split("_")
    return int(parts[2][1:]), int(parts[3][2:])


@pytest.mark.parametrize("name", sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "spin_basis_*.npz"))))
def test_spin_basis_bit_exact(gpu, name):
    z = golden(name)
    L, sz = _parse(name)
    ch = gpu.Spin1_2Chain(L, sz)
    words, _ = ch.states()
    assert np.array_equal(words, z["words"])
    assert np.array_equal(ch.FindStateIndex(words), np.arange(len(words)))


@pytest.mark.parametrize("name", sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "spin_matvec_*.npz"))))
def test_spin_matvec_vs_reference(gpu, orc, name):
    z = golden(name)
    parts = name[:-4].split("_")
    L, sz = int(parts[2][1:]), int(parts[3][2:])
    j1, j2 = float(parts[4][1:]), float(parts[5])
    ch = gpu.Spin1_2Chain(L, sz)
    H = gpu.SpinChainJ1J2Hamiltonian(ch, j1, j2)
    x = orc.random_vector(3, ch.dim)
    y = H.LowLevelMultiply(x)
    assert np.max(np.abs(y - z["y"])) < 1e-12
    H.set_precision("fp32")
    y32 = H.LowLevelMultiply(x)
    assert np.max(np.abs(y32 - z["y"])) < 2e-6 * np.max(np.abs(z["y"]))


@pytest.mark.parametrize("L,sz", [(20, 0), (21, 1), (18, 4), (32, 28)])
def test_spin_matvec_vs_oracle_wrap_bonds(gpu, orc, L, sz):
    # every bond incl. the three that wrap around the chain, against the oracle's full rank
    ch = gpu.Spin1_2Chain(L, sz)
    words = orc.spin_basis(L, sz)
    H = gpu.SpinChainJ1J2Hamiltonian(ch, 1.0, 0.37)
    x = orc.random_vector(11, ch.dim)
    ref = orc.spin_j1j2_multiply(L, sz, words, 1.0, 0.37, x, shift=0.5)
    H.ShiftHamiltonian(0.5)
    assert np.max(np.abs(H.LowLevelMultiply(x) - ref)) < 1e-12


def test_spin_column_range(gpu, orc):
    L, sz = 14, 0
    ch = gpu.Spin1_2Chain(L, sz)
    words = orc.spin_basis(L, sz)
    H = gpu.SpinChainJ1J2Hamiltonian(ch, 1.0, 0.5)
    x = orc.random_vector(1, ch.dim)
    first, nbr = 500, 1200
    xm = np.zeros_like(x)
    xm[first:first + nbr] = x[first:first + nbr]
    ref = orc.spin_j1j2_multiply(L, sz, words, 1.0, 0.5, xm)
    y = np.zeros(ch.dim)
    H.LowLevelAddMultiply(x, y, first, nbr)
    assert np.max(np.abs(y - ref)) < 1e-12


def test_majumdar_ghosh_point(gpu):
    # J2 = J1 / 2: E0 = -3L/8 exactly (two dimer coverings)
    ch = gpu.Spin1_2Chain(20, 0)
    H = gpu.SpinChainJ1J2Hamiltonian(ch, 1.0, 0.5)
    lz = gpu.BasicLanczosAlgorithm(H, 1, 400)
    lz.InitializeLanczosAlgorithm(seed=0)
    r = lz.solve(400)
    assert abs(r["eigenvalues"][0] + 7.5) < 1e-10


@pytest.mark.parametrize("name", sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "spin_lanczos_*.npz"))))
def test_spin_lanczos_vs_reference(gpu, orc, name):
    z = golden(name)
    parts = name[:-4].split("_")
    L, sz = int(parts[2][1:]), int(parts[3][2:])
    j1, j2 = float(parts[4][1:]), float(parts[5])
    ch = gpu.Spin1_2Chain(L, sz)
    H = gpu.SpinChainJ1J2Hamiltonian(ch, j1, j2)
    lz = gpu.BasicLanczosAlgorithm(H, 1, 400)
    lz.InitializeLanczosAlgorithm(orc.random_vector(0, ch.dim))
    r = lz.solve(400, graph_batch=1)
    e = float(z["eigenvalues"][0])
    assert abs(r["eigenvalues"][0] - e) < 1e-10 * abs(e)
    assert abs(r["iterations"] - int(z["iterations"])) <= 2
