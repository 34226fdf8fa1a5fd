"""BosonOnSphereShort beyond 41-bit words (lz_max + N - 1 = 41 to 62, the reference's range for this
class) on the GPU, where target indices come from the fermionic sector's count table instead of the
split-word rank tables, against the reference's fixtures and the oracle:

- the basis: the words equal the reference's (or their SHA-256), FindStateIndex returns every state's
  own index and -1 outside the sector;
- the product: FP64 within 1e-13 of max|y| of the reference's product with exact interaction factors
  (its own factors drift at these 2S), FP32 within 2e-6, shift, blocks of 2 and 4 in both layouts,
  column ranges against the oracle's push form, for few bosons (the row's prefix sums in shared
  memory) and for more than 20 (both sides of the correction walked);
- Lanczos: the reference's E0 (1e-10; its own factors, within 5e-12 of exact at these 2S)."""
import glob
import hashlib
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, golden

pytestmark = pytest.mark.gpu

NAMES = sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "boson_large_*.npz")))


def _sector(name):
    return tuple(int(v) for v in re.search(r"n(\d+)_2s(\d+)_lz(-?\d+)", name).groups())


def _setup(gpu, name):
    z = golden(name)
    n, s, lz = _sector(name)
    sp = gpu.BosonOnSphereShort(n, lz, s)
    return z, sp, gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, z["v"])


@pytest.mark.parametrize("name", NAMES)
def test_boson_large_basis_matches_reference(gpu, name):
    z, sp, _ = _setup(gpu, name)
    words, _ = sp.states()
    assert sp.dim == int(z["dim"])
    if "words" in z.files:
        assert np.array_equal(words, z["words"])
    else:
        assert hashlib.sha256(np.ascontiguousarray(words, np.uint64).tobytes()).hexdigest() == str(z["words_sha256"])
    assert np.array_equal(sp.FindStateIndex(words), np.arange(sp.dim))
    n, s, lz = _sector(name)
    w = words[: min(16, sp.dim)]
    top = np.uint64(1) << np.uint64(s + n)  # beyond the last bit of the sector
    assert np.all(sp.FindStateIndex(w | top) == -1)
    assert np.all(sp.FindStateIndex(w >> np.uint64(1)) == -1)  # other orbital sum


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
@pytest.mark.parametrize("name", NAMES)
def test_boson_large_product_matches_reference(gpu, orc, name, prec, tol):
    z, sp, H = _setup(gpu, name)
    H.set_precision(prec)
    x = orc.random_vector(int(z["seed"]), sp.dim)
    for shift in (0.0, 0.37):
        if "y_shift%g" % shift not in z.files:
            continue
        H.ShiftHamiltonian(shift)
        ref = z["y_shift%g" % shift]
        assert np.max(np.abs(H.LowLevelMultiply(x) - ref)) <= tol * np.max(np.abs(ref)), shift
    H.ShiftHamiltonian(0.0)
    ref = z["y_shift0"]
    scale = np.max(np.abs(ref))
    for k in (2, 4):
        X = np.stack([x * c for c in (1.0, -0.5, 2.0, 0.25)[:k]], axis=1)
        Y = H.block_multiply(X)
        dsts = np.zeros((k, sp.dim))
        H.LowLevelMultipleAddMultiply(np.ascontiguousarray(X.T), dsts)
        for j in range(k):
            c = X[0, j] / x[0]
            assert np.max(np.abs(Y[:, j] - c * ref)) <= tol * abs(c) * scale, (k, j)
            assert np.max(np.abs(dsts[j] - c * ref)) <= tol * abs(c) * scale, (k, j)


@pytest.mark.parametrize("n,s,lz", [(3, 40, 0), (4, 45, 2), (40, 2, 0), (38, 4, 0)])
def test_boson_large_column_range_matches_oracle(gpu, orc, n, s, lz):
    # (40, 2) and (38, 4): more than 20 bosons, lz_max + N - 1 = 41
    v = orc.coulomb_pseudopotentials(s)
    v[1::2] = 0.0
    sp = gpu.BosonOnSphereShort(n, lz, s)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v)
    O = orc.BosonFQHE(n, s, lz, v, shift=0.3)
    assert np.array_equal(sp.states()[0], O.words)
    H.ShiftHamiltonian(0.3)
    x = orc.random_vector(6, sp.dim)
    ref = O.push(x)
    assert np.max(np.abs(H.LowLevelMultiply(x) - ref)) <= 1e-13 * np.max(np.abs(ref))
    first, nbr = sp.dim // 5, max(1, sp.dim // 3)
    y = np.zeros(sp.dim)
    H.LowLevelAddMultiply(x, y, first, nbr)
    ref = O.push(x, first, nbr)
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.parametrize("name", [n for n in NAMES if "eigenvalues" in golden(n).files])
def test_boson_large_lanczos_matches_reference(gpu, orc, name):
    z, sp, H = _setup(gpu, name)
    lz = gpu.BasicLanczosAlgorithm(H, 1, 600)
    lz.InitializeLanczosAlgorithm(orc.random_vector(int(z["seed"]), sp.dim))
    r = lz.solve(600)
    e_ref = float(z["eigenvalues"][0])
    assert abs(r["eigenvalues"][0] - e_ref) <= 1e-10 * abs(e_ref)


@pytest.mark.parametrize("n,s,lz", [(3, 40, 0), (4, 45, 2), (5, 50, 0)])
def test_boson_large_stored_elements_match_oracle(gpu, orc, n, s, lz):
    # stored elements whose targets come from the count-table ranks
    v = orc.coulomb_pseudopotentials(s)
    v[1::2] = 0.0
    sp = gpu.BosonOnSphereShort(n, lz, s)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v)
    x = orc.random_vector(6, sp.dim)
    y_fly = H.LowLevelMultiply(x)
    assert H.EnableFastMultiplication()[0]
    ref = orc.BosonFQHE(n, s, lz, v).push(x)
    y = H.LowLevelMultiply(x)
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))
    assert np.max(np.abs(y - y_fly)) <= 1e-15 * np.max(np.abs(ref))


@pytest.mark.parametrize("n,s,lz", [(2, 61, 0), (3, 40, 0)])
def test_boson_large_pseudopotential_adjoint(gpu, orc, n, s, lz):
    # g . r = <u|H(r)|v> for random V = r against the oracle; 2S = 61 has 41 K bosonic factors, beyond
    # shared memory (atomics into the global bins), 2S = 40 keeps them in shared memory
    v0 = orc.coulomb_pseudopotentials(s)
    v0[1::2] = 0.0
    sp = gpu.BosonOnSphereShort(n, lz, s)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v0)
    u = orc.random_vector(31, sp.dim)
    w = orc.random_vector(32, sp.dim)
    g = H.pseudopotential_adjoint(u, w)
    rng = np.random.default_rng(7)
    for _ in range(3):
        r = rng.uniform(-1.0, 1.0, s + 1)
        ref = float(u @ orc.BosonFQHE(n, s, lz, r).pull(w))
        assert abs(float(g @ r) - ref) <= 1e-12 * max(1.0, float(np.abs(g) @ np.abs(r)))
