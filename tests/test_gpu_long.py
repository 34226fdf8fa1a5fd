"""FermionOnSphereLong (lz_max up to 126) and FermionOnSphere beyond the split-word tables (41 <= lz_max
<= 62) on the GPU, against the reference's fixtures and the oracle:

- the basis: the words equal the reference's in order (or their SHA-256 for the large sectors),
  FindStateIndex returns every state's own index and -1 outside the sector;
- the product (ParticleOnSphereGenericHamiltonian, on the fly): FP64 within 1e-13 of max|y| of the
  reference's product with exact interaction factors (FermionOnSphereLong; the reference's own factors
  drift from 2S = 62 on, 87% off at 2S = 126) or within 1e-12 of its product with its own factors
  (FermionOnSphere, factors within 3.6e-13); FP32 within 2e-6; blocks of 2 and 4 vectors in both
  layouts; a column range against the oracle's push form;
- Lanczos: the reference's E0 (1e-10) where its factors are accurate, the lowest eigenvalue of the
  dense matrix at 2S = 126, and E0 = 0 with <L^2> = 0 for the Laughlin 1/M state of its parent
  pseudopotentials at 2S = 66; block and FP32-refined solves reach the same energy;
- stored elements (EnableFastMultiplication, uint32 factor index | sign payloads, factors read
  through the cache): the same products and Lanczos runs;
- the pseudopotential adjoint (shared-memory bins up to 2S of about 54, atomics beyond) against
  products of the oracle;
- counts, and what the 128-bit engine does not offer is refused with an error."""
import glob
import hashlib
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, golden

pytestmark = pytest.mark.gpu

NAMES = sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "long_*.npz")))


def _sector(name):
    space, n, s, lz = re.match(r"long_(\w+?)_n(\d+)_2s(\d+)_lz(-?\d+)", name).groups()
    return space, int(n), int(s), int(lz)


def _space(gpu, name):
    space, n, s, lz = _sector(name)
    if space == "long":
        return gpu.FermionOnSphereLong(n, lz, s)
    return gpu.FermionOnSphere(n, lz, s)


def _pairs(sp):
    if isinstance(sp, __import__("diagham_b200").FermionOnSphereLong):
        return sp.states()[0]
    w = sp.states()[0]
    return np.stack([w, np.zeros_like(w)], axis=1)


@pytest.mark.parametrize("name", NAMES)
def test_long_basis_matches_reference(gpu, name):
    z = golden(name)
    sp = _space(gpu, name)
    pairs = _pairs(sp)
    if "words" in z.files:
        assert np.array_equal(pairs, z["words"])
    else:
        assert sp.dim == int(z["dim"])
        assert hashlib.sha256(np.ascontiguousarray(pairs).tobytes()).hexdigest() == str(z["words_sha256"])
    if isinstance(sp, gpu.FermionOnSphereLong):
        idx = sp.FindStateIndex(pairs)
    else:
        idx = sp.FindStateIndex(pairs[:, 0])
    assert np.array_equal(idx, np.arange(sp.dim))


def test_long_find_rejects_words_outside_the_sector(gpu):
    sp = gpu.FermionOnSphereLong(4, 0, 70)
    words = sp.word_values(sp.states(0, 8)[0])
    bad = [w | 1 if not w & 1 else w & ~1 for w in words]           # one fermion more or less
    bad += [w | (1 << 71) for w in words]                            # beyond lz_max
    moved = []
    for w in words:                                                  # same count, other sum
        top = w.bit_length() - 1
        if not (w >> (top + 1)) & 1 and top + 1 <= 70:
            moved.append((w & ~(1 << top)) | (1 << (top + 1)))
    assert np.all(sp.FindStateIndex(bad + moved) == -1)
    assert np.array_equal(sp.FindStateIndex(words), np.arange(8))


@pytest.mark.parametrize("prec,tol64", [("fp64", None), ("fp32", 2e-6)])
@pytest.mark.parametrize("name", NAMES)
def test_long_product_matches_reference(gpu, orc, name, prec, tol64):
    z = golden(name)
    space, n, s, lz = _sector(name)
    sp = _space(gpu, name)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, z["v"])
    H.set_precision(prec)
    tol = tol64 if tol64 is not None else (1e-13 if space == "long" else 1e-12)
    x = orc.random_vector(int(z["seed"]), sp.dim)
    shifts = [0.0] + ([0.37] if "y_shift0.37" in z.files else [])
    for shift in shifts:
        H.ShiftHamiltonian(shift)
        ref = z["y_shift%g" % shift]
        y = H.LowLevelMultiply(x)
        assert np.max(np.abs(y - ref)) <= tol * np.max(np.abs(ref)), shift
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


@pytest.mark.parametrize("n,s,lz", [(3, 63, 1), (3, 126, 0), (4, 50, 0)])
def test_long_column_range_matches_oracle_push(gpu, orc, n, s, lz):
    v = orc.coulomb_pseudopotentials(s)
    v[0::2] = 0.0
    sp = gpu.FermionOnSphereLong(n, lz, s)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v)
    H.ShiftHamiltonian(0.3)
    O = orc.FQHELong(n, s, lz, v, shift=0.3)
    x = orc.random_vector(2, sp.dim)
    first, nbr = sp.dim // 5, sp.dim // 3
    y = np.zeros(sp.dim)
    H.LowLevelAddMultiply(x, y, first, nbr)
    ref = O.push(x, first, nbr)
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.parametrize("name", [n for n in NAMES if "eigenvalues" in golden(n).files])
def test_long_lanczos_matches_reference(gpu, orc, name):
    z = golden(name)
    space, n, s, lz = _sector(name)
    sp = _space(gpu, name)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, z["v"])
    lz_ = gpu.BasicLanczosAlgorithm(H, 1, 600)
    lz_.InitializeLanczosAlgorithm(orc.random_vector(int(z["seed"]), sp.dim))
    r = lz_.solve(600)
    e_ref = float(z["eigenvalues"][0])
    assert abs(r["eigenvalues"][0] - e_ref) <= 1e-10 * abs(e_ref)


def test_long_lanczos_matches_dense_at_2s_126(gpu, orc):
    z = golden("long_long_n3_2s126_lz0.npz")
    sp = gpu.FermionOnSphereLong(3, 0, 126)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 3, 126, z["v"])
    dim = sp.dim
    cols = []
    for c0 in range(0, dim, 4):
        k = min(4, dim - c0)
        E = np.zeros((dim, k))
        E[c0 + np.arange(k), np.arange(k)] = 1.0
        cols.append(H.block_multiply(E) if k > 1 else H.LowLevelMultiply(E[:, 0])[:, None])
    M = np.concatenate(cols, axis=1)
    assert np.max(np.abs(M - M.T)) <= 1e-13 * np.max(np.abs(M))
    e_dense = np.linalg.eigvalsh(0.5 * (M + M.T))[0]
    # the bottom of this spectrum is dense (gap 9e-5): basic Lanczos needs 600 to 730 iterations
    lz_ = gpu.BasicLanczosAlgorithm(H, 1, 1500)
    lz_.InitializeLanczosAlgorithm(seed=1)
    r = lz_.solve(1500)
    assert r["converged"]
    assert abs(r["eigenvalues"][0] - e_dense) <= 1e-12 * abs(e_dense)


def test_laughlin_state_at_2s_66(gpu):
    # N = 3 at 2S = 33 (N - 1) = 66: the 1/33 Laughlin state is the unique zero mode of V_m = 1 for odd
    # m < 33 and has L = 0
    n, s = 3, 66
    v = np.zeros(s + 1)
    v[1:33:2] = 1.0
    sp = gpu.FermionOnSphereLong(n, 0, s)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v)
    lz2 = gpu.BasicLanczosAlgorithm(H, 2, 600)
    lz2.InitializeLanczosAlgorithm(seed=2)
    e = lz2.solve(600)["eigenvalues"]
    assert abs(e[0]) < 1e-10 and e[1] > 1.0  # 1.18 by dense diagonalisation of the oracle's matrix
    lz_ = gpu.BasicLanczosAlgorithmWithGroundState(H, 1, 600)
    lz_.InitializeLanczosAlgorithm(seed=2)
    lz_.solve(600)
    psi = lz_.GetGroundState()
    L2 = gpu.ParticleOnSphereL2Hamiltonian(sp, n, s, 0)
    assert abs(L2.total_angular_momentum(psi)) < 1e-6


def test_long_block_and_refined_solves(gpu):
    z = golden("long_long_n4_2s70_lz0.npz")
    sp = gpu.FermionOnSphereLong(4, 0, 70)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 4, 70, z["v"])
    e_ref = float(z["eigenvalues"][0])
    b = gpu.BasicBlockLanczosAlgorithm(H, 1, 600, block_size=2)
    b.InitializeLanczosAlgorithm(seed=4)
    assert abs(b.solve(600)["eigenvalues"][0] - e_ref) <= 1e-10 * abs(e_ref)
    H.set_precision("fp32")
    lz_ = gpu.BasicLanczosAlgorithmWithGroundState(H, 1, 600)
    lz_.InitializeLanczosAlgorithm(seed=5)
    r = lz_.solve_refined(600, precision=1e-12)
    assert abs(r["energy"] - e_ref) <= 1e-10 * abs(e_ref)


def test_long_counts(gpu, orc):
    n, s, lz = 3, 63, 1
    v = orc.coulomb_pseudopotentials(s)
    sp = gpu.FermionOnSphereLong(n, lz, s)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v)
    moves = 0
    for w in orc.fermion_basis_long(n, s, lz):
        occ = [m for m in range(s + 1) if (w >> m) & 1]
        for i, m1 in enumerate(occ):
            for m2 in occ[:i]:
                a = w & ~(1 << m1) & ~(1 << m2)
                M = m1 + m2
                moves += sum(1 for m3 in range(M // 2 + 1, min(M, s) + 1)
                             if not (a >> m3) & 1 and not (a >> (M - m3)) & 1)
    assert H.count_elements() == moves
    assert H.count_diagonal_elements() == 3 * sp.dim


def test_long_refusals(gpu):
    v = np.ones(71)
    sp = gpu.FermionOnSphereLong(4, 0, 70)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 4, 70, v)
    with pytest.raises(gpu.DiagHamError, match="error -4"):
        sp.set_index_mode("lookup")
    with pytest.raises(gpu.DiagHamError, match="error -4"):
        gpu._Space.states(sp)  # 128-bit words need the pair form
    with pytest.raises(gpu.DiagHamError):
        gpu.FermionOnSphere(3, 1, 63)
    with pytest.raises(gpu.DiagHamError):
        gpu.FermionOnSphereLong(3, 0, 128)
    with pytest.raises(gpu.DiagHamError, match="error -4"):
        gpu.fqhe_sectors_block_lanczos(3, 50, [0, 2], np.ones(51))
    # 41 <= lz_max <= 62 through FermionOnSphere: 64-bit words at the interface
    f = gpu.FermionOnSphere(3, 0, 50)
    w, lzm = f.states()
    assert w.dtype == np.uint64 and np.all(lzm <= 50)
    # orbital cuts work on these words too (against the oracle in test_gpu_entanglement.py)
    assert f.EvaluatePartialDensityMatrix(20, 1, 0, np.ones(f.dim)).shape == (1, 1)
    lng = gpu.FermionOnSphereLong(3, 0, 70)  # 128-bit words: no orbital cuts
    with pytest.raises(gpu.DiagHamError, match="error -4"):
        gpu._cut_matrix(lng, gpu.load().dh_fermion_on_sphere_partial_density_matrix, np.ones(lng.dim), (20, 1, 0), True)


@pytest.mark.parametrize("n,s,lz", [(1, 100, 10), (64, 63, 0), (3, 100, 294), (2, 126, -250)])
def test_long_one_state_sectors(gpu, orc, n, s, lz):
    # one fermion, the filled shell (every pair returns to itself), the highest and the lowest Lz
    v = orc.coulomb_pseudopotentials(s)
    v[0::2] = 0.0
    sp = gpu.FermionOnSphereLong(n, lz, s)
    assert sp.dim == 1
    assert sp.word_values(sp.states()[0]) == orc.fermion_basis_long(n, s, lz)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v)
    H.ShiftHamiltonian(0.25)
    y = H.LowLevelMultiply(np.array([1.0]))
    ref = orc.FQHELong(n, s, lz, v, shift=0.25).push(np.array([1.0]))
    assert abs(y[0] - ref[0]) <= 1e-13 * max(1.0, abs(ref[0]))
    assert H.count_elements() == n * (n - 1) // 2


def test_long_empty_and_oversized_sectors(gpu):
    with pytest.raises(gpu.DiagHamError, match="empty sector"):
        gpu.FermionOnSphereLong(4, -312, 80)
    with pytest.raises(gpu.DiagHamError, match="2\\^31"):
        gpu.FermionOnSphereLong(40, 0, 126)
    with pytest.raises(gpu.DiagHamError, match="not reachable"):
        gpu.FermionOnSphereLong(3, 1, 100)
    f = gpu.FermionOnSphere(63, 0, 62)  # the filled 64-bit shell through FermionOnSphere
    assert f.dim == 1 and int(f.states()[0][0]) == (1 << 63) - 1


def test_many_fermion_sectors_walk_both_sides(gpu, orc):
    # more than 20 fermions: no per-row prefix sums, the rank correction walks row and target;
    # near-full shells (3 and 2 holes) keep the sectors small
    v = orc.coulomb_pseudopotentials(62)
    v[0::2] = 0.0
    f = gpu.FermionOnSphere(59, 0, 62)
    O = orc.FQHE(59, 62, 0, v, shift=0.2)
    assert np.array_equal(f.states()[0], O.words)
    H = gpu.ParticleOnSphereGenericHamiltonian(f, 59, 62, v)
    H.ShiftHamiltonian(0.2)
    x = orc.random_vector(3, f.dim)
    ref = O.push(x)
    assert np.max(np.abs(H.LowLevelMultiply(x) - ref)) <= 1e-13 * np.max(np.abs(ref))
    v41 = orc.coulomb_pseudopotentials(41)
    v41[0::2] = 0.0
    sp = gpu.FermionOnSphereLong(40, 2, 41)
    assert sp.word_values(sp.states()[0]) == orc.fermion_basis_long(40, 41, 2)
    Hl = gpu.ParticleOnSphereGenericHamiltonian(sp, 40, 41, v41)
    xl = orc.random_vector(4, sp.dim)
    ref = orc.FQHELong(40, 41, 2, v41).push(xl)
    assert np.max(np.abs(Hl.LowLevelMultiply(xl) - ref)) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.parametrize("prec,tol64", [("fp64", None), ("fp32", 2e-6)])
@pytest.mark.parametrize("name", NAMES)
def test_long_stored_elements_match_reference(gpu, orc, name, prec, tol64):
    # EnableFastMultiplication on the count-table engine (AbstractQHEOnSphereHamiltonian.cc:3625, 3814):
    # the rows' (target, factor index, sign) in device memory, then products from them
    z = golden(name)
    space, n, s, lz = _sector(name)
    sp = _space(gpu, name)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, z["v"])
    H.set_precision(prec)
    tol = tol64 if tol64 is not None else (1e-13 if space == "long" else 1e-12)
    x = orc.random_vector(int(z["seed"]), sp.dim)
    y_fly = H.LowLevelMultiply(x)
    enabled, nbytes = H.EnableFastMultiplication()
    assert enabled and nbytes >= 8 * (H.count_elements() - H.count_diagonal_elements())
    shifts = [0.0] + ([0.37] if "y_shift0.37" in z.files else [])
    for shift in shifts:
        H.ShiftHamiltonian(shift)
        ref = z["y_shift%g" % shift]
        assert np.max(np.abs(H.LowLevelMultiply(x) - ref)) <= tol * np.max(np.abs(ref)), shift
    H.ShiftHamiltonian(0.0)
    ref = z["y_shift0"]
    scale = np.max(np.abs(ref))
    # the same elements in the same order as the on-the-fly kernel, the diagonal summed apart
    assert np.max(np.abs(H.LowLevelMultiply(x) - y_fly)) <= (1e-14 if prec == "fp64" else 1e-6) * scale
    for k in (2, 4):
        X = np.stack([x * c for c in (1.0, -0.5, 2.0, 0.25)[:k]], axis=1)
        Y = H.block_multiply(X)
        for j in range(k):
            c = X[0, j] / x[0]
            assert np.max(np.abs(Y[:, j] - c * ref)) <= tol * abs(c) * scale, (k, j)


def test_long_stored_elements_new_pseudopotentials_and_lanczos(gpu, orc):
    n, s, lz = 4, 70, 0
    z = golden("long_long_n4_2s70_lz0.npz")
    sp = gpu.FermionOnSphereLong(n, lz, s)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, z["v"])
    e_fly = gpu.BasicLanczosAlgorithm(H, 1, 600)
    e_fly.InitializeLanczosAlgorithm(orc.random_vector(3, sp.dim))
    r_fly = e_fly.solve(600)
    assert H.EnableFastMultiplication()[0]
    lz_ = gpu.BasicLanczosAlgorithm(H, 1, 600)
    lz_.InitializeLanczosAlgorithm(orc.random_vector(3, sp.dim))
    r = lz_.solve(600)
    assert abs(r["eigenvalues"][0] - r_fly["eigenvalues"][0]) <= 1e-10 * abs(r_fly["eigenvalues"][0])
    # new pseudopotentials: the stored elements hold factor indices, only the diagonal is recomputed
    v2 = np.array(z["v"]) * 0.5
    v2[1] += 0.25
    H.set_pseudopotentials(v2)
    x = orc.random_vector(4, sp.dim)
    ref = orc.FQHELong(n, s, lz, v2).push(x)
    assert np.max(np.abs(H.LowLevelMultiply(x) - ref)) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.parametrize("space,n,s,lz", [("fermion", 4, 50, 0), ("long", 3, 63, 1), ("long", 3, 126, 0)])
def test_long_pseudopotential_adjoint(gpu, orc, space, n, s, lz):
    # <u|H(V)|v> is linear in V, so g . r = <u|H(r)|v> for any V = r: three random r against the oracle's
    # 128-bit product (2S = 50: shared-memory bins; 63 and above: atomics into the global bins)
    sp = gpu.FermionOnSphere(n, lz, s) if space == "fermion" else gpu.FermionOnSphereLong(n, lz, s)
    v0 = orc.coulomb_pseudopotentials(s)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v0)
    H.ShiftHamiltonian(0.7)  # the shift does not depend on V
    u = orc.random_vector(21, sp.dim)
    w = orc.random_vector(22, sp.dim)
    g = H.pseudopotential_adjoint(u, w)
    rng = np.random.default_rng(5)
    for _ in range(3):
        r = rng.uniform(-1.0, 1.0, s + 1)
        ref = float(u @ orc.FQHELong(n, s, lz, r).push(w))
        assert abs(float(g @ r) - ref) <= 1e-12 * max(1.0, float(np.abs(g) @ np.abs(r)))
    # only odd relative angular momenta enter spin-polarised factors
    assert np.all(g[0::2] == 0.0)
    assert np.max(np.abs(H.pseudopotential_adjoint(w, u) - g)) <= 1e-12 * np.max(np.abs(g))
