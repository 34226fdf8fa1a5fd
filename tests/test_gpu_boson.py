"""BosonOnSphereShort on the GPU against the reference's fixtures and the oracle:

- the basis: the occupations of the stored words equal the reference's (PrintState) in order, and
  FindStateIndex returns every state's own index;
- the product (ParticleOnSphereGenericHamiltonian on bosons, on the fly): FP64 within 1e-13 and FP32
  within 2e-6 of max|y|, shift 0 and 0.37, single vectors, blocks of 2, 3 and 4 vectors in both
  layouts, and a column range against the oracle's push form;
- Lanczos: the reference's E0 (1e-10 relative, iteration counter within 2) and E0 = 0 (1e-10
  absolute) for the Laughlin state of the delta interaction; block Lanczos and the FP32 + FP64
  refined solve reach the same energy;
- stored elements (EnableFastMultiplication): the same products from device-resident rows, and
  the same Lanczos run;
- the pseudopotential adjoint against products of the oracle with single pseudopotentials;
- what bosons do not offer is refused with an error."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden, parse_sector

pytestmark = pytest.mark.gpu

NAMES = sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "boson_n*.npz")))


def _setup(gpu, name):
    z = golden(name)
    n, s, lz = parse_sector(name)
    sp = gpu.BosonOnSphereShort(n, lz, s)
    return z, sp, gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, z["v"])


@pytest.mark.parametrize("name", NAMES)
def test_boson_basis_matches_reference(gpu, name):
    z, sp, _ = _setup(gpu, name)
    assert sp.dim == z["occupations"].shape[0]
    words, _ = sp.states()
    assert np.array_equal(sp.occupations(words), z["occupations"])
    assert np.array_equal(sp.FindStateIndex(words), np.arange(sp.dim))


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
@pytest.mark.parametrize("name", NAMES)
def test_boson_product_matches_reference(gpu, orc, name, prec, tol):
    z, sp, H = _setup(gpu, name)
    H.set_precision(prec)
    x = orc.random_vector(int(z["seed"]), sp.dim)
    for shift in (0.0, 0.37):
        H.ShiftHamiltonian(shift)
        ref = z["y_shift%g" % shift]
        y = H.LowLevelMultiply(x)
        assert np.max(np.abs(y - ref)) <= tol * np.max(np.abs(ref)), shift
    H.ShiftHamiltonian(0.0)
    ref = z["y_shift0"]
    for k in (2, 3, 4):
        X = np.stack([x * c for c in (1.0, -0.5, 2.0, 0.25)[:k]], axis=1)
        Y = H.block_multiply(X)  # row-interleaved (dim, k)
        for j in range(k):
            c = X[0, j] / x[0]
            assert np.max(np.abs(Y[:, j] - c * ref)) <= tol * abs(c) * np.max(np.abs(ref)), (k, j)
        srcs = np.ascontiguousarray(X.T)
        dsts = np.zeros_like(srcs)
        H.LowLevelMultipleAddMultiply(srcs, dsts)  # vectors one after the other
        for j in range(k):
            c = X[0, j] / x[0]
            assert np.max(np.abs(dsts[j] - c * ref)) <= tol * abs(c) * np.max(np.abs(ref)), (k, j)


@pytest.mark.parametrize("name", ["boson_n7_2s12_lz2_coulomb.npz", "boson_n8_2s8_lz0_coulomb.npz"])
def test_boson_column_range_matches_oracle_push(gpu, orc, name):
    z, sp, H = _setup(gpu, name)
    n, s, lz = parse_sector(name)
    O = orc.BosonFQHE(n, s, lz, z["v"], shift=0.3)
    H.ShiftHamiltonian(0.3)
    x = orc.random_vector(3, sp.dim)
    first, nbr = sp.dim // 5, sp.dim // 3
    y = np.zeros(sp.dim)
    H.LowLevelAddMultiply(x, y, first, nbr)
    ref = O.push(x, first, nbr)
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.parametrize("name", NAMES)
def test_boson_lanczos_matches_reference(gpu, orc, name):
    z, sp, H = _setup(gpu, name)
    lz = gpu.BasicLanczosAlgorithm(H, 1, 400)
    lz.InitializeLanczosAlgorithm(orc.random_vector(int(z["seed"]), sp.dim))
    r = lz.solve(int(z["max_iter"]))
    e_ref = float(z["eigenvalues"][0])
    if bool(z["converged"]):
        assert abs(r["eigenvalues"][0] - e_ref) <= 1e-10 * abs(e_ref)
        assert abs(r["iterations"] - int(z["iterations"])) <= 2
    else:
        assert abs(r["eigenvalues"][0]) < 1e-10  # Laughlin state of the delta interaction


def test_boson_block_and_refined_solves(gpu, orc):
    z, sp, H = _setup(gpu, "boson_n8_2s14_lz0_coulomb.npz")
    e_ref = float(z["eigenvalues"][0])
    b = gpu.BasicBlockLanczosAlgorithm(H, 1, 400, block_size=2)
    b.InitializeLanczosAlgorithm(seed=4)
    rb = b.solve(400)
    assert abs(rb["eigenvalues"][0] - e_ref) <= 1e-10 * abs(e_ref)
    H.set_precision("fp32")
    lz = gpu.BasicLanczosAlgorithmWithGroundState(H, 1, 400)
    lz.InitializeLanczosAlgorithm(seed=5)
    r = lz.solve_refined(400, precision=1e-12)
    assert abs(r["energy"] - e_ref) <= 1e-11 * abs(e_ref)
    psi = lz.GetGroundState()
    H.set_precision("fp64")
    assert abs(H.MatrixElement(psi, psi) - e_ref) <= 1e-10 * abs(e_ref)


def test_boson_errors(gpu, orc):
    z, sp, H = _setup(gpu, "boson_n6_2s10_lz0_coulomb.npz")
    with pytest.raises(gpu.DiagHamError, match="error -4"):
        sp.set_index_mode("lookup")
    with pytest.raises(gpu.DiagHamError, match="not reachable"):
        gpu.BosonOnSphereShort(5, 0, 9)
    # stored elements keep occupation products of at most 16 bosons in 8 bits
    big = gpu.BosonOnSphereShort(17, 0, 2)
    Hb = gpu.ParticleOnSphereGenericHamiltonian(big, 17, 2, np.array([1.0, 0.0, 0.3]))
    with pytest.raises(gpu.DiagHamError, match="error -4"):
        Hb.EnableFastMultiplication()
    # new pseudopotentials are taken by the boson tables too
    v2 = np.array(z["v"]) * 0.5
    H.set_pseudopotentials(v2)
    x = orc.random_vector(1, sp.dim)
    ref = orc.BosonFQHE(6, 10, 0, v2).pull(x)
    assert np.max(np.abs(H.LowLevelMultiply(x) - ref)) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
@pytest.mark.parametrize("name", NAMES)
def test_boson_stored_elements_match_reference(gpu, orc, name, prec, tol):
    # EnableFastMultiplication on BosonOnSphereShort (AbstractQHEOnSphereHamiltonian.cc:3625, 3814):
    # every row's (target, factor, occupation products) in device memory, then products from them
    z, sp, H = _setup(gpu, name)
    n, s, lz = parse_sector(name)
    H.set_precision(prec)
    x = orc.random_vector(int(z["seed"]), sp.dim)
    y_fly = H.LowLevelMultiply(x)
    enabled, nbytes = H.EnableFastMultiplication()
    assert enabled and nbytes > 8 * (H.count_elements() - H.count_diagonal_elements())
    for shift in (0.0, 0.37):
        H.ShiftHamiltonian(shift)
        ref = z["y_shift%g" % shift]
        assert np.max(np.abs(H.LowLevelMultiply(x) - ref)) <= tol * np.max(np.abs(ref)), shift
    H.ShiftHamiltonian(0.0)
    ref = z["y_shift0"]
    scale = np.max(np.abs(ref))
    # the same elements as the on-the-fly product, in the same order
    assert np.max(np.abs(H.LowLevelMultiply(x) - y_fly)) <= (1e-15 if prec == "fp64" else 1e-6) * scale
    for k in (2, 4):
        X = np.stack([x * c for c in (1.0, -0.5, 2.0, 0.25)[:k]], axis=1)
        Y = H.block_multiply(X)
        dsts = np.zeros((k, sp.dim))
        H.LowLevelMultipleAddMultiply(np.ascontiguousarray(X.T), dsts)
        for j in range(k):
            c = X[0, j] / x[0]
            assert np.max(np.abs(Y[:, j] - c * ref)) <= tol * abs(c) * scale, (k, j)
            assert np.max(np.abs(dsts[j] - c * ref)) <= tol * abs(c) * scale, (k, j)
    # new pseudopotentials: the stored elements hold factor indices, only the diagonal is recomputed
    v2 = np.array(z["v"]) * 0.5
    v2[0] += 0.25
    H.set_pseudopotentials(v2)
    ref2 = orc.BosonFQHE(n, s, lz, v2).pull(x)
    assert np.max(np.abs(H.LowLevelMultiply(x) - ref2)) <= tol * np.max(np.abs(ref2))


def test_boson_stored_lanczos_matches_reference(gpu, orc):
    z, sp, H = _setup(gpu, "boson_n8_2s14_lz0_coulomb.npz")
    assert H.EnableFastMultiplication()[0]
    lz = gpu.BasicLanczosAlgorithm(H, 1, 400)
    lz.InitializeLanczosAlgorithm(orc.random_vector(int(z["seed"]), sp.dim))
    r = lz.solve(int(z["max_iter"]))
    e_ref = float(z["eigenvalues"][0])
    assert abs(r["eigenvalues"][0] - e_ref) <= 1e-10 * abs(e_ref)
    assert abs(r["iterations"] - int(z["iterations"])) <= 2


@pytest.mark.parametrize("name", ["boson_n6_2s10_lz0_v0.npz", "boson_n7_2s12_lz2_coulomb.npz",
                                  "boson_n8_2s14_lz0_coulomb.npz"])
def test_boson_pseudopotential_adjoint(gpu, orc, name):
    # <u|H(V)|v> is linear in V: its derivative along V_m is <u|H(e_m)|v>, the product of the oracle
    # with the single pseudopotential V_m = 1
    z, sp, H = _setup(gpu, name)
    n, s, lz = parse_sector(name)
    u = orc.random_vector(11, sp.dim)
    v = orc.random_vector(12, sp.dim)
    H.ShiftHamiltonian(0.5)  # the shift does not depend on V
    g = H.pseudopotential_adjoint(u, v)
    ref = np.array([float(u @ orc.BosonFQHE(n, s, lz, np.eye(s + 1)[m]).pull(v)) for m in range(s + 1)])
    assert np.max(np.abs(g - ref)) <= 1e-12 * np.max(np.abs(ref))
    # symmetric H: swapping the vectors gives the same derivative
    assert np.max(np.abs(H.pseudopotential_adjoint(v, u) - g)) <= 1e-12 * np.max(np.abs(ref))
    # with u = v the chain rule of <v|H|v> / <v|v> against a difference of energies
    e = lambda vv: float(v @ orc.BosonFQHE(n, s, lz, vv).pull(v)) / float(v @ v)
    vv = np.array(z["v"])
    gv = H.pseudopotential_adjoint(v, v) / float(v @ v)
    m = 0
    h = 1e-3
    fd = (e(vv + h * np.eye(s + 1)[m]) - e(vv - h * np.eye(s + 1)[m])) / (2 * h)
    assert abs(gv[m] - fd) <= 1e-9 * max(1.0, abs(fd))


def test_boson_element_counts(gpu):
    # moves per row: every pair m1 >= m2 that a_m1 a_m2 can empty, times its creations m3 >= m4, one of
    # which (m3 = m1) returns to the row
    z, sp, H = _setup(gpu, "boson_n7_2s12_lz2_coulomb.npz")
    L = 12
    moves = diag = 0
    for row in z["occupations"]:
        for m1 in range(L + 1):
            if row[m1] == 0:
                continue
            for m2 in range(m1 + 1):
                if row[m2] == 0 or (m2 == m1 and row[m1] < 2):
                    continue
                M = m1 + m2
                moves += min(M, L) - (M + 1) // 2 + 1
                diag += 1
    assert H.count_elements() == moves
    assert H.count_diagonal_elements() == diag
    f = gpu.FermionOnSphere(7, 2, 18)
    Hf = gpu.ParticleOnSphereGenericHamiltonian(f, 7, 18, gpu.coulomb_pseudopotentials(18))
    assert Hf.count_diagonal_elements() == 21 * f.dim


@pytest.mark.parametrize("n,s,lz", [(1, 6, 2), (16, 2, 0), (16, 3, 2), (2, 0, 0)])
def test_boson_stored_elements_edge_sectors(gpu, orc, n, s, lz):
    # one boson (no pairs: only the shift), sixteen bosons (the largest occupation products a stored
    # element holds: 16 x 15 = 240), and a single orbital
    v = np.linspace(1.0, 0.1, s + 1)
    sp = gpu.BosonOnSphereShort(n, lz, s)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v)
    H.ShiftHamiltonian(0.25)
    x = orc.random_vector(9, sp.dim)
    ref = orc.BosonFQHE(n, s, lz, v, shift=0.25).pull(x)
    assert np.max(np.abs(H.LowLevelMultiply(x) - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))
    assert H.EnableFastMultiplication()[0]
    assert np.max(np.abs(H.LowLevelMultiply(x) - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))
