"""The oracle (CPU restatement of the reference path) pinned against the reference's own outputs.

Every fixture was produced by the reference compiled from its sources (tests/golden/make_golden.py);
the oracle must reproduce integer results bit for bit and FP64 results to rounding.
"""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden, parse_sector


@pytest.mark.parametrize("name", sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "fqhe_basis_*.npz"))))
def test_fermion_basis_bit_exact(orc, name):
    z = golden(name)
    n, s, lz = parse_sector(name)
    words, lzmax = orc.fermion_basis(n, s, lz)
    assert np.array_equal(words, z["words"])
    assert np.array_equal(lzmax, z["lzmax"])
    # TestFindAllStates invariant of the reference (AbstractHilbertSpace.h:127)
    assert np.array_equal(z["find"], np.arange(len(words)))


def test_documented_basis_order(orc):
    # FQHE/docs/DataFormat/FermionOnSphere.xml:19-40: N = 4, S = 4, Lz = 1, first and last states
    words, _ = orc.fermion_basis(4, 8, 2)
    assert len(words) == 11
    assert int(words[0]) == 0b110000101 and int(words[-1]) == 0b001110100


def test_lookup_table_find_state_index(orc):
    z = golden("fqhe_basis_n8_2s21_lz0.npz")
    for shift in (17, 9, 4, 1):
        H = orc.FQHE(8, 21, 0, np.eye(22)[1], max_shift=shift)
        for i in range(0, H.dim, 37):
            assert H.find(z["words"][i]) == i


@pytest.mark.parametrize("two_s", [8, 21, 27, 33])
def test_coulomb_pseudopotentials(orc, two_s):
    v = orc.coulomb_pseudopotentials(two_s)
    ref = golden("pseudopotentials_2s%d.npz" % two_s)["v"]
    assert np.max(np.abs(v - ref) / np.abs(ref)) < 1e-13


@pytest.mark.parametrize("name", ["factors_2s21_v1.npz", "factors_2s27_coulomb.npz", "factors_2s33_coulomb.npz"])
def test_interaction_factors(orc, name):
    z = golden(name)
    two_s = int(name.split("_")[1][2:])
    t = orc.interaction_tables(two_s, z["v"])
    assert np.array_equal(t["m1"], z["m1"]) and np.array_equal(t["m2"], z["m2"])
    assert np.array_equal(t["nbr_m3"], z["nbr_m3"]) and np.array_equal(t["m3"], z["m3"])
    scale = np.max(np.abs(z["factors"]))
    assert np.max(np.abs(t["factors"] - z["factors"])) < 1e-13 * scale


def test_interaction_derivatives_linear(orc):
    z = golden("factors_2s27_coulomb.npz")
    d = orc.interaction_derivatives(27)
    assert np.max(np.abs(d @ z["v"] - z["factors"])) < 1e-13 * np.max(np.abs(z["factors"]))


def test_clebsch_gordan_orthonormal(orc):
    # sum_J <j1 m1 j2 m2|J M><j1 m1' j2 m2'|J M> = delta for j1 = j2 = 33/2 (doubled projections)
    j = 33
    for M in (2, 14):
        ms = [m for m in range(-j, j + 1, 2) if abs(M - m) <= j]
        Js = list(range(abs(M), 2 * j + 1, 2))
        C = np.array([[orc.clebsch_gordan(j, m, j, M - m, J) for J in Js] for m in ms])
        assert np.max(np.abs(C @ C.T - np.eye(len(ms)))) < 1e-13


@pytest.mark.parametrize("name", ["rows_n8_2s21_lz0_v1.npz", "rows_n8_2s21_lz0_coulomb.npz",
                                  "rows_n7_2s18_lz2_coulomb.npz", "rows_n10_2s27_lz0_coulomb.npz"])
def test_row_elements_bit_exact(orc, name):
    z = golden(name)
    n, s, lz = parse_sector(name)
    H = orc.FQHE(n, s, lz, z["v"])
    for k, r in enumerate(z["rows"]):
        a, b = z["offsets"][k], z["offsets"][k + 1]
        t, sg, f = H.row(int(r))
        assert np.array_equal(t, z["targets"][a:b])
        assert np.array_equal(sg, z["signs"][a:b])
        assert np.array_equal(f, z["factor_index"][a:b])


@pytest.mark.parametrize("tag", ["n8_2s21_lz0_v1", "n8_2s21_lz0_coulomb", "n7_2s18_lz2_coulomb"])
@pytest.mark.parametrize("shift", [0.0, 0.37])
def test_matvec_push_and_pull(orc, tag, shift):
    z = golden("matvec_%s_shift%g.npz" % (tag, shift))
    n, s, lz = parse_sector(tag)
    H = orc.FQHE(n, s, lz, z["v"], shift=shift)
    x = orc.random_vector(0, H.dim)
    tol = 1e-13 * max(1.0, np.max(np.abs(z["y"])))
    assert np.max(np.abs(H.push(x) - z["y"])) < tol
    assert np.max(np.abs(H.pull(x) - z["y"])) < tol


@pytest.mark.parametrize("tag,algo", [("n8_2s21_lz0_coulomb", "basic"), ("n8_2s21_lz0_v1", "basic"),
                                      ("n7_2s18_lz2_coulomb", "basic")])
def test_lanczos_energy_and_iterations(orc, tag, algo):
    z = golden("lanczos_%s_%s.npz" % (tag, algo))
    n, s, lz = parse_sector(tag)
    H = orc.FQHE(n, s, lz, z["v"])
    r = H.lanczos(orc.random_vector(0, H.dim), 1, int(z["max_iter"]), 1e-14)
    e_ref = float(z["eigenvalues"][0])
    assert abs(r["eigenvalues"][0] - e_ref) <= 1e-10 * max(abs(e_ref), 1.0)
    assert r["iterations"] == int(z["iterations"]) and r["converged"] == bool(z["converged"])


def test_laughlin_exact_zero(orc):
    z = golden("lanczos_n8_2s21_lz0_v1_basic.npz")
    assert abs(float(z["eigenvalues"][0])) < 1e-10


def test_hellmann_feynman_expectation(orc):
    # <psi|H_m|psi> of the reference ground state, from the oracle's per-factor bins
    z = golden("lanczos_n8_2s21_lz0_coulomb_ground.npz")
    H = orc.FQHE(8, 21, 0, z["v"])
    r = H.lanczos(orc.random_vector(0, H.dim), 1, 200, 1e-14)
    assert abs(r["eigenvalues"][0] - z["energy_expectation"]) < 1e-10


@pytest.mark.parametrize("name", sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "spin_basis_*.npz"))))
def test_spin_basis_bit_exact(orc, name):
    z = golden(name)
    L = int(name.split("_")[2][1:])
    sz = int(name.split("_")[3][2:-4])
    w = orc.spin_basis(L, sz)
    assert np.array_equal(w, z["words"])
    assert np.array_equal(z["find"], np.arange(len(w)))
    for i in range(0, len(w), max(1, len(w) // 50)):
        assert orc.spin_find(L, sz, w[i]) == i


@pytest.mark.parametrize("name", sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "spin_matvec_*.npz"))))
def test_spin_matvec(orc, name):
    z = golden(name)
    parts = name[:-4].split("_")
    L, sz = int(parts[2][1:]), int(parts[3][2:])
    j1, j2 = float(parts[4][1:]), float(parts[5])
    w = orc.spin_basis(L, sz)
    x = orc.random_vector(3, len(w))
    y = orc.spin_j1j2_multiply(L, sz, w, j1, j2, x)
    assert np.max(np.abs(y - z["y"])) < 1e-13


def test_spin_majumdar_ghosh(orc):
    z = golden("spin_lanczos_L16_sz0_j1_0.5.npz")
    assert abs(float(z["eigenvalues"][0]) + 6.0) < 1e-10  # E0 = -3L/8
    w = orc.spin_basis(16, 0)
    r = orc.python_lanczos(lambda v: orc.spin_j1j2_multiply(16, 0, w, 1.0, 0.5, v), len(w),
                           orc.random_vector(0, len(w)), 1, 400, 1e-14)
    assert abs(r["eigenvalues"][0] + 6.0) < 1e-10


def test_random_vector_matches_fixture_generator(orc):
    from golden.make_golden import splitmix_vector
    a = orc.random_vector(7, 1000)
    b = splitmix_vector(7, 1000)
    assert np.max(np.abs(a - b)) < 1e-15


def test_block_lanczos_fixture_against_dense(orc):
    # the reference's BasicBlockLanczosAlgorithm (k = 4) against a dense diagonalisation of the
    # oracle's Hamiltonian for N = 6, 2S = 15, Lz = 0 (dimension 338)
    z = golden("lanczos_n6_2s15_lz0_coulomb_block4.npz")
    H = orc.FQHE(6, 15, 0, z["v"])
    M = np.stack([H.pull(np.eye(H.dim)[j]) for j in range(H.dim)], axis=1)
    w = np.linalg.eigvalsh(0.5 * (M + M.T))
    assert abs(w[0] - float(z["eigenvalues"][0])) < 1e-10 * abs(w[0])
    assert bool(z["converged"])


@pytest.mark.parametrize("tag", ["n6_2s15_lz0", "n6_2s15_lz4", "n7_2s18_lz2", "n8_2s21_lz0", "n8_2s21_lz6"])
def test_l2_table_matches_reference(orc, tag):
    # the oracle's two-body form of L^2 (plus its constant) against the reference's
    # ParticleOnSphereL2Hamiltonian product, and <x|L^2|x> against |L+ x|^2 + Lz (Lz + 1)
    z = golden("l2_%s.npz" % tag)
    n, s, lz = parse_sector(tag)
    O = orc.FQHE(n, s, lz, np.zeros(s + 1))
    f, c = orc.l2_factors(n, s, lz)
    O.tabs["factors"][:len(f)] = f
    x = orc.random_vector(int(z["seed"]), O.dim)
    y = O.pull(x) + c * x
    assert np.max(np.abs(y - z["y"])) <= 1e-13 * np.max(np.abs(z["y"]))
    if O.dim < 2000:
        up = orc.l2_raise(n, s, lz, x)
        assert abs(float(x @ y) - (float(up @ up) + c)) <= 1e-12 * abs(float(x @ y))


def disk_files(z, prefix):
    return {str(n): bytes(z["%s_f%d" % (prefix, i)]) for i, n in enumerate(z["%s_names" % prefix])}


@pytest.mark.parametrize("fmt", ["basic", "ground"])
def test_disk_state_files_of_the_reference(orc, fmt):
    # what the reference's disk-storage classes leave on disk after 14 iterations, read with the
    # oracle's parsers: V1 = v_Index, V2 = v_Index+1 (normalised), V3 = H V2, the last tridiagonal
    # elements are <V1|V3> and <V2|V3>, the first is <v0|H|v0>; the ground-state format also
    # stores the start vector as vector.0
    z = golden("disk_%s_n7_2s18_lz2.npz" % fmt)
    files = disk_files(z, "interrupted")
    st = orc.read_lanczos_state(files["lanczos.dat"], fmt)
    O = orc.FQHE(7, 18, 2, z["v"])
    names = st["names"] if fmt == "basic" else ["vector.1", "vector.2", "vector.3"]
    v1, v2, v3 = (orc.read_vector_bytes(files[n]) for n in names)
    i = st["index"]
    assert i == int(z["stop"]) - 3 and st["nbr_row"] == i + 2 and st["precision"] == 1e-14
    assert abs(v1 @ v1 - 1) < 1e-13 and abs(v2 @ v2 - 1) < 1e-13
    hv2 = O.pull(v2)
    assert np.max(np.abs(v3 - hv2)) <= 1e-13 * np.max(np.abs(hv2))
    assert abs(st["upper"][i] - v1 @ v3) < 1e-12 and abs(st["diag"][i + 1] - v2 @ v3) < 1e-12
    x0 = orc.random_vector(int(z["seed"]), O.dim)
    assert abs(st["diag"][0] - x0 @ O.pull(x0)) < 1e-12
    if fmt == "ground":
        assert st["ground_flag"] == 0 and st["nbr_eigenvalue"] == 1
        assert np.max(np.abs(orc.read_vector_bytes(files["vector.0"]) - x0)) < 1e-15
        # the state left by an interrupted ground-state assembly: flag 1 and the finished run's matrix
        a = orc.read_lanczos_state(disk_files(z, "assembly")["lanczos.dat"], fmt)
        assert a["ground_flag"] == 1
        e = orc.tridiagonal_eigenvalues(a["diag"], a["upper"])
        assert abs(e.min() - float(z["full_eigenvalue"])) < 1e-13 * abs(float(z["full_eigenvalue"]))
    # the resumed reference run ends where the uninterrupted one does
    assert int(z["resumed_iterations"]) + int(z["stop"]) == int(z["full_iterations"])
    assert float(z["resumed_eigenvalue"]) == float(z["full_eigenvalue"])


BOSON_FIXTURES = sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "boson_n*.npz")))


@pytest.mark.parametrize("name", BOSON_FIXTURES)
def test_boson_oracle_matches_reference(orc, name):
    # BosonOnSphereShort: the basis (occupations of the fermionic words, in the reference's order),
    # the product at shift 0 and 0.37 (push and pull forms), and the Lanczos ground-state energy
    z = golden(name)
    n, s, lz = parse_sector(name)
    O = orc.BosonFQHE(n, s, lz, z["v"])
    assert O.dim == z["occupations"].shape[0]
    assert np.array_equal(O.occupations(), z["occupations"])
    x = orc.random_vector(int(z["seed"]), O.dim)
    for shift in (0.0, 0.37):
        O.s.shift = shift
        ref = z["y_shift%g" % shift]
        tol = 1e-13 * np.max(np.abs(ref))
        assert np.max(np.abs(O.pull(x) - ref)) <= tol
        assert np.max(np.abs(O.push(x) - ref)) <= tol
    O.s.shift = 0.0
    e_ref = float(z["eigenvalues"][0])
    if bool(z["converged"]):
        r = O.lanczos(x, max_iter=int(z["max_iter"]))
        assert abs(r["eigenvalues"][0] - e_ref) <= 1e-10 * abs(e_ref)
        assert abs(r["iterations"] - int(z["iterations"])) <= 2
    else:
        # the Laughlin state of the delta interaction at 2S = 2 (N - 1): E0 = 0
        assert abs(e_ref) < 1e-12


def test_entanglement_oracle_matches_reference(orc):
    # FermionOnSphere::EvaluatePartialEntanglementMatrix / EvaluatePartialDensityMatrix of a vector on
    # N=8 2S=21 2Lz=0: the oracle's M equals the reference's for every regular cut, and the reference's
    # rho is M M^T
    z = golden("entanglement_n8_2s21_lz0.npz")
    x = orc.random_vector(int(z["seed"]), 8512)
    for l, na, lza in z["cases"]:
        tag = "l%d_na%d_lz%d" % (l, na, lza)
        ref = z["m_" + tag]
        if 0 < l <= 21:
            m = orc.entanglement_matrix(8, 21, 0, x, int(l), int(na), int(lza))
            assert m.shape == ref.shape, tag
            # the start vector's normalisation may differ in the last bit between generators
            assert m.size == 0 or np.max(np.abs(m - ref)) <= 1e-15, tag
        if "rho_" + tag in z.files and ref.size and na > 1:
            assert np.max(np.abs(ref @ ref.T - z["rho_" + tag])) < 1e-15, tag


TRANSLATION_FIXTURES = sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "translations_L*.npz")))


@pytest.mark.parametrize("name", TRANSLATION_FIXTURES)
def test_translation_oracle_matches_reference(orc, name):
    # Spin1_2ChainWithTranslations + SpinChainJ1J2RealHamiltonianWithTranslations: the representatives
    # bit for bit, the product within 1e-13 of max|y| (sectors up to 2,438 states; the 9,252-state
    # one is checked on the GPU only)
    import re
    z = golden(name)
    L, sz, k = (int(v) for v in re.search(r"L(\d+)_sz(-?\d+)_k(\d+)", name).groups())
    if len(z["words"]) > 3000:
        pytest.skip("large sector: GPU test only")
    reps, _ = orc.translation_basis(L, sz, k)
    assert np.array_equal(reps, z["words"])
    x = orc.random_vector(int(z["seed"]), len(reps))
    y = orc.translation_j1j2_push(L, sz, k, float(z["j1"]), float(z["j2"]), x)
    assert np.max(np.abs(y - z["y"])) <= 1e-13 * np.max(np.abs(z["y"]))


LONG_FIXTURES = sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "long_*.npz")))


def long_sector(name):
    import re
    space, n, s, lz = re.match(r"long_(\w+?)_n(\d+)_2s(\d+)_lz(-?\d+)", name).groups()
    return space, int(n), int(s), int(lz)


@pytest.mark.parametrize("name", [n for n in LONG_FIXTURES if "words" in golden(n).files])
def test_long_oracle_matches_reference(orc, name):
    # FermionOnSphere beyond 2S = 40 and FermionOnSphereLong up to 2S = 126: the words bit for bit, the
    # product at shift 0.37 within 1e-13 of max|y| (FermionOnSphereLong: the reference's product with
    # exact factors in its tables) or within 1e-12 (FermionOnSphere with the reference's own factors,
    # which deviate from the exact ones by up to 3.6e-13 at 2S = 62)
    z = golden(name)
    space, n, s, lz = long_sector(name)
    words = orc.fermion_basis_long(n, s, lz)
    assert words == [int(a) | (int(b) << 64) for a, b in z["words"]]
    H = orc.FQHELong(n, s, lz, z["v"], shift=0.37)
    y = H.push(orc.random_vector(int(z["seed"]), H.dim))
    ref = z["y_shift0.37"]
    tol = 1e-13 if space == "long" else 1e-12
    assert np.max(np.abs(y - ref)) <= tol * np.max(np.abs(ref))


@pytest.mark.parametrize("name", [n for n in LONG_FIXTURES if "words_sha256" in golden(n).files])
def test_long_oracle_basis_matches_reference_digest(orc, name):
    import hashlib
    z = golden(name)
    _, n, s, lz = long_sector(name)
    m = (1 << 64) - 1
    words = np.array([[w & m, w >> 64] for w in orc.fermion_basis_long(n, s, lz)], np.uint64)
    assert words.shape[0] == int(z["dim"])
    assert hashlib.sha256(words.tobytes()).hexdigest() == str(z["words_sha256"])


def _cg_exact(j1, m1, j2, m2, j):
    """Racah's formula in exact rational arithmetic (doubled arguments), rounded once."""
    from fractions import Fraction
    from math import factorial as F
    m = m1 + m2
    a, b, c, d = (j1 + j2 - j) // 2, (j1 - j2 + j) // 2, (j2 - j1 + j) // 2, (j1 + j2 + j) // 2 + 1
    jm1, jp1, jm2, jp2 = (j1 - m1) // 2, (j1 + m1) // 2, (j2 - m2) // 2, (j2 + m2) // 2
    Jm, Jp = (j - m) // 2, (j + m) // 2
    e1, e2 = (j - j2 + m1) // 2, (j - j1 - m2) // 2
    pre = Fraction((j + 1) * F(a) * F(b) * F(c) * F(Jp) * F(Jm) * F(jm1) * F(jp1) * F(jm2) * F(jp2), F(d))
    S = sum(Fraction((-1) ** k, F(k) * F(a - k) * F(jm1 - k) * F(jp2 - k) * F(e1 + k) * F(e2 + k))
            for k in range(max(0, -e1, -e2), min(a, jm1, jp2) + 1))
    v = pre * S * S
    # sqrt of the rational to double precision through an integer square root
    from math import isqrt
    scale = 1 << 200
    r = isqrt(v.numerator * scale * scale // v.denominator)
    return (1 if S >= 0 else -1) * r / scale


@pytest.mark.parametrize("two_s", [62, 100, 126])
def test_clebsch_gordan_exact_at_large_2s(orc, dh, two_s):
    # the pair coefficients <S m1; S m2 | J M> of the interaction factors, oracle and library, against
    # exact rationals (the reference's own evaluation drifts here; see the fixtures above)
    rng = np.random.default_rng(two_s)
    for _ in range(40):
        i1, i2 = (int(v) for v in rng.integers(0, two_s + 1, 2))
        m1, m2 = 2 * i1 - two_s, 2 * i2 - two_s
        J = int(rng.integers(abs(m1 + m2) // 2, two_s + 1)) * 2
        e = _cg_exact(two_s, m1, two_s, m2, J)
        if abs(e) < 1e-200:
            continue
        assert abs(orc.clebsch_gordan(two_s, m1, two_s, m2, J) - e) <= 4.5e-16 * abs(e)
        assert abs(dh.clebsch_gordan(two_s, m1, two_s, m2, J) - e) <= 4.5e-16 * abs(e)


def test_pseudopotentials_at_large_2s(orc, dh):
    # closed form in exact arithmetic (fixture); the reference's EvaluatePseudopotentials is kept in the
    # fixture beside it and agrees to 3e-14 up to 2S = 100 (5% off at 126)
    z = golden("pseudopotentials_large_2s.npz")
    for s in z["sizes"]:
        ref = z["closed_form_%d" % s]
        assert np.max(np.abs(orc.coulomb_pseudopotentials(int(s)) - ref)) <= 1e-14 * np.max(ref)
        assert np.max(np.abs(dh.coulomb_pseudopotentials(int(s)) - ref)) <= 1e-14 * np.max(ref)
        if s <= 100:
            assert np.max(np.abs(z["reference_%d" % s] - ref)) <= 3e-14 * np.max(ref)


COMPLEX_TRANSLATION_FIXTURES = sorted(os.path.basename(f) for f in
                                      glob.glob(os.path.join(GOLDEN, "translations_complex_*.npz")))


@pytest.mark.parametrize("name", COMPLEX_TRANSLATION_FIXTURES)
def test_complex_translation_oracle_matches_reference(orc, name):
    # SpinChainJ1J2HamiltonianWithTranslations at any K: the complex product within 1e-13 of max|y|, and
    # the reference's own dense matrix Hermitian (sectors up to 2,700 states on the CPU)
    import re
    z = golden(name)
    L, sz, k = (int(v) for v in re.search(r"L(\d+)_sz(-?\d+)_k(\d+)", name).groups())
    if "hermitian_error" in z.files:
        assert float(z["hermitian_error"]) < 1e-13
    if len(z["words"]) > 3000:
        pytest.skip("large sector: GPU test only")
    reps, _ = orc.translation_basis(L, sz, k)
    assert np.array_equal(reps, z["words"])
    x = orc.random_vector(int(z["seed_re"]), len(reps)) + 1j * orc.random_vector(int(z["seed_im"]), len(reps))
    y = orc.translation_j1j2_push_complex(L, sz, k, float(z["j1"]), float(z["j2"]), x)
    assert np.max(np.abs(y - z["y"])) <= 1e-13 * np.max(np.abs(z["y"]))


BOSON_LARGE_FIXTURES = sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "boson_large_*.npz")))


@pytest.mark.parametrize("name", BOSON_LARGE_FIXTURES)
def test_boson_large_oracle_matches_reference(orc, name):
    # BosonOnSphereShort with lz_max + N - 1 = 42 to 62: the words bit for bit (or their SHA-256), the
    # product within 1e-13 of max|y| of the reference's product with exact factors in its tables (its
    # own factors deviate from the exact ones by up to 4.8e-12 at 2S = 60)
    import hashlib
    import re
    z = golden(name)
    n, s, lz = (int(v) for v in re.search(r"n(\d+)_2s(\d+)_lz(-?\d+)", name).groups())
    B = orc.BosonFQHE(n, s, lz, z["v"])
    if "words" in z.files:
        assert np.array_equal(B.words, z["words"])
    else:
        assert hashlib.sha256(np.ascontiguousarray(B.words, np.uint64).tobytes()).hexdigest() == str(z["words_sha256"])
    if B.dim > 13000:
        pytest.skip("large sector: GPU product test only")
    y = B.push(orc.random_vector(int(z["seed"]), B.dim))
    assert np.max(np.abs(y - z["y_shift0"])) <= 1e-13 * np.max(np.abs(z["y_shift0"]))


@pytest.mark.parametrize("tag", ["n6_2s10_lz0", "n5_2s9_lz1", "n7_2s12_lz2", "n8_2s14_lz0", "n8_2s8_lz4"])
def test_boson_l2_table_matches_reference(orc, tag):
    # the oracle's bosonic two-body form of L^2 (plus its constant) against the reference's
    # ParticleOnSphereL2Hamiltonian product on BosonOnSphereShort
    z = golden("boson_l2_%s.npz" % tag)
    n, s, lz = parse_sector(tag)
    O = orc.BosonFQHE(n, s, lz, np.zeros(s + 1))
    f, c = orc.boson_l2_factors(n, s, lz)
    O.tabs["factors"][:len(f)] = f
    x = orc.random_vector(int(z["seed"]), O.dim)
    y = O.pull(x) + c * x
    assert np.max(np.abs(y - z["y"])) <= 1e-13 * np.max(np.abs(z["y"]))
