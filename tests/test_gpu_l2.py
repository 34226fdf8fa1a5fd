"""L^2 on the GPU: the ParticleOnSphereL2Hamiltonian product against the reference's (FP64 1e-13,
FP32 2e-6 of max|y|) in every product form (single vector, row-interleaved blocks, stored
elements); the l2Factor term of the generic Hamiltonian as V + l2Factor L^2; and the total angular
momentum of Lanczos ground states: L = 0 for the Laughlin state (V1 only, 2S = 3(N-1)) and integer
L (within 1e-8) for Coulomb ground states of other sectors."""
import numpy as np
import pytest

from conftest import golden, parse_sector

pytestmark = pytest.mark.gpu

TAGS = ["n6_2s15_lz0", "n6_2s15_lz4", "n7_2s18_lz2", "n8_2s21_lz0", "n8_2s21_lz6"]


def _l2(gpu, tag, l2_factor=1.0):
    n, s, lz = parse_sector(tag)
    sp = gpu.FermionOnSphere(n, lz, s)
    return sp, gpu.ParticleOnSphereL2Hamiltonian(sp, n, s, lz, l2_factor)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
@pytest.mark.parametrize("tag", TAGS)
def test_l2_product_matches_reference(gpu, orc, tag, prec, tol):
    z = golden("l2_%s.npz" % tag)
    sp, L2 = _l2(gpu, tag)
    L2.set_precision(prec)
    x = orc.random_vector(int(z["seed"]), sp.dim)
    y = L2.LowLevelMultiply(x)
    assert np.max(np.abs(y - z["y"])) <= tol * np.max(np.abs(z["y"]))
    X = np.stack([x, 2.0 * x, -x, 0.5 * x], axis=1)
    Y = L2.block_multiply(X)
    for j, c in enumerate((1.0, 2.0, -1.0, 0.5)):
        assert np.max(np.abs(Y[:, j] - c * z["y"])) <= tol * abs(c) * np.max(np.abs(z["y"]))
    assert L2.EnableFastMultiplication()[0]
    y = L2.LowLevelMultiply(x)
    assert np.max(np.abs(y - z["y"])) <= tol * np.max(np.abs(z["y"]))


def test_generic_hamiltonian_with_l2_term(gpu, orc):
    z = golden("l2_n8_2s21_lz6.npz")
    v = golden("lanczos_n8_2s21_lz0_coulomb_basic.npz")["v"]
    sp = gpu.FermionOnSphere(8, 6, 21)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 8, 21, v, l2_factor=0.3)
    x = orc.random_vector(int(z["seed"]), sp.dim)
    ref = orc.FQHE(8, 21, 6, v).pull(x) + 0.3 * z["y"]
    y = H.LowLevelMultiply(x)
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))
    H.ShiftHamiltonian(1.5)  # the user shift adds to the L^2 constant
    y = H.LowLevelMultiply(x)
    assert np.max(np.abs(y - ref - 1.5 * x)) <= 1e-13 * np.max(np.abs(ref))
    # the adjoint still differentiates the interaction only
    g = H.pseudopotential_adjoint(x, x)
    g0 = gpu.ParticleOnSphereGenericHamiltonian(sp, 8, 21, v).pseudopotential_adjoint(x, x)
    assert np.max(np.abs(g - g0)) <= 1e-12 * np.max(np.abs(g0))


def test_laughlin_state_has_zero_angular_momentum(gpu):
    v = np.zeros(16)
    v[1] = 1.0
    sp = gpu.FermionOnSphere(6, 0, 15)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 6, 15, v)
    lz = gpu.BasicLanczosAlgorithmWithGroundState(H, 1, 300)
    lz.InitializeLanczosAlgorithm(seed=1)
    r = lz.solve(300)
    assert abs(r["eigenvalues"][0]) < 1e-10
    psi = lz.GetGroundState()
    L2 = gpu.ParticleOnSphereL2Hamiltonian(sp, 6, 15, 0)
    assert L2.total_angular_momentum(psi) < 1e-6


@pytest.mark.parametrize("tag", ["n7_2s18_lz2", "n8_2s21_lz6"])
def test_ground_states_have_integer_angular_momentum(gpu, tag):
    n, s, lz = parse_sector(tag)
    v = gpu.coulomb_pseudopotentials(s)
    v[0::2] = 0.0
    sp = gpu.FermionOnSphere(n, lz, s)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v)
    lzz = gpu.BasicLanczosAlgorithmWithGroundState(H, 1, 400)
    lzz.InitializeLanczosAlgorithm(seed=2)
    lzz.solve(400)
    psi = lzz.GetGroundState()
    L = gpu.ParticleOnSphereL2Hamiltonian(sp, n, s, lz).total_angular_momentum(psi)
    assert abs(L - round(L)) < 1e-6 and round(L) >= abs(lz) / 2, L


BOSON_TAGS = ["n6_2s10_lz0", "n5_2s9_lz1", "n7_2s12_lz2", "n8_2s14_lz0", "n8_2s8_lz4"]


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
@pytest.mark.parametrize("tag", BOSON_TAGS)
def test_boson_l2_product_matches_reference(gpu, orc, tag, prec, tol):
    # the bosonic branch of ParticleOnSphereL2Hamiltonian on BosonOnSphereShort, single vectors and blocks
    z = golden("boson_l2_%s.npz" % tag)
    n, s, lz = parse_sector(tag)
    sp = gpu.BosonOnSphereShort(n, lz, s)
    L2 = gpu.ParticleOnSphereL2Hamiltonian(sp, n, s, lz)
    L2.set_precision(prec)
    x = orc.random_vector(int(z["seed"]), sp.dim)
    y = L2.LowLevelMultiply(x)
    assert np.max(np.abs(y - z["y"])) <= tol * np.max(np.abs(z["y"]))
    X = np.stack([x, 2.0 * x, -x, 0.5 * x], axis=1)
    Y = L2.block_multiply(X)
    for j, c in enumerate((1.0, 2.0, -1.0, 0.5)):
        assert np.max(np.abs(Y[:, j] - c * z["y"])) <= tol * abs(c) * np.max(np.abs(z["y"]))


def test_boson_generic_hamiltonian_with_l2_term(gpu, orc):
    z = golden("boson_l2_n8_2s14_lz0.npz")
    v = golden("boson_n8_2s14_lz0_coulomb.npz")["v"]
    sp = gpu.BosonOnSphereShort(8, 0, 14)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 8, 14, v, l2_factor=0.3)
    x = orc.random_vector(int(z["seed"]), sp.dim)
    ref = orc.BosonFQHE(8, 14, 0, v).pull(x) + 0.3 * z["y"]
    y = H.LowLevelMultiply(x)
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_bosonic_laughlin_state_has_zero_angular_momentum(gpu):
    # nu = 1/2 bosonic Laughlin state: the zero-energy ground state of the delta interaction V_0 at
    # 2S = 2 (N - 1), an L = 0 singlet
    n, s = 6, 10
    v = np.zeros(s + 1)
    v[0] = 1.0
    sp = gpu.BosonOnSphereShort(n, 0, s)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v)
    lz = gpu.BasicLanczosAlgorithmWithGroundState(H, 1, 300)
    lz.InitializeLanczosAlgorithm(seed=1)
    r = lz.solve(300)
    assert abs(r["eigenvalues"][0]) < 1e-10
    psi = lz.GetGroundState()
    L2 = gpu.ParticleOnSphereL2Hamiltonian(sp, n, s, 0)
    assert L2.total_angular_momentum(psi) < 1e-6
