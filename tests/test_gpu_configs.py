"""The benchmark configurations themselves against the reference.

Precision configuration (N = 12, 2S = 33, Lz = 0, 7,764,392 states, LLL Coulomb V_m odd m): the full
FP64 product of a seeded vector against the reference's own SMP product (a strided sample of y, its
norm and three dot products; tests/golden/make_golden.py --only product_n12), and the ground energy
of plain FP64 Lanczos and of FP32 products + FP64 refinement against the reference's Lanczos E0 of
the sector (1e-10 relative).

Batching configuration (N = 10, 2S = 27, all 91 sectors 2Lz = 0..180, V_1 = 1, V_3,5,7 uniform in
[0, 0.5) from splitmix64 seed 1): the lowest energy of every sector from the batched block solve
(FP32 + refinement and FP64) against the reference's block Lanczos (k = 4) or full diagonalisation
per sector (1e-10 relative).

Large-spin-chain configuration (J1-J2, J2 = J1/2, Sz = 0): block k = 2, FP32 products + FP64
refinement against the exact E0 = -3L/8 at L = 28 (40,116,600 states) and against the reference
harness's Lanczos E0 at L = 16.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sector_b(gpu):
    z = golden("product_n12_2s33_lz0_coulomb_seed5.npz")
    sp = gpu.FermionOnSphere(12, 0, 33)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 12, 33, z["v"])
    return sp, H, z


@pytest.mark.parametrize("precision, tol", [("fp64", 1e-12), ("fp32", 2e-6)])
def test_precision_config_full_product(gpu, orc, sector_b, precision, tol):
    sp, H, z = sector_b
    dim = sp.dim
    H.set_precision(precision)
    y = H.LowLevelMultiply(orc.random_vector(5, dim))
    scale = float(z["max_abs"])
    assert np.max(np.abs(y[::int(z["stride"])] - z["sample"])) < tol * scale
    assert abs(np.linalg.norm(y) - float(z["norm"])) < tol * float(z["norm"])
    ynorm = float(z["norm"])
    for seed, key in ((6, "dot_seed6"), (7, "dot_seed7"), (5, "x_dot_y")):
        d = float(np.dot(y, orc.random_vector(seed, dim)))
        assert abs(d - float(z[key])) < tol * ynorm, (key, d, float(z[key]))
    H.set_precision("fp64")


def test_precision_config_ground_energy(gpu, sector_b):
    sp, H, _ = sector_b
    e_ref = float(golden("lanczos_n12_2s33_lz0_coulomb_basic.npz")["eigenvalues"][0])
    H.set_precision("fp64")
    lz = gpu.BasicLanczosAlgorithm(H, 1, 600)
    lz.SetEigenvaluePrecision(1e-13)
    lz.InitializeLanczosAlgorithm(seed=0)
    e64 = float(lz.solve(600, graph_batch=16)["eigenvalues"][0])
    assert abs(e64 - e_ref) < 1e-10 * abs(e_ref)
    H.set_precision("fp32")
    for k in (1, 2):
        lzr = gpu.BasicLanczosAlgorithm(H, 1, 600) if k == 1 else gpu.BasicBlockLanczosAlgorithm(H, 1, 600, block_size=k)
        lzr.InitializeLanczosAlgorithm(seed=0)
        r = lzr.solve_refined(600, precision=1e-10)
        assert abs(r["energy"] - e_ref) < 1e-10 * abs(e_ref), (k, r)
        assert r["fp64_matvecs"] > 0
    H.set_precision("fp64")


@pytest.mark.parametrize("memory", [0, -1])
@pytest.mark.parametrize("fp32", [True, False])
def test_batching_config_every_sector_against_reference(gpu, fp32, memory):
    # memory = -1: the batch's elements stored once (one sliced ELL over the concatenated sectors)
    z = golden("sectors_n10_2s27_block4.npz")
    sectors = [int(s) for s in z["two_lz"]]
    assert len(sectors) == 91 and int(z["dims"].sum()) == 6684779
    r = gpu.fqhe_sectors_block_lanczos(10, 27, sectors, z["v"], block_size=2, max_iter=800, precision=1e-10 if fp32 else 1e-13,
                                       fp32=fp32, full_diag_limit=200, memory=memory)
    assert (r["stored_bytes"] > 0) == (memory != 0)
    e_ref = z["e0"]
    rel = np.abs(r["energies"] - e_ref) / np.abs(e_ref)
    assert np.max(rel) < 1e-10, (sectors[int(np.argmax(rel))], float(np.max(rel)))


def test_chain_config_block2_refined_l28(gpu):
    chain = gpu.Spin1_2Chain(28, 0)
    H = gpu.SpinChainJ1J2Hamiltonian(chain, 1.0, 0.5)
    H.set_precision("fp32")
    lz = gpu.BasicBlockLanczosAlgorithm(H, 1, 400, block_size=2)
    lz.InitializeLanczosAlgorithm(seed=0)
    r = lz.solve_refined(400, precision=1e-10)
    exact = -0.375 * 28
    assert abs(r["energy"] - exact) < 1e-10 * abs(exact), r
    assert r["fp32_matvecs"] > 0 and r["fp64_matvecs"] > 0


def test_chain_config_block2_refined_against_reference_l16(gpu):
    z = golden("spin_lanczos_L16_sz0_j1_0.5.npz")
    chain = gpu.Spin1_2Chain(16, 0)
    H = gpu.SpinChainJ1J2Hamiltonian(chain, 1.0, 0.5)
    H.set_precision("fp32")
    lz = gpu.BasicBlockLanczosAlgorithm(H, 1, 400, block_size=2)
    lz.InitializeLanczosAlgorithm(seed=0)
    r = lz.solve_refined(400, precision=1e-10)
    e_ref = float(z["eigenvalues"][0])
    assert abs(r["energy"] - e_ref) < 1e-10 * abs(e_ref), (r, e_ref)
    assert abs(e_ref + 6.0) < 1e-10
