"""Block Lanczos over all Lz sectors in lockstep (one launch per block product) against the
reference's block Lanczos, the single-vector GPU Lanczos and dense diagonalisation of the oracle's
Hamiltonian.  Energies within 1e-10 relative (FP64 products) and after FP64 refinement of FP32."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def dense_e0(orc, n, s, lz, v):
    O = orc.FQHE(n, s, lz, v)
    d = O.dim
    H = np.zeros((d, d))
    for j in range(d):
        e = np.zeros(d)
        e[j] = 1.0
        H[:, j] = O.pull(e)
    return float(np.linalg.eigvalsh(0.5 * (H + H.T))[0])


def test_matches_reference_block_lanczos(gpu):
    z = golden("lanczos_n6_2s15_lz0_coulomb_block4.npz")
    r = gpu.fqhe_sectors_block_lanczos(6, 15, [0], z["v"], block_size=4, max_iter=400, full_diag_limit=0)
    e_ref = float(z["eigenvalues"][0])
    assert abs(r["energies"][0] - e_ref) < 1e-10 * abs(e_ref)


@pytest.mark.parametrize("k", [1, 2, 4])
def test_all_sectors_against_dense(gpu, orc, k):
    v = golden("lanczos_n6_2s15_lz0_coulomb_block4.npz")["v"]
    sectors = list(range(0, 31, 2))  # 2Lz = 0 .. 30 for N = 6, 2S = 15 (the top sectors are tiny)
    r = gpu.fqhe_sectors_block_lanczos(6, 15, sectors, v, block_size=k, max_iter=600, full_diag_limit=16)
    for lz, e in zip(sectors, r["energies"]):
        ref = dense_e0(orc, 6, 15, lz, v)
        assert abs(e - ref) < 1e-10 * max(1.0, abs(ref)), (lz, e, ref)


def test_fp32_products_refined_to_fp64(gpu, orc):
    v = golden("lanczos_n8_2s21_lz0_coulomb_basic.npz")["v"]
    sectors = [0, 2, 4, 6]
    r64 = gpu.fqhe_sectors_block_lanczos(8, 21, sectors, v, block_size=4, max_iter=800)
    r32 = gpu.fqhe_sectors_block_lanczos(8, 21, sectors, v, block_size=4, max_iter=800, fp32=True, precision=1e-12)
    e_basic = float(golden("lanczos_n8_2s21_lz0_coulomb_basic.npz")["eigenvalues"][0])
    assert abs(r64["energies"][0] - e_basic) < 1e-10 * abs(e_basic)
    assert np.max(np.abs(r32["energies"] - r64["energies"]) / np.abs(r64["energies"])) < 1e-10, (r32, r64)
    assert r32["refined_sectors"] >= 1 and 0 < r32["max_refine_shift"] < 1e-5
    assert r64["block_products"] > 0 and r64["product_seconds"] > 0 and r64["refined_sectors"] == 0


@pytest.mark.parametrize("k", [2, 4])
def test_every_sector_fp32_refined_against_dense(gpu, orc, k):
    # all 31 sectors 2Lz = 0 .. 60 of N = 6, 2S = 15, dimensions 1 .. 1242
    v = golden("lanczos_n6_2s15_lz0_coulomb_block4.npz")["v"]
    sectors = list(range(0, 61, 2))
    r = gpu.fqhe_sectors_block_lanczos(6, 15, sectors, v, block_size=k, max_iter=600, fp32=True, precision=1e-13,
                                       full_diag_limit=16)
    for lz, e in zip(sectors, r["energies"]):
        ref = dense_e0(orc, 6, 15, lz, v)
        assert abs(e - ref) < 1e-10 * max(1.0, abs(ref)), (lz, e, ref)


@pytest.mark.parametrize("k", [1, 2, 4])
def test_all_sectors_stored_elements_against_dense(gpu, orc, k):
    # the batch's stored elements (one ELL over the concatenated sectors, converged sectors skipped):
    # FP64 and FP32 + refinement, against dense diagonalisation and the on-the-fly batch
    v = golden("lanczos_n6_2s15_lz0_coulomb_block4.npz")["v"]
    sectors = list(range(0, 61, 2))
    r_fly = gpu.fqhe_sectors_block_lanczos(6, 15, sectors, v, block_size=k, max_iter=600, full_diag_limit=16)
    r64 = gpu.fqhe_sectors_block_lanczos(6, 15, sectors, v, block_size=k, max_iter=600, full_diag_limit=16, memory=-1)
    r32 = gpu.fqhe_sectors_block_lanczos(6, 15, sectors, v, block_size=k, max_iter=600, fp32=True, precision=1e-13,
                                         full_diag_limit=16, memory=-1)
    assert r64["stored_bytes"] > 0 and r32["stored_bytes"] > 0 and r_fly["stored_bytes"] == 0
    for lz, e_fly, e64, e32 in zip(sectors, r_fly["energies"], r64["energies"], r32["energies"]):
        ref = dense_e0(orc, 6, 15, lz, v)
        assert abs(e64 - ref) < 1e-10 * max(1.0, abs(ref)), (lz, e64, ref)
        assert abs(e32 - ref) < 1e-10 * max(1.0, abs(ref)), (lz, e32, ref)
        assert abs(e64 - e_fly) < 1e-11 * max(1.0, abs(ref)), (lz, e64, e_fly)
    # a budget below the structure's size keeps the products on the fly
    r_small = gpu.fqhe_sectors_block_lanczos(6, 15, sectors, v, block_size=k, max_iter=600, full_diag_limit=16,
                                             memory=1024)
    assert r_small["stored_bytes"] == 0


def test_fp32_refined_restarts_from_stored_elements(gpu, orc):
    # a stored batch restarts the sectors it could not certify from stored elements of their own
    v = golden("lanczos_n8_2s21_lz0_coulomb_basic.npz")["v"]
    sectors = [0, 2, 4, 6]
    r64 = gpu.fqhe_sectors_block_lanczos(8, 21, sectors, v, block_size=4, max_iter=800)
    r32 = gpu.fqhe_sectors_block_lanczos(8, 21, sectors, v, block_size=4, max_iter=800, fp32=True, precision=1e-12,
                                         memory=-1)
    assert r32["stored_bytes"] > 0 and r32["refined_sectors"] >= 1
    assert np.max(np.abs(r32["energies"] - r64["energies"]) / np.abs(r64["energies"])) < 1e-10, (r32, r64)
