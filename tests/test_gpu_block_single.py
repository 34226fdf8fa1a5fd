"""Block Lanczos on one Hamiltonian (DH_LANCZOS_BLOCK through the Lanczos handle) against the
reference's BasicBlockLanczosAlgorithm run (same start block), dense diagonalisation of the oracle's
Hamiltonian and the exact Majumdar-Ghosh energy -3L/8 of the J1-J2 chain at J2 = J1/2.
Eigenvalues within 1e-10 relative; iteration counters within two block steps of the reference
(FP64 reduction order differs); Ritz vectors orthonormal to 1e-10."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _fqhe(gpu, v, n=6, s=15, lz=0):
    sp = gpu.FermionOnSphere(n, lz, s)
    return sp, gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v)


def _reference_block(orc, dim, k):
    # the fixture's start block: splitmix vectors from seeds 100.. orthonormalised
    q, _ = np.linalg.qr(np.stack([orc.random_vector(100 + b, dim) for b in range(k)], axis=1))
    return np.ascontiguousarray(q.T)


def test_run_loop_matches_reference(gpu, orc):
    z = golden("lanczos_n6_2s15_lz0_coulomb_block4.npz")
    nev, k = int(z["nev"]), 4
    sp, H = _fqhe(gpu, z["v"])
    lz = gpu.BasicBlockLanczosAlgorithm(H, nev, 400, block_size=k)
    lz.InitializeLanczosAlgorithm(_reference_block(orc, sp.dim, k))
    # the reference harness's loop (QHEOnSphereMainTask.cc:732-753 with a block algorithm)
    lz.RunLanczosAlgorithm(nev + 2)
    count = (nev + 3) * k
    hist = []
    while not lz.TestConvergence() and count < 400:
        count += k
        lz.RunLanczosAlgorithm(1)
        hist.append(lz.GetEigenvalues(1)[0])
    e, e_ref = lz.GetEigenvalues(nev), z["eigenvalues"]
    assert np.max(np.abs(e - e_ref) / np.abs(e_ref)) < 1e-10, (e, e_ref)
    assert abs(count - int(z["iterations"])) <= 2 * k
    n = min(12, len(hist), len(z["history"]))
    assert np.max(np.abs(np.array(hist[:n]) - z["history"][:n]) / np.abs(z["history"][:n])) < 1e-9
    m, rows = lz.counters()
    assert rows % k == 0 and m == rows


@pytest.mark.parametrize("k", [1, 2, 4])
def test_solve_against_dense(gpu, orc, k):
    from test_gpu_block import dense_e0
    v = golden("lanczos_n6_2s15_lz0_coulomb_block4.npz")["v"]
    sp, H = _fqhe(gpu, v, lz=2)
    lz = gpu.BasicBlockLanczosAlgorithm(H, 1, 600, block_size=k)
    lz.InitializeLanczosAlgorithm(seed=7)
    r = lz.solve(600)
    ref = dense_e0(orc, 6, 15, 2, v)
    assert r["converged"]
    assert abs(r["eigenvalues"][0] - ref) < 1e-10 * abs(ref), (r, ref)


@pytest.mark.parametrize("keep", [True, False])
def test_eigenstates_stored_or_replayed(gpu, orc, keep):
    v = golden("lanczos_n6_2s15_lz0_coulomb_block4.npz")["v"]
    sp, H = _fqhe(gpu, v)
    lz = gpu.BasicBlockLanczosAlgorithm(H, 2, 400, block_size=2)
    lz.set_vector_storage(keep)
    lz.InitializeLanczosAlgorithm(seed=3)
    r = lz.solve(400)
    psi = lz.GetEigenstates(2)
    assert np.max(np.abs(psi @ psi.T - np.eye(2))) < 1e-10
    O = orc.FQHE(6, 15, 0, v)
    for c in range(2):
        hpsi = O.pull(psi[c])
        e = float(psi[c] @ hpsi)
        assert abs(e - r["eigenvalues"][c]) < 1e-9 * abs(e)
        assert np.linalg.norm(hpsi - e * psi[c]) < 1e-5
    g = lz.GetGroundState()
    assert abs(abs(float(g @ psi[0])) - 1.0) < 1e-12


def test_stored_and_replayed_ritz_vectors_agree(gpu):
    v = golden("lanczos_n6_2s15_lz0_coulomb_block4.npz")["v"]
    out = []
    for keep in (True, False):
        sp, H = _fqhe(gpu, v)
        lz = gpu.BasicBlockLanczosAlgorithm(H, 1, 400, block_size=4)
        lz.set_vector_storage(keep)
        lz.InitializeLanczosAlgorithm(seed=11)
        lz.solve(400)
        out.append(lz.GetGroundState())
    assert abs(abs(float(out[0] @ out[1])) - 1.0) < 1e-12


def test_majumdar_ghosh_chain_fp64_and_fp32_refined(gpu):
    z = golden("spin_lanczos_L16_sz0_j1_0.5.npz")
    exact = -3.0 * 16 / 8
    assert abs(float(z["eigenvalues"][0]) - exact) < 1e-12
    chain = gpu.Spin1_2Chain(16, 0)
    H = gpu.SpinChainJ1J2Hamiltonian(chain, 1.0, 0.5)
    lz = gpu.BasicBlockLanczosAlgorithm(H, 1, 800, block_size=2)
    lz.InitializeLanczosAlgorithm(seed=0)
    r = lz.solve(800)
    assert abs(r["eigenvalues"][0] - exact) < 1e-10 * abs(exact), r
    H.set_precision("fp32")
    lz32 = gpu.BasicBlockLanczosAlgorithm(H, 1, 800, block_size=2)
    lz32.InitializeLanczosAlgorithm(seed=0)
    q = lz32.solve_refined(800, precision=1e-12)
    assert abs(q["energy"] - exact) < 1e-10 * abs(exact), q
    assert q["fp32_matvecs"] > 0 and q["fp64_matvecs"] > 0


def test_fqhe_fp32_refined_block(gpu):
    z = golden("lanczos_n8_2s21_lz0_coulomb_basic.npz")
    sp, H = _fqhe(gpu, z["v"], 8, 21, 0)
    H.set_precision("fp32")
    lz = gpu.BasicBlockLanczosAlgorithm(H, 1, 800, block_size=4)
    lz.InitializeLanczosAlgorithm(seed=0)
    q = lz.solve_refined(800, precision=1e-12)
    e_ref = float(z["eigenvalues"][0])
    assert abs(q["energy"] - e_ref) < 1e-10 * abs(e_ref), q
    assert abs(q["energy_fp32"] - e_ref) < 1e-6 * abs(e_ref)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_exhausted_space_falls_back_to_dense(gpu, orc, prec):
    # 2Lz = 42 of N = 6, 2S = 15 has dimension 26: with k = 4 the last block only has rank 2
    from test_gpu_block import dense_e0
    v = golden("lanczos_n6_2s15_lz0_coulomb_block4.npz")["v"]
    sp, H = _fqhe(gpu, v, lz=42)
    assert sp.dim == 26
    H.set_precision(prec)
    lz = gpu.BasicBlockLanczosAlgorithm(H, 1, 400, block_size=4)
    lz.InitializeLanczosAlgorithm(seed=5)
    r = lz.solve(400)
    ref = dense_e0(orc, 6, 15, 42, v)
    assert r["converged"] and abs(r["eigenvalues"][0] - ref) < 1e-10 * abs(ref), (r, ref)
    psi = lz.GetGroundState()
    hpsi = orc.FQHE(6, 15, 42, v).pull(psi)
    assert np.linalg.norm(hpsi - ref * psi) < 1e-10


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_block_multiply_matches_oracle(gpu, orc, prec, tol, k):
    v = golden("lanczos_n8_2s21_lz0_coulomb_basic.npz")["v"]
    sp, H = _fqhe(gpu, v, 8, 21, 0)
    H.set_precision(prec)
    H.ShiftHamiltonian(0.37)
    x = np.random.default_rng(k).uniform(-1.0, 1.0, (sp.dim, k))
    y = H.block_multiply(x)
    O = orc.FQHE(8, 21, 0, v)
    for j in range(k):
        ref = O.pull(np.ascontiguousarray(x[:, j])) + 0.37 * x[:, j]
        assert np.max(np.abs(y[:, j] - ref)) <= tol * np.max(np.abs(ref)), (j, prec)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
@pytest.mark.parametrize("k", [2, 4])
def test_spin_block_multiply_matches_oracle(gpu, orc, prec, tol, k):
    L, sz = 14, 0
    chain = gpu.Spin1_2Chain(L, sz)
    H = gpu.SpinChainJ1J2Hamiltonian(chain, 1.0, 0.5)
    H.set_precision(prec)
    words = orc.spin_basis(L, sz)
    x = np.random.default_rng(k).uniform(-1.0, 1.0, (chain.dim, k))
    y = H.block_multiply(x)
    for j in range(k):
        ref = orc.spin_j1j2_multiply(L, sz, words, 1.0, 0.5, x[:, j])
        assert np.max(np.abs(y[:, j] - ref)) <= tol * np.max(np.abs(ref)), (j, prec)


@pytest.mark.parametrize("refined", [True, False])
def test_block_size_tuner(gpu, refined):
    # the tuner solves the sector with k = 1, 2, 4 and keeps the fastest; whatever it picks, the
    # block Lanczos with that k reaches the reference's energy
    z = golden("lanczos_n8_2s21_lz0_coulomb_basic.npz")
    sp, H = _fqhe(gpu, z["v"], n=8, s=21, lz=0)
    H.set_precision("fp64")
    k, times = H.tune_block_size(max_iter=600, precision=1e-10, refined=refined)
    assert k in (1, 2, 4) and all(t > 0 for t in times.values())
    assert times[k] == min(times.values())
    if refined:
        H.set_precision("fp32")
    lz = gpu.BasicLanczosAlgorithm(H, 1, 600) if k == 1 else gpu.BasicBlockLanczosAlgorithm(H, 1, 600, block_size=k)
    lz.InitializeLanczosAlgorithm(seed=0)
    e = lz.solve_refined(600, precision=1e-10)["energy"] if refined else lz.solve(600)["eigenvalues"][0]
    e_ref = float(z["eigenvalues"][0])
    assert abs(e - e_ref) < 1e-10 * abs(e_ref)
    H.set_precision("fp64")
