"""Lanczos on the GPU against the reference's own Lanczos runs (same start vector).
Eigenvalues within 1e-10 relative (1e-10 absolute for E0 = 0), iteration counts within two of
the reference (FP64 reduction order differs), Hellmann-Feynman gradients within 1e-8."""
import numpy as np
import pytest

from conftest import golden, parse_sector

pytestmark = pytest.mark.gpu


def _setup(gpu, orc, tag):
    z = golden("lanczos_%s_basic.npz" % tag)
    n, s, lz = parse_sector(tag)
    sp = gpu.FermionOnSphere(n, lz, s)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, z["v"])
    return z, sp, H, orc.random_vector(0, sp.dim)


@pytest.mark.parametrize("tag", ["n8_2s21_lz0_coulomb", "n7_2s18_lz2_coulomb", "n8_2s21_lz0_v1"])
def test_run_loop_matches_reference(gpu, orc, tag):
    z, sp, H, x0 = _setup(gpu, orc, tag)
    lz = gpu.BasicLanczosAlgorithm(H, 1, 300)
    lz.InitializeLanczosAlgorithm(x0)
    # QHEOnSphereMainTask.cc:732-753, driven from the host through the C ABI
    lz.RunLanczosAlgorithm(3)
    count = 4
    while not lz.TestConvergence() and count < int(z["max_iter"]):
        count += 1
        lz.RunLanczosAlgorithm(1)
    e, e_ref = lz.GetEigenvalues(1)[0], float(z["eigenvalues"][0])
    assert abs(e - e_ref) <= 1e-10 * max(abs(e_ref), 1.0)
    assert abs(count - int(z["iterations"])) <= 2
    assert lz.TestConvergence() == bool(z["converged"])


@pytest.mark.parametrize("batch", [1, 7, 16])
def test_solve_graph_batches_match_run_loop(gpu, orc, batch):
    z, sp, H, x0 = _setup(gpu, orc, "n8_2s21_lz0_coulomb")
    lz = gpu.BasicLanczosAlgorithm(H, 1, 300)
    lz.InitializeLanczosAlgorithm(x0)
    r = lz.solve(200, graph_batch=batch)
    assert r["converged"]
    assert abs(r["eigenvalues"][0] - float(z["eigenvalues"][0])) < 1e-10 * abs(float(z["eigenvalues"][0]))
    assert abs(r["iterations"] - int(z["iterations"])) <= 2


@pytest.mark.parametrize("tag,precision", [("n8_2s21_lz0_coulomb", 1e-10), ("n8_2s21_lz0_coulomb", 1e-13),
                                           ("n7_2s18_lz2_coulomb", 1e-12)])
def test_graph_batches_stop_near_convergence(gpu, orc, tag, precision):
    """Graph batches sized by the predicted convergence: the per-iteration run's energy and iteration
    count, with no more products than batches of 16 would take (3 + 16 per batch) and at most eight
    past the converged iteration (0, 0 and 7 when the policy is replayed on the oracle's runs of these
    cases, against 3, 9 and 12 for batches of 16)."""
    z, sp, H, x0 = _setup(gpu, orc, tag)
    runs = {}
    for batch in (1, 16):
        lz = gpu.BasicLanczosAlgorithm(H, 1, 400)
        lz.SetEigenvaluePrecision(precision)
        lz.InitializeLanczosAlgorithm(x0)
        r = lz.solve(400, graph_batch=batch)
        assert r["converged"]
        runs[batch] = (r["eigenvalues"][0], r["iterations"], lz.counters()[0])
    (e1, it1, mv1), (e16, it16, mv16) = runs[1], runs[16]
    assert it16 == it1
    assert abs(e16 - e1) <= 1e-13 * abs(e1)
    fixed = 3 + 16 * -(-(mv1 - 3) // 16)
    assert mv1 <= mv16 <= min(fixed, mv1 + 8)


def test_full_reorthogonalized(gpu, orc):
    z = golden("lanczos_n8_2s21_lz0_coulomb_full.npz")
    _, sp, H, x0 = _setup(gpu, orc, "n8_2s21_lz0_coulomb")
    lz = gpu.FullReorthogonalizedLanczosAlgorithm(H, 1, 300)
    lz.InitializeLanczosAlgorithm(x0)
    r = lz.solve(200)
    assert abs(r["eigenvalues"][0] - float(z["eigenvalues"][0])) < 1e-10 * abs(float(z["eigenvalues"][0]))


def test_ground_state_and_hellmann_feynman(gpu, orc):
    z = golden("lanczos_n8_2s21_lz0_coulomb_ground.npz")
    _, sp, H, x0 = _setup(gpu, orc, "n8_2s21_lz0_coulomb")
    lz = gpu.BasicLanczosAlgorithmWithGroundState(H, 1, 300)
    lz.InitializeLanczosAlgorithm(x0)
    lz.solve(200, graph_batch=1)
    psi = lz.GetGroundState()
    assert abs(np.linalg.norm(psi) - 1.0) < 1e-12
    e = H.MatrixElement(psi, psi)
    assert abs(e - float(z["energy_expectation"])) < 1e-10 * abs(e)
    # dE0/dV_m = <psi|H_m|psi> against the reference's <psi_ref|H_m|psi_ref>
    g = H.pseudopotential_adjoint(psi, psi)
    assert np.max(np.abs(g - z["expectation"])) < 1e-8


def test_ground_state_by_replay(gpu, orc):
    # a run whose Krylov basis is not kept rebuilds the Ritz vector by a second pass
    z = golden("lanczos_n8_2s21_lz0_coulomb_ground.npz")
    _, sp, H, x0 = _setup(gpu, orc, "n8_2s21_lz0_coulomb")
    lz = gpu.BasicLanczosAlgorithmWithGroundState(H, 1, 80)
    lz.set_vector_storage(False)
    lz.InitializeLanczosAlgorithm(x0)
    lz.solve(80, graph_batch=1)
    psi = lz.GetGroundState()
    assert abs(H.MatrixElement(psi, psi) - float(z["energy_expectation"])) < 1e-9


def test_fp32_refined_energy(gpu, orc):
    z, sp, H, x0 = _setup(gpu, orc, "n8_2s21_lz0_coulomb")
    lz = gpu.BasicLanczosAlgorithm(H, 1, 400)
    lz.InitializeLanczosAlgorithm(x0)
    r = lz.solve_refined(400, precision=1e-12)
    e_ref = float(z["eigenvalues"][0])
    assert abs(r["energy"] - e_ref) < 1e-10 * abs(e_ref), r
    assert r["fp32_matvecs"] > 0
