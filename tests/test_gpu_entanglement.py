"""Orbital-cut entanglement on the GPU (FermionOnSphere::EvaluatePartialEntanglementMatrix and
EvaluatePartialDensityMatrix) against the reference's matrices for twelve cuts of a vector on N=8 2S=21
2Lz=0 (M within 1e-15, rho within 1e-14; the edge cases l = 0, l > 2S, N_A <= 1, empty sectors), a
larger sector against the oracle, device input and output, and the normalisation: the traces of
rho_A over every sector (N_A, Lz_A) of a cut add up to |psi|^2."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def test_cuts_match_reference(gpu, orc):
    z = golden("entanglement_n8_2s21_lz0.npz")
    sp = gpu.FermionOnSphere(8, 0, 21)
    x = orc.random_vector(int(z["seed"]), sp.dim)
    for l, na, lza in z["cases"]:
        l, na, lza = int(l), int(na), int(lza)
        tag = "l%d_na%d_lz%d" % (l, na, lza)
        ref = z["m_" + tag]
        m = sp.EvaluatePartialEntanglementMatrix(l, na, lza, x)
        assert m.shape == ref.shape, tag
        assert m.size == 0 or np.max(np.abs(m - ref)) <= 1e-15, tag
        if "rho_" + tag in z.files:
            rho = sp.EvaluatePartialDensityMatrix(l, na, lza, x)
            rref = z["rho_" + tag]
            assert rho.shape == rref.shape, tag
            assert rho.size == 0 or np.max(np.abs(rho - rref)) <= 1e-14, tag
        elif 0 < l <= 21 and ref.size:
            rho = sp.EvaluatePartialDensityMatrix(l, na, lza, x)
            assert np.max(np.abs(rho - ref @ ref.T)) <= 1e-14, tag


def test_larger_sector_and_normalisation(gpu, orc):
    import torch
    sp = gpu.FermionOnSphere(10, 0, 27)
    x = orc.random_vector(3, sp.dim)
    l = 14
    m_ref = orc.entanglement_matrix(10, 27, 0, x, l, 5, 1)
    m = sp.EvaluatePartialEntanglementMatrix(l, 5, 1, x)
    assert m.shape == m_ref.shape and np.max(np.abs(m - m_ref)) <= 1e-15
    # device state and device output
    xd = torch.from_numpy(x).cuda()
    rho = sp.EvaluatePartialDensityMatrix(l, 5, 1, xd)
    assert np.max(np.abs(rho - m_ref @ m_ref.T)) <= 1e-14
    r = m_ref.shape[0]
    out = torch.zeros(r * r, dtype=torch.float64, device="cuda")
    n = __import__("ctypes").c_int64(0)
    lib = gpu.load()
    rc = lib.dh_fermion_on_sphere_partial_density_matrix(sp._handle, xd.data_ptr(), l, 5, 1, out.data_ptr(), r * r,
                                                         __import__("ctypes").byref(n))
    assert rc == 0 and n.value == r
    assert np.max(np.abs(out.cpu().numpy().reshape(r, r) - rho)) == 0.0
    # sum over the sectors of the cut of tr(rho_A) = |x|^2 (N_A >= 2 here, where rho = M M^T)
    total = 0.0
    for na in range(2, 11):
        for lza in range(-na * (l - 1), na * (l - 1) + 1, 2):
            rho = sp.EvaluatePartialDensityMatrix(l, na, lza, x)
            total += float(np.trace(rho)) if rho.size else 0.0
    low = 0.0
    words, _ = sp.states()
    a = words & np.uint64((1 << l) - 1)
    npart = np.array([bin(int(w)).count("1") for w in a])
    low = float(np.sum(x[npart < 2] ** 2))
    assert abs(total + low - float(x @ x)) <= 1e-12


@pytest.mark.parametrize("n,s,lz,cuts", [(4, 50, 0, [(25, 2, 2), (45, 3, 1), (5, 1, 0), (12, 1, 3)]),
                                          (5, 41, 1, [(20, 2, 1), (35, 4, 2), (6, 2, -1)])])
def test_cuts_beyond_the_split_tables(gpu, orc, n, s, lz, cuts):
    # FermionOnSphere above 2S = 40 (the 128-bit engine's words), and subsystems of more than 41
    # orbitals on either side of the cut, against the oracle
    sp = gpu.FermionOnSphere(n, lz, s)
    x = orc.random_vector(3, sp.dim)
    for l, na, lza in cuts:
        ref = orc.entanglement_matrix(n, s, lz, x, l, na, lza)
        m = sp.EvaluatePartialEntanglementMatrix(l, na, lza, x)
        assert m.shape == ref.shape and (m.size == 0 or np.max(np.abs(m - ref)) <= 1e-15), (l, na, lza)
        rho = sp.EvaluatePartialDensityMatrix(l, na, lza, x)
        if na > 1 and ref.size:
            assert np.max(np.abs(rho - ref @ ref.T)) <= 1e-14, (l, na, lza)
    # sum over the sectors of a cut of tr(rho_A) = |x|^2
    l = 25
    total = 0.0
    for na in range(0, n + 1):
        for lza in range(-na * (l - 1), na * (l - 1) + 1, 2):
            rho = sp.EvaluatePartialDensityMatrix(l, na, lza, x)
            total += float(np.trace(rho)) if rho.size else 0.0
    assert abs(total - float(x @ x)) <= 1e-12
