"""FermionOnSphere + ParticleOnSphereGenericHamiltonian on the GPU against the reference fixtures
and the oracle.  Indices and signs must be bit-exact; FP64 products agree to rounding
(|dy| <= 1e-12 max|y|); FP32 products within 2e-6 max|y| of FP64."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden, parse_sector

pytestmark = pytest.mark.gpu

MODES = ["rank", "lookup", "rank-generic", "rank-smem"]


def make_space(gpu, n, lz, s, mode):
    """A FermionOnSphere in one of the index modes; rank-generic is the rank mode on the generic
    (non split-word) product kernel."""
    import os
    if mode in ("rank-generic", "rank-smem"):
        os.environ["DH_FQHE_KERNEL"] = mode.split("-")[1]
        try:
            sp = gpu.FermionOnSphere(n, lz, s)
        finally:
            del os.environ["DH_FQHE_KERNEL"]
        return sp
    sp = gpu.FermionOnSphere(n, lz, s)
    sp.set_index_mode(mode)
    return sp


@pytest.mark.parametrize("name", sorted(os.path.basename(f) for f in glob.glob(os.path.join(GOLDEN, "fqhe_basis_*.npz"))))
def test_basis_words_bit_exact(gpu, name):
    z = golden(name)
    n, s, lz = parse_sector(name)
    sp = gpu.FermionOnSphere(n, lz, s)
    words, lzmax = sp.states()
    assert np.array_equal(words, z["words"]) and np.array_equal(lzmax, z["lzmax"])


@pytest.mark.parametrize("mode", MODES)
def test_find_state_index(gpu, orc, mode):
    sp = make_space(gpu, 8, 0, 21, mode)
    words, _ = sp.states()
    assert np.array_equal(sp.FindStateIndex(words), np.arange(len(words)))
    # words outside the sector are reported as -1
    bad = np.array([0, 1, (1 << 22) - 1, int(words[0]) ^ 1], np.uint64)
    assert np.all(sp.FindStateIndex(bad) == -1)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", ["rows_n8_2s21_lz0_v1.npz", "rows_n8_2s21_lz0_coulomb.npz",
                                  "rows_n7_2s18_lz2_coulomb.npz", "rows_n10_2s27_lz0_coulomb.npz",
                                  "rows_n12_2s33_lz0_coulomb.npz"])
def test_row_elements_bit_exact(gpu, name, mode):
    z = golden(name)
    n, s, lz = parse_sector(name)
    sp = make_space(gpu, n, lz, s, mode)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, z["v"])
    for k, r in enumerate(z["rows"]):
        a, b = z["offsets"][k], z["offsets"][k + 1]
        t, sg, f = H.row_elements(int(r))
        assert np.array_equal(t, z["targets"][a:b]), r
        assert np.array_equal(sg, z["signs"][a:b]), r
        assert np.array_equal(f, z["factor_index"][a:b]), r


@pytest.mark.parametrize("name", ["factors_2s21_v1.npz", "factors_2s27_coulomb.npz", "factors_2s33_coulomb.npz"])
def test_interaction_factors(gpu, name):
    z = golden(name)
    two_s = int(name.split("_")[1][2:])
    sp = gpu.FermionOnSphere(2, 0, two_s) if two_s % 2 == 0 else gpu.FermionOnSphere(2, 1 - 1, two_s)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 2, two_s, z["v"])
    f = H.interaction_factors()
    assert np.max(np.abs(f - z["factors"])) < 1e-13 * np.max(np.abs(z["factors"]))


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("tag", ["n8_2s21_lz0_v1", "n8_2s21_lz0_coulomb", "n7_2s18_lz2_coulomb"])
@pytest.mark.parametrize("shift", [0.0, 0.37])
def test_matvec_fp64_vs_reference(gpu, orc, tag, shift, mode):
    z = golden("matvec_%s_shift%g.npz" % (tag, shift))
    n, s, lz = parse_sector(tag)
    sp = make_space(gpu, n, lz, s, mode)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, z["v"])
    H.ShiftHamiltonian(shift)
    x = orc.random_vector(0, sp.dim)
    y = H.LowLevelMultiply(x)
    assert np.max(np.abs(y - z["y"])) <= 1e-12 * max(1.0, np.max(np.abs(z["y"])))


@pytest.mark.parametrize("mode", MODES)
def test_matvec_fp32_vs_fp64(gpu, orc, mode):
    z = golden("matvec_n8_2s21_lz0_coulomb_shift0.37.npz")
    sp = make_space(gpu, 8, 0, 21, mode)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 8, 21, z["v"])
    H.ShiftHamiltonian(0.37)
    H.set_precision("fp32")
    y = H.LowLevelMultiply(orc.random_vector(0, sp.dim))
    assert np.max(np.abs(y - z["y"])) <= 2e-6 * np.max(np.abs(z["y"]))


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("first,nbr", [(0, 100), (1234, 3000), (8000, 512), (4000, -1)])
def test_low_level_add_multiply_column_range(gpu, orc, first, nbr, mode):
    # push-form contract: dst += H[:, first:first+nbr] src[first:first+nbr], dst accumulated
    z = golden("factors_2s21_v1.npz")
    v = golden("matvec_n8_2s21_lz0_coulomb_shift0.npz")["v"]
    O = orc.FQHE(8, 21, 0, v, shift=0.25)
    sp = make_space(gpu, 8, 0, 21, mode)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 8, 21, v)
    H.ShiftHamiltonian(0.25)
    x = orc.random_vector(1, sp.dim)
    y0 = orc.random_vector(2, sp.dim)
    nb = sp.dim - first if nbr < 0 else nbr
    ref = y0 + O.push(x, first, nb)
    y = y0.copy()
    H.LowLevelAddMultiply(x, y, first, nbr)
    assert np.max(np.abs(y - ref)) < 1e-12
    del z


@pytest.mark.parametrize("mode", MODES)
def test_multiple_add_multiply(gpu, orc, mode):
    v = golden("matvec_n8_2s21_lz0_coulomb_shift0.npz")["v"]
    sp = make_space(gpu, 8, 0, 21, mode)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 8, 21, v)
    for k in (1, 2, 3, 4, 7):
        xs = np.stack([orc.random_vector(10 + j, sp.dim) for j in range(k)])
        ys = np.stack([orc.random_vector(20 + j, sp.dim) for j in range(k)])
        ref = ys + np.stack([H.LowLevelMultiply(xs[j]) for j in range(k)])
        out = ys.copy()
        H.LowLevelMultipleAddMultiply(xs, out)
        assert np.max(np.abs(out - ref)) < 1e-12


def test_matrix_element_and_device_pointers(gpu, orc):
    import torch
    v = golden("matvec_n8_2s21_lz0_coulomb_shift0.npz")["v"]
    O = orc.FQHE(8, 21, 0, v)
    sp = gpu.FermionOnSphere(8, 0, 21)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 8, 21, v)
    a, b = orc.random_vector(3, sp.dim), orc.random_vector(4, sp.dim)
    ref = float(a @ O.pull(b))
    assert abs(H.MatrixElement(a, b) - ref) < 1e-12
    ta = torch.tensor(a, device="cuda")
    tb = torch.tensor(b, device="cuda")
    ty = torch.zeros_like(tb)
    H.LowLevelMultiply(tb, ty)
    torch.cuda.synchronize()
    assert np.max(np.abs(ty.cpu().numpy() - O.pull(b))) < 1e-12
    assert abs(H.MatrixElement(ta, tb) - ref) < 1e-12


@pytest.mark.parametrize("mode", MODES)
def test_precision_workload_symmetry_and_rows(gpu, orc, mode):
    """N = 12, 2S = 33, Lz = 0 (dimension 7,764,392): size-independent properties of the product."""
    z = golden("rows_n12_2s33_lz0_coulomb.npz")
    sp = make_space(gpu, 12, 0, 33, mode)
    assert sp.dim == 7764392
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 12, 33, z["v"])
    x, y = orc.random_vector(5, sp.dim), orc.random_vector(6, sp.dim)
    hx, hy = H.LowLevelMultiply(x), H.LowLevelMultiply(y)
    # real symmetric: <y|Hx> = <x|Hy>; linear: H(x + 2y) = Hx + 2Hy
    assert abs(y @ hx - x @ hy) < 1e-11 * np.linalg.norm(hx)
    assert np.max(np.abs(H.LowLevelMultiply(x + 2 * y) - (hx + 2 * hy))) < 1e-11 * np.max(np.abs(hx))
    # the row sums of |elements| agree with the reference element lists
    for k, r in enumerate(z["rows"][:4]):
        a, b = z["offsets"][k], z["offsets"][k + 1]
        e = np.zeros(sp.dim)
        e[int(r)] = 1.0
        col = H.LowLevelMultiply(e)
        f = H.interaction_factors()
        expect = np.zeros(sp.dim)
        np.add.at(expect, z["targets"][a:b], z["signs"][a:b] * f[z["factor_index"][a:b]])
        assert np.max(np.abs(col - expect)) < 1e-12


def test_pseudopotential_adjoint_vs_oracle(gpu, orc):
    v = golden("matvec_n8_2s21_lz0_coulomb_shift0.npz")["v"]
    O = orc.FQHE(8, 21, 0, v)
    sp = gpu.FermionOnSphere(8, 0, 21)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 8, 21, v)
    u, w = orc.random_vector(8, sp.dim), orc.random_vector(9, sp.dim)
    ref = O.bins(u, w) @ orc.interaction_derivatives(21)
    got = H.pseudopotential_adjoint(u, w)
    assert np.max(np.abs(got - ref)) < 1e-12
    # linearity in V: sum_m V_m <u|dH/dV_m|w> = <u|H|w>
    assert abs(got @ v - u @ O.pull(w)) < 1e-12


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_autotune_keeps_parity(gpu, orc, prec):
    # every candidate form computes the same product: after tuning the product still matches the
    # oracle, and the tuner reports the form it kept
    z = golden("lanczos_n8_2s21_lz0_coulomb_basic.npz")
    sp = gpu.FermionOnSphere(8, 0, 21)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 8, 21, z["v"])
    H.set_precision(prec)
    x = orc.random_vector(5, sp.dim)
    ref = orc.FQHE(8, 21, 0, z["v"]).pull(x)
    tol = 1e-13 if prec == "fp64" else 2e-6
    r = H.autotune(block_size=2, repeats=2)
    assert r["candidates"] >= 5 and r["best_ms"] > 0 and r["kernel_variant"] in ("split", "generic", "split+smem")
    assert 0 < r["ms_k1"] and 0 < r["ms_k4"]
    y = H.LowLevelMultiply(x)
    assert np.max(np.abs(y - ref)) <= tol * np.max(np.abs(ref))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("k", [1, 2, 4])
def test_launch_forms_bit_identical(gpu, orc, precision, k):
    # every launch form of the split-word kernel (threads per block, register budget, gather
    # pipeline) computes the same sums in the same order: bit-identical blocks, and the form-0
    # FP64 product matches the oracle
    import torch
    v = golden("matvec_n8_2s21_lz0_coulomb_shift0.npz")["v"]
    sp = gpu.FermionOnSphere(8, 0, 21)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 8, 21, v)
    H.set_precision(precision)
    x = torch.tensor(np.stack([orc.random_vector(70 + j, sp.dim) for j in range(k)], axis=1), device="cuda")
    ys = []
    for form in range(len(gpu.SPLIT_FORMS)):
        sp.set_split_form(form)
        ys.append(H.block_multiply(x).cpu().numpy())
    for form in range(1, len(ys)):
        assert np.array_equal(ys[form], ys[0]), form
    if precision == "fp64":
        ref = orc.FQHE(8, 21, 0, v)
        for j in range(k):
            assert np.max(np.abs(ys[0][:, j] - ref.pull(x[:, j].cpu().numpy()))) < 1e-12
    with pytest.raises(Exception):
        sp.set_split_form(len(gpu.SPLIT_FORMS))
