"""Differentiation through the C ABI.

* The VJP of y = H(V) x (adjoint kernel for V, the product for x) against torch.autograd.gradcheck
  and against exact directional derivatives (H is linear in V).
* Hellmann-Feynman gradients of E0 and of the neutral gap for N = 10, 2S = 27, Lz = 0 and 1
  (Coulomb + uniform noise from seed 2) against the reference's FP64 gradient
  <psi_ref|H_m|psi_ref> and against central finite differences of the GPU E0 (h = 1e-6).
* The same VJP on BosonOnSphereShort and FermionOnSphereLong, and a bosonic Hellmann-Feynman
  gradient against central differences.
Tolerances: gradcheck at its FP64 defaults; energies 1e-10 relative; gradients against the reference
1e-7 absolute (both sides carry Lanczos eigenvector errors, first order in a Hellmann-Feynman
gradient); finite differences 2e-6 absolute (E0 converged to 1e-14 relative over 2h = 2e-6)."""
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def _hamiltonian(gpu, n, s, lz, v):
    sp = gpu.FermionOnSphere(n, lz, s)
    return sp, gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v)


def test_product_gradcheck(gpu):
    from diagham_b200.autograd import hamiltonian_product
    v0 = gpu.coulomb_pseudopotentials(12)
    sp, H = _hamiltonian(gpu, 5, 12, 2, v0)
    V = torch.tensor(v0, dtype=torch.float64, requires_grad=True)
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.rand(sp.dim, 2, dtype=torch.float64, device="cuda", generator=g).requires_grad_(True)
    assert torch.autograd.gradcheck(lambda V_, x_: hamiltonian_product(V_, x_, H), (V, x), eps=1e-6, atol=1e-8,
                                    rtol=1e-6)


@pytest.mark.parametrize("k", [1, 4])
def test_product_vjp_is_exact_directional_derivative(gpu, k):
    from diagham_b200.autograd import hamiltonian_product
    z = golden("lanczos_n8_2s21_lz0_coulomb_basic.npz")
    sp, H = _hamiltonian(gpu, 8, 21, 0, z["v"])
    V = torch.tensor(z["v"], dtype=torch.float64, requires_grad=True)
    gen = torch.Generator(device="cuda").manual_seed(k)
    shape = (sp.dim,) if k == 1 else (sp.dim, k)
    x = (torch.rand(shape, dtype=torch.float64, device="cuda", generator=gen) - 0.5).requires_grad_(True)
    w = torch.rand(shape, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    y = hamiltonian_product(V, x, H)
    (y * w).sum().backward()
    # dV_m: <w|H(e_m)|x>; dx: H w (symmetric H)
    with torch.no_grad():
        for m in (1, 3, 7, 21):
            e = np.zeros_like(z["v"])
            e[m] = 1.0
            ym = hamiltonian_product(torch.tensor(e), x.detach(), H)
            assert abs(float((ym * w).sum()) - float(V.grad[m])) < 1e-10 * max(1.0, abs(float(V.grad[m])))
        hw = hamiltonian_product(V.detach(), w, H)
        assert float((hw - x.grad).abs().max()) < 1e-12 * float(hw.abs().max())


@pytest.fixture(scope="module")
def config_d(gpu):
    z0 = golden("gradient_n10_2s27_lz0.npz")
    z1 = golden("gradient_n10_2s27_lz2.npz")
    _, H0 = _hamiltonian(gpu, 10, 27, 0, z0["v"])
    _, H1 = _hamiltonian(gpu, 10, 27, 2, z0["v"])
    return z0, z1, H0, H1


def test_energy_and_gap_gradients_against_reference(gpu, config_d):
    from diagham_b200.autograd import ground_state_energy, neutral_gap
    z0, z1, H0, H1 = config_d
    odd = np.arange(1, 28, 2)
    V = torch.tensor(z0["v"], dtype=torch.float64, requires_grad=True)
    e0 = ground_state_energy(V, H0)
    e0.backward()
    ref0 = float(z0["eigenvalues"][0])
    assert abs(float(e0.detach()) - ref0) < 1e-10 * abs(ref0)
    assert np.max(np.abs(V.grad.numpy()[odd] - z0["expectation"][odd])) < 1e-7
    assert np.max(np.abs(V.grad.numpy()[0::2])) < 1e-12  # even m do not act on fermions
    V.grad = None
    gap = neutral_gap(V, H0, H1)
    gap.backward()
    ref_gap = float(z1["eigenvalues"][0]) - ref0
    assert abs(float(gap.detach()) - ref_gap) < 1e-10 * abs(ref0)
    ref_grad = z1["expectation"][odd] - z0["expectation"][odd]
    assert np.max(np.abs(V.grad.numpy()[odd] - ref_grad)) < 1e-7


def test_gradients_against_central_differences(gpu, config_d):
    from diagham_b200.autograd import ground_state_energy
    z0, z1, H0, H1 = config_d
    h = 1e-6
    v = z0["v"]
    odd = list(range(1, 28, 2))
    for H, z in ((H0, z0), (H1, z1)):
        V = torch.tensor(v, dtype=torch.float64, requires_grad=True)
        ground_state_energy(V, H).backward()
        fd = []
        for m in odd:
            vp, vm = v.copy(), v.copy()
            vp[m] += h
            vm[m] -= h
            ep = float(ground_state_energy(torch.tensor(vp), H))
            em = float(ground_state_energy(torch.tensor(vm), H))
            fd.append((ep - em) / (2 * h))
        err = np.abs(np.array(fd) - V.grad.numpy()[odd])
        assert np.max(err) < 2e-6, (err, fd)


@pytest.mark.parametrize("space", ["boson", "long"])
def test_product_gradcheck_bosons_and_128_bit_words(gpu, space):
    # the same VJP on BosonOnSphereShort (its bosonic adjoint) and on the 128-bit fermion engine
    from diagham_b200.autograd import hamiltonian_product
    if space == "boson":
        n, s, lz = 5, 9, 1
        v0 = gpu.coulomb_pseudopotentials(s)
        v0[1::2] = 0.0
        sp = gpu.BosonOnSphereShort(n, lz, s)
    else:
        n, s, lz = 3, 63, 1
        v0 = gpu.coulomb_pseudopotentials(s)
        sp = gpu.FermionOnSphereLong(n, lz, s)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, n, s, v0)
    V = torch.tensor(v0, dtype=torch.float64, requires_grad=True)
    g = torch.Generator(device="cuda").manual_seed(4)
    x = torch.rand(sp.dim, 2, dtype=torch.float64, device="cuda", generator=g).requires_grad_(True)
    assert torch.autograd.gradcheck(lambda V_, x_: hamiltonian_product(V_, x_, H), (V, x), eps=1e-6, atol=1e-8,
                                    rtol=1e-6)


def test_boson_ground_state_gradient_against_central_differences(gpu):
    # Hellmann-Feynman dE0/dV_m of BosonOnSphereShort N = 8, 2S = 14 (even m enter the bosonic factors)
    from diagham_b200.autograd import ground_state_energy
    z = golden("boson_n8_2s14_lz0_coulomb.npz")
    v = np.array(z["v"])
    sp = gpu.BosonOnSphereShort(8, 0, 14)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 8, 14, v)
    V = torch.tensor(v, dtype=torch.float64, requires_grad=True)
    e0 = ground_state_energy(V, H)
    assert abs(float(e0.detach()) - float(z["eigenvalues"][0])) <= 1e-10 * abs(float(z["eigenvalues"][0]))
    e0.backward()
    g = V.grad.numpy()
    h = 1e-6
    for m in (0, 2, 4):
        vp, vm = v.copy(), v.copy()
        vp[m] += h
        vm[m] -= h
        fd = (float(ground_state_energy(torch.tensor(vp), H)) - float(ground_state_energy(torch.tensor(vm), H))) / (2 * h)
        assert abs(fd - g[m]) < 2e-6, (m, fd, g[m])
    assert np.all(g[1::2] == 0.0)  # odd m never enter a bosonic factor
