"""Products into host memory run in row chunks whose device-to-host copies overlap the next chunk's
product.  On sectors large enough to be split (>= 2^19 rows) the result must equal, bit for bit, the
same product into device memory (one launch over every row): FQHE fermions on the fly and from stored
elements, the J1-J2 chain and bosons; single vectors, several vectors one after the other, and
row-interleaved blocks; FP64 and FP32; LowLevelAddMultiply with a column range into a non-zero
destination."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _compare(H, dim, torch):
    g = torch.Generator(device="cuda").manual_seed(11)
    X = torch.rand(dim, 4, dtype=torch.float64, device="cuda", generator=g) - 0.5
    # row-interleaved block of 4
    Yd = H.block_multiply(X)
    Yh = H.block_multiply(X.cpu().numpy())
    assert np.array_equal(Yh, Yd.cpu().numpy())
    # one vector, host destination
    x = X[:, 0].contiguous()
    yd = torch.empty(dim, dtype=torch.float64, device="cuda")
    H.LowLevelMultiply(x, yd)
    yh = H.LowLevelMultiply(x)
    assert np.array_equal(yh, yd.cpu().numpy())
    # three vectors one after the other
    S = X[:, :3].T.contiguous()
    Dd = torch.zeros_like(S)
    H.LowLevelMultipleAddMultiply(S, Dd)
    Dh = np.zeros((3, dim))
    H.LowLevelMultipleAddMultiply(S.cpu().numpy(), Dh)
    assert np.array_equal(Dh, Dd.cpu().numpy())
    # column range into a non-zero destination
    first, nbr = dim // 7, dim // 2
    y0 = X[:, 3].contiguous()
    yd = y0.clone()
    H.LowLevelAddMultiply(x, yd, first, nbr)
    yh = y0.cpu().numpy().copy()
    H.LowLevelAddMultiply(x, yh, first, nbr)
    assert np.array_equal(yh, yd.cpu().numpy())


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_fermion_products_into_host_memory(gpu, prec):
    import torch
    v = gpu.coulomb_pseudopotentials(30)
    v[0::2] = 0.0
    sp = gpu.FermionOnSphere(11, 0, 30)
    assert sp.dim >= 1 << 19
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 11, 30, v)
    H.set_precision(prec)
    H.ShiftHamiltonian(0.3)
    _compare(H, sp.dim, torch)
    assert H.EnableFastMultiplication()[0]
    _compare(H, sp.dim, torch)


def test_spin_products_into_host_memory(gpu):
    import torch
    ch = gpu.Spin1_2Chain(24, 0)
    H = gpu.SpinChainJ1J2Hamiltonian(ch, 1.0, 0.5)
    H.set_precision("fp32")
    H.ShiftHamiltonian(-0.2)
    _compare(H, ch.dim, torch)


def test_boson_products_into_host_memory(gpu):
    import torch
    v = gpu.coulomb_pseudopotentials(20)
    v[1::2] = 0.0
    sp = gpu.BosonOnSphereShort(11, 0, 20)
    assert sp.dim >= 1 << 19
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 11, 20, v)
    _compare(H, sp.dim, torch)
