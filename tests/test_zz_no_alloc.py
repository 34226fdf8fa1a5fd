"""The allocation-free pseudopotential adjoint, called through the C ABI.

Some callers cannot allocate device memory (applications whose framework owns all device memory
through its own allocator or arena); dh_hamiltonian_pseudopotential_adjoint_static serves them
with a static device scratch array.  It must give the allocating entry point's result (same
1e-12 tolerance as the other adjoint tests) on consecutive calls, which reuse the array, in both
index modes, and must leave the device's free memory unchanged once its module is loaded.
This file is collected last so that a failure here comes after every other test has run.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _entry(gpu):
    lib = ctypes.CDLL(gpu.library_path())
    fn = lib.dh_hamiltonian_pseudopotential_adjoint_static
    fn.argtypes = [ctypes.c_void_p] * 4
    fn.restype = ctypes.c_int
    lib.dh_last_error.restype = ctypes.c_char_p
    return lib, fn


@pytest.mark.parametrize("mode", ["rank", "lookup"])
def test_static_adjoint_matches_allocating_entry_point(gpu, orc, mode):
    import torch
    lib, fn = _entry(gpu)
    v = golden("matvec_n8_2s21_lz0_coulomb_shift0.npz")["v"]
    sp = gpu.FermionOnSphere(8, 0, 21)
    sp.set_index_mode(mode)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 8, 21, v)
    for call in range(2):
        u = torch.tensor(orc.random_vector(40 + call, sp.dim), device="cuda")
        w = torch.tensor(orc.random_vector(50 + call, sp.dim), device="cuda")
        ref = H.pseudopotential_adjoint(u, w)
        out = np.zeros(22, np.float64)
        rc = fn(H._handle, ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(w.data_ptr()),
                ctypes.c_void_p(out.ctypes.data))
        assert rc == 0, lib.dh_last_error()
        assert np.max(np.abs(out - ref)) < 1e-12
    # device output buffer
    out_dev = torch.zeros(22, dtype=torch.float64, device="cuda")
    rc = fn(H._handle, ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(out_dev.data_ptr()))
    assert rc == 0, lib.dh_last_error()
    assert np.max(np.abs(out_dev.cpu().numpy() - ref)) < 1e-12


def test_static_adjoint_leaves_free_memory_unchanged(gpu, orc):
    import torch
    lib, fn = _entry(gpu)
    v = golden("matvec_n8_2s21_lz0_coulomb_shift0.npz")["v"]
    sp = gpu.FermionOnSphere(8, 0, 21)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 8, 21, v)
    u = torch.tensor(orc.random_vector(60, sp.dim), device="cuda")
    w = torch.tensor(orc.random_vector(61, sp.dim), device="cuda")
    out = np.zeros(22, np.float64)
    args = (H._handle, ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(out.ctypes.data))
    assert fn(*args) == 0, lib.dh_last_error()  # loads the kernels' module and looks up the array
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert fn(*args) == 0, lib.dh_last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before


def test_static_adjoint_rejects_what_it_cannot_hold(gpu, orc):
    import torch
    lib, fn = _entry(gpu)
    # host vectors would need staging buffers
    v = np.zeros(22)
    v[1] = 1.0
    sp = gpu.FermionOnSphere(8, 0, 21)
    H = gpu.ParticleOnSphereGenericHamiltonian(sp, 8, 21, v)
    x = orc.random_vector(1, sp.dim)
    out = np.zeros(22)
    rc = fn(H._handle, ctypes.c_void_p(x.ctypes.data), ctypes.c_void_p(x.ctypes.data), ctypes.c_void_p(out.ctypes.data))
    assert rc != 0
    assert b"device pointers" in lib.dh_last_error()
    # 2S = 35 has more interaction factors than the static scratch holds
    sp35 = gpu.FermionOnSphere(2, 0, 35)
    H35 = gpu.ParticleOnSphereGenericHamiltonian(sp35, 2, 35, np.eye(36)[1])
    t = torch.zeros(sp35.dim, dtype=torch.float64, device="cuda")
    out35 = np.zeros(36)
    rc = fn(H35._handle, ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(out35.ctypes.data))
    assert rc != 0 and b"static scratch" in lib.dh_last_error()
