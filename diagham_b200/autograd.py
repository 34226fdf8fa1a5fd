"""torch.autograd views of the on-the-fly FQHE product and of Lanczos ground-state energies.

The two-body Hamiltonian is linear in the pseudopotentials: its interaction factors are
-4 sum_J V_J CG CG sums (ParticleOnSphereGenericHamiltonian::EvaluateInteractionFactors,
ParticleOnSphereGenericHamiltonian.cc:509-601), so H(V) = sum_m V_m H_m with H_m = dH/dV_m.

* ``hamiltonian_product(V, x, H)``: y = H(V) x for x of shape (dim,) or a row-interleaved block
  (dim, k).  Backward (the bilinear VJP, g = dL/dy): dL/dx = H(V) g (H is real symmetric) through
  the same product kernels, and dL/dV_m = sum_j <g_j|H_m|x_j> through the adjoint kernel
  (dh_hamiltonian_pseudopotential_adjoint), which bins every matrix element's g*x contribution
  by interaction factor and contracts the bins with dfactor/dV_m.
* ``ground_state_energy(V, H)``: E0(V) of one sector by GPU Lanczos (FP64).  Backward is
  Hellmann-Feynman: dE0/dV_m = <psi|H_m|psi> with the normalised Ritz vector psi.
* ``neutral_gap(V, H_ground, H_excited)``: E0 of the excited sector minus E0 of the ground sector
  (on the sphere: lowest Lz = 1 state minus the Lz = 0 ground state), differentiable the same way.

Every call fails loudly when the CUDA library is missing: there is no CPU path.
"""
import numpy as np
import torch

from . import BasicLanczosAlgorithmWithGroundState, DiagHamError


def _as_numpy_v(V):
    return V.detach().to("cpu", torch.float64).numpy()


def _block_multiply(h, x):
    x = x.detach().contiguous()
    y = torch.empty_like(x)
    h.block_multiply(x, y)
    return y


class HamiltonianProduct(torch.autograd.Function):
    """y = H(V) x (see the module docstring)."""

    @staticmethod
    def forward(ctx, V, x, hamiltonian):
        if not x.is_cuda or x.dtype != torch.float64:
            raise DiagHamError("hamiltonian_product: x must be a CUDA float64 tensor")
        hamiltonian.set_pseudopotentials(_as_numpy_v(V))
        ctx.hamiltonian = hamiltonian
        ctx.save_for_backward(V, x)
        return _block_multiply(hamiltonian, x)

    @staticmethod
    def backward(ctx, gy):
        V, x = ctx.saved_tensors
        h = ctx.hamiltonian
        h.set_pseudopotentials(_as_numpy_v(V))
        gy = gy.contiguous()
        gV = gx = None
        if ctx.needs_input_grad[1]:
            gx = _block_multiply(h, gy)
        if ctx.needs_input_grad[0]:
            g2 = gy.reshape(gy.shape[0], -1)
            x2 = x.reshape(x.shape[0], -1)
            acc = np.zeros(V.numel(), np.float64)
            for j in range(x2.shape[1]):
                acc += h.pseudopotential_adjoint(g2[:, j].contiguous(), x2[:, j].contiguous())[: V.numel()]
            gV = torch.as_tensor(acc, dtype=V.dtype, device=V.device)
        return gV, gx, None


def hamiltonian_product(V, x, hamiltonian):
    return HamiltonianProduct.apply(V, x, hamiltonian)


class GroundStateEnergy(torch.autograd.Function):
    """E0(V) of the Hamiltonian's sector (see the module docstring)."""

    @staticmethod
    def forward(ctx, V, hamiltonian, precision, max_iter, seed):
        hamiltonian.set_pseudopotentials(_as_numpy_v(V))
        hamiltonian.set_precision("fp64")
        lz = BasicLanczosAlgorithmWithGroundState(hamiltonian, 1, max_iter)
        lz.SetEigenvaluePrecision(precision)
        lz.InitializeLanczosAlgorithm(seed=seed)
        r = lz.solve(max_iter, graph_batch=16)
        if not r["converged"]:
            raise DiagHamError("ground_state_energy: Lanczos did not converge in %d iterations" % max_iter)
        psi = torch.empty(hamiltonian.dim, dtype=torch.float64, device="cuda")
        lz.GetGroundState(psi)
        ctx.hamiltonian = hamiltonian
        ctx.psi = psi
        ctx.nv = V.numel()
        ctx.v = _as_numpy_v(V).copy()
        return torch.tensor(float(r["eigenvalues"][0]), dtype=V.dtype, device=V.device)

    @staticmethod
    def backward(ctx, g):
        h = ctx.hamiltonian
        h.set_pseudopotentials(ctx.v)
        grad = h.pseudopotential_adjoint(ctx.psi, ctx.psi)[: ctx.nv]
        gV = g * torch.as_tensor(grad, dtype=g.dtype, device=g.device)
        return gV, None, None, None, None


def ground_state_energy(V, hamiltonian, precision=1e-14, max_iter=1000, seed=0):
    return GroundStateEnergy.apply(V, hamiltonian, precision, max_iter, seed)


def neutral_gap(V, h_ground, h_excited, precision=1e-14, max_iter=1000, seed=0):
    return (ground_state_energy(V, h_excited, precision, max_iter, seed) -
            ground_state_energy(V, h_ground, precision, max_iter, seed))
