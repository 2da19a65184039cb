"""Final-time observables and the torch.autograd harness of the adjoint.

The library differentiates (tb_adjoint_* in include/tortoise_b200.h); this
module states the observables as weight vectors and wraps the C ABI in
``torch.autograd.Function`` so that gradients flow into ordinary torch code:

    f_obs = DP45Solve.apply(f0, amplitudes, engine, t0, t1, dense_step)
    J = (w * f_obs).sum();  J.backward()        # f0.grad, amplitudes.grad

Observables are linear functionals J = <w, f> of one band's linear-form
coefficients (c0 = f(v0), c1 = f(v1) - f(v0), c2 = f(v2) - f(v0) per element),
integrated with the mass matrix of the reference (Gauss 3-point rule of
Mesh<2>, src/Geometry/Structured/DirectSpace/Mesh.cpp:95-123):
  density   n = int f dk            w_e = M (1, 0, 0)
  energy    U = int E f dk          w_e = M e_e      (e_e: band dispersion)
  current   j = int dE/dk_x f dk    w_e = (dE/dk_x)_e M (1, 0, 0)
"""
import numpy as np
import torch

from .engine import Engine

_GP_A, _GP_B, _GW = 0.16666666666667, 0.66666666666667, 0.33333333333333


def element_mass(mesh):
    """3x3 mass matrix of one element of ``mesh`` (all elements are equal)."""
    pts = [(_GP_A, _GP_A), (_GP_B, _GP_A), (_GP_A, _GP_B)]
    M = np.zeros((3, 3))
    for x, y in pts:
        phi = np.array([1.0, x, y])
        M += _GW * np.outer(phi, phi)
    return mesh.elemVolume * M


def observable_weights(material, band, kind="energy", component=0):
    """Weight vector w (length of the state) with J = w . f for one band.

    kind: "density", "energy" or "current" (band velocity component
    ``component`` of the P1 dispersion, constant per element)."""
    offs, total = material.band_offsets()
    b = material.bands[band]
    M = element_mass(b.mesh)
    ne = b.mesh.ne
    if kind == "density":
        wb = np.tile(M[:, 0], ne)
    elif kind == "energy":
        e = b.dispersion_coeffs.reshape(ne, 3)
        wb = (e @ M.T).reshape(-1)
    elif kind == "current":
        v = b.mesh.vertices()
        J = np.stack([v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]], axis=-1)  # (ne, 2, 2): columns are the edges
        e = b.dispersion_coeffs.reshape(ne, 3)
        grad = np.linalg.solve(np.transpose(J, (0, 2, 1)), e[:, 1:3, None])[..., 0]  # J^-T (e1, e2)
        wb = (grad[:, component][:, None] * M[None, :, 0]).reshape(-1)
    else:
        raise ValueError("unknown observable %r" % kind)
    w = np.zeros(total)
    w[offs[band]:offs[band] + wb.size] = wb
    return w


def _as_np(t):
    return t.detach().to("cpu", torch.float64).contiguous().numpy()


def set_amplitudes(engine, amps):
    """Pushes per-channel amplitudes into the handle (only the changed ones)."""
    a = np.asarray(amps, dtype=np.float64).reshape(-1)
    cur = getattr(engine, "_amps", None)
    for c in range(engine.channel_count()):
        if cur is None or cur[c] != a[c]:
            engine.set_amplitude(c, float(a[c]))
    engine._amps = a.copy()


class RHS(torch.autograd.Function):
    """dfdt = F(f; amplitudes) with F^T products from tb_adjoint_rhs_vjp."""

    @staticmethod
    def forward(ctx, f, amps, engine, drift=True):
        set_amplitudes(engine, _as_np(amps))
        out = engine.rhs(_as_np(f), drift=drift)
        ctx.engine, ctx.drift = engine, drift
        ctx.save_for_backward(f)
        return torch.as_tensor(out, dtype=torch.float64, device=f.device)

    @staticmethod
    def backward(ctx, grad_out):
        (f,) = ctx.saved_tensors
        g, ga = ctx.engine.rhs_vjp(_as_np(f), _as_np(grad_out), drift=ctx.drift)
        return (torch.as_tensor(g, dtype=torch.float64, device=f.device),
                torch.as_tensor(ga, dtype=torch.float64, device=f.device), None, None)


class DP45Solve(torch.autograd.Function):
    """f(t_obs) of the adaptive Dormand-Prince integration from f0 (t_obs =
    the last dense output time, t1 when (t1 - t0) / dense_step is whole).

    Forward: tb_adjoint_forward (checkpoints every ``checkpoint_every``
    accepted steps stay in the handle).  Backward: tb_adjoint_backward with
    the incoming gradient as lambda_T.  One handle keeps the checkpoints of
    its latest forward only, so call backward before the next forward on the
    same engine."""

    @staticmethod
    def forward(ctx, f0, amps, engine, t0, t1, dense_step, checkpoint_every=16, max_steps=16384, drift=True):
        set_amplitudes(engine, _as_np(amps))
        fo, st = engine.adjoint_forward(_as_np(f0), t0, t1, dense_step, checkpoint_every, max_steps, drift=drift)
        engine._adj_token = object()
        ctx.engine, ctx.token, ctx.stats = engine, engine._adj_token, st
        ctx.device = f0.device
        return torch.as_tensor(fo, dtype=torch.float64, device=f0.device)

    @staticmethod
    def backward(ctx, grad_out):
        if ctx.engine._adj_token is not ctx.token:
            raise RuntimeError("another forward sweep ran on this engine since this one; its checkpoints are gone")
        g, ga, st = ctx.engine.adjoint_backward(_as_np(grad_out))
        ctx.engine.last_adjoint_stats = st
        dev = ctx.device
        return (torch.as_tensor(g, dtype=torch.float64, device=dev), torch.as_tensor(ga, dtype=torch.float64, device=dev),
                None, None, None, None, None, None, None)


def gradient(engine, f0, amps, w, t0, t1, dense_step, checkpoint_every=16, max_steps=16384, drift=True):
    """J = <w, f(t_obs)> and its gradients wrt f0 and the channel amplitudes
    through the C ABI (no torch).  Returns (J, grad_f0, grad_amps, stats)."""
    set_amplitudes(engine, amps)
    fo, _ = engine.adjoint_forward(f0, t0, t1, dense_step, checkpoint_every, max_steps, drift=drift)
    g, ga, st = engine.adjoint_backward(w)
    return float(np.dot(w, fo)), g, ga, st


__all__ = ["Engine", "RHS", "DP45Solve", "element_mass", "observable_weights", "gradient", "set_amplitudes"]
