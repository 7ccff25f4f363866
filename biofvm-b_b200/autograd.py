"""torch.autograd bridge over the reverse-mode C ABI (bfb_adjoint_run).

``simulate(env, rho0, D, lam, dt, n_steps, ...)`` runs n_steps LOD
diffusion-decay steps (and, given ``agents``, the agents' implicit
secretion/uptake after each) on ``env`` and returns the final field as a CUDA
tensor. Its backward pass calls bfb_adjoint_run, which re-runs the steps from
rho0 with a checkpoint every ``checkpoint_every`` steps and returns the
gradients with respect to

* rho0 (CUDA tensor of the env precision, shape (nx, ny, nz, S)),
* D and lam (host float64 tensors of shape (S,)),
* the agents' secretion, uptake and saturation (host float64, (n_agents, S)).

PyTorch is the harness here: the forward and backward work runs in the
library's own kernels, on the env's stream. The env is left holding the final
field. The reference has no reverse mode; the derivative is the one of the
step as the library computes it (LOD splitting, fixed-value Dirichlet faces,
factors held at this dt, agents' update x <- (x + t1)/t2 with
t1 = c*S*rho*, t2 = 1 + c*S + c*U, c = dt*volume/dx^3).
"""
from __future__ import annotations

import torch

from . import FP32, FP64, STEP_CELLS, STEP_DIFFUSION


def _precision(t: torch.Tensor) -> int:
    if t.dtype == torch.float64:
        return FP64
    if t.dtype == torch.float32:
        return FP32
    raise TypeError(f"field dtype {t.dtype} is neither float64 nor float32")


class _Simulate(torch.autograd.Function):
    @staticmethod
    def forward(ctx, env, dt, n_steps, checkpoint_every, agents, rho0, D, lam, sec, upt, sat):
        prec = _precision(rho0)
        if prec != env.precision:
            raise TypeError("rho0 must have the env's precision")
        rho0 = rho0.contiguous()
        _configure(env, D, lam, agents, sec, upt, sat)
        flags = STEP_DIFFUSION | (STEP_CELLS if agents is not None else 0)
        torch.cuda.synchronize(rho0.device)  # rho0 is written on torch's stream, the env works on its own
        env.set_field_device(rho0.data_ptr(), prec)
        env.simulate(dt, n_steps, flags)
        out = torch.empty_like(rho0)
        env.get_field_device(out.data_ptr(), prec)
        env.synchronize()
        ctx.env, ctx.dt, ctx.n, ctx.K, ctx.agents, ctx.flags = env, dt, n_steps, checkpoint_every, agents, flags
        ctx.save_for_backward(rho0, D, lam, sec, upt, sat)
        return out

    @staticmethod
    def backward(ctx, g):
        rho0, D, lam, sec, upt, sat = ctx.saved_tensors
        env = ctx.env
        prec = env.precision
        _configure(env, D, lam, ctx.agents, sec, upt, sat)
        g = g.contiguous()
        if g.dtype != rho0.dtype:
            g = g.to(rho0.dtype)
        grad_rho0 = torch.empty_like(rho0)
        torch.cuda.synchronize(rho0.device)
        env.set_field_device(rho0.data_ptr(), prec)
        want_agents = ctx.agents is not None and any(t is not None and t.requires_grad for t in (sec, upt, sat))
        want_coef = ctx.needs_input_grad[6] or ctx.needs_input_grad[7]  # D, lam; else their sums are skipped
        r = env.adjoint_run(ctx.dt, ctx.n, g.data_ptr(), flags=ctx.flags, checkpoint_every=ctx.K,
                            dL_dinitial_ptr=grad_rho0.data_ptr(), agent_grads=want_agents, coef_grads=want_coef)
        gD = torch.from_numpy(r["D"]).to(D.dtype) if want_coef else None
        gL = torch.from_numpy(r["lambda"]).to(lam.dtype) if want_coef else None
        gs = gu = gt = None
        if want_agents:
            gs = torch.from_numpy(r["secretion"]).to(sec.dtype)
            gu = torch.from_numpy(r["uptake"]).to(upt.dtype)
            gt = torch.from_numpy(r["saturation"]).to(sat.dtype)
        return None, None, None, None, None, grad_rho0, gD, gL, gs, gu, gt


def _configure(env, D, lam, agents, sec, upt, sat):
    env.set_coefficients(D.detach().cpu().double().numpy(), lam.detach().cpu().double().numpy())
    if agents is not None:
        env.set_agents(agents["pos"], agents["volume"], sec.detach().cpu().double().numpy(),
                       upt.detach().cpu().double().numpy(), sat.detach().cpu().double().numpy(), agents["dt"],
                       agents.get("active"))


def simulate(env, rho0: torch.Tensor, D: torch.Tensor, lam: torch.Tensor, dt: float, n_steps: int,
             checkpoint_every: int | None = None, agents: dict | None = None, secretion: torch.Tensor | None = None,
             uptake: torch.Tensor | None = None, saturation: torch.Tensor | None = None) -> torch.Tensor:
    """Differentiable n_steps of the LOD step (plus agents) on ``env``.

    ``agents`` = {"pos": (n, 3), "volume": (n,), "dt": float, "active": (n,) or None}
    holds the non-differentiated agent data; secretion / uptake / saturation
    are the differentiable per-agent rates (host float64 tensors, (n, S))."""
    K = checkpoint_every or max(1, int(round(n_steps ** 0.5)))
    if agents is not None and (secretion is None or uptake is None or saturation is None):
        raise ValueError("agents need secretion, uptake and saturation tensors")
    return _Simulate.apply(env, dt, n_steps, K, agents, rho0, D, lam, secretion, uptake, saturation)
