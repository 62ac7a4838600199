"""Differentiable orbit loss: torch.autograd.Function over the reverse-mode
adjoint of the modulated Henon map (hm_adjoint in include/henon_b200.h).

    theta = torch.tensor([2*pi*0.168, 2*pi*0.201, 16.0, 0.1], dtype=torch.float64,
                         requires_grad=True)       # (omega_x0, omega_y0, epsilon, mu)
    loss = orbit_loss(x0, px0, y0, py0, theta, n_turns=10_000, checkpoint_every=100)
    loss.backward()        # x0.grad ... py0.grad and theta.grad

The loss is the mean over particles that survive all n_turns of the
Birkhoff-weighted average of x^2+px^2+y^2+py^2 along the orbit:
    L = (1/|S|) sum_{i in S} sum_{k<N} w_k A(x_i after turn k),
w = birkhoff_weights(N).  The survivor set S is piecewise constant in the
inputs and is not differentiated.  omega_{x,y}0 = 2 pi tune_{x,y} with an
SPS modulation omega(k) = omega0 (1 + epsilon S_k).

With torch.distributed initialised and `group` given, particles are taken as
this rank's shard: the loss sum, survivor count and theta gradient are summed
over the ranks (one all_reduce of 6 doubles) before normalising.
"""
from __future__ import annotations

import math

import torch

from . import _capi as C

_cache: dict = {}


def _tracker(n_turns: int, omega_x0: float, omega_y0: float, epsilon: float, arith: int):
    key = (n_turns, omega_x0, omega_y0, epsilon)
    t = _cache.get(key)
    if t is None:
        _cache.clear()
        t = C.Tracker(n_turns, omega_x0 / (2 * math.pi), omega_y0 / (2 * math.pi), "sps",
                      float("nan"), epsilon, 0)
        _cache[key] = t
    t.arith = arith
    return t


def _run(x0, px0, y0, py0, theta, n_turns, barrier, checkpoint_every, arith, mode):
    wx, wy, eps, mu = (float(v) for v in theta.detach().cpu().tolist())
    t = _tracker(n_turns, wx, wy, eps, arith)
    dev = x0.device
    xs = [a.detach().to(dev, torch.float64).contiguous() for a in (x0, px0, y0, py0)]
    n = xs[0].numel()
    loss = torch.empty(n, dtype=torch.float64, device=dev)
    surv = torch.empty(n, dtype=torch.uint8, device=dev)
    steps = torch.empty(n, dtype=torch.int32, device=dev)
    g_ic = torch.empty((4, n), dtype=torch.float64, device=dev)
    g_th = torch.empty((4, n), dtype=torch.float64, device=dev)
    ws = None
    if mode in (0, 3):
        nb = C.load().hm_adjoint_workspace_bytes(n, n_turns, checkpoint_every)
        ws = torch.empty(nb, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize(dev)
    C.call("hm_adjoint", t.h, *[a.data_ptr() for a in xs], n, mu, barrier, n_turns,
           checkpoint_every, mode, loss.data_ptr(), surv.data_ptr(), steps.data_ptr(),
           g_ic.data_ptr(), g_th.data_ptr(), ws.data_ptr() if ws is not None else None,
           torch.cuda.current_stream(dev).cuda_stream)
    return loss, surv, steps, g_ic, g_th


class OrbitLoss(torch.autograd.Function):
    """Forward runs the adjoint too (one kernel does both sweeps); backward
    scales the stored gradients."""

    @staticmethod
    def forward(ctx, x0, px0, y0, py0, theta, n_turns, barrier, checkpoint_every, arith, group,
                reverse_mode):
        need = any(ctx.needs_input_grad[:5])
        loss, surv, _, g_ic, g_th = _run(x0, px0, y0, py0, theta, n_turns, barrier,
                                         checkpoint_every, arith, reverse_mode if need else 2)
        sums = torch.cat([loss.sum().reshape(1), surv.sum(dtype=torch.float64).reshape(1),
                          g_th.sum(dim=1) if need else torch.zeros(4, dtype=torch.float64,
                                                                    device=loss.device)])
        if group is not None:
            import torch.distributed as dist
            dist.all_reduce(sums, group=group)
        count = sums[1]
        ctx.save_for_backward(g_ic, sums[2:] / count)
        ctx.count = count
        ctx.theta_device = theta.device
        return sums[0] / count

    @staticmethod
    def backward(ctx, grad_out):
        g_ic, g_th = ctx.saved_tensors
        s = grad_out / ctx.count
        gx, gpx, gy, gpy = (g_ic[k] * s for k in range(4))
        return (gx, gpx, gy, gpy, (g_th * grad_out).to(ctx.theta_device), None, None, None, None,
                None, None)


# Reverse sweeps: "inverse" rebuilds each segment backwards with the map's
# exact inverse from the next checkpoint (no scratch traffic); "replay"
# recomputes it forward from its checkpoint into a scratch buffer (states
# identical to the forward orbit).
_REVERSE = {"inverse": 3, "replay": 0}


def orbit_loss(x0, px0, y0, py0, theta, n_turns: int, barrier: float = 10.0,
               checkpoint_every: int = 100, arith: str = "exact", group=None,
               reverse: str = "inverse"):
    """Mean Birkhoff-weighted orbit action over surviving particles (a 0-d
    tensor that backpropagates to x0..py0 and theta)."""
    mode = C.ARITH_FAST if arith == "fast" else C.ARITH_EXACT
    return OrbitLoss.apply(x0, px0, y0, py0, theta, int(n_turns), float(barrier),
                           int(checkpoint_every), mode, group, _REVERSE[reverse])


def per_particle(x0, px0, y0, py0, theta, n_turns: int, barrier: float = 10.0,
                 checkpoint_every: int = 100, arith: str = "exact", mode: str = "adjoint",
                 reverse: str = "inverse"):
    """Per-particle values without autograd: dict with loss, survived, steps
    and grad_ic [4, n], grad_theta [4, n]: by the reverse sweep (mode
    "adjoint") or by forward-mode propagation of the tangent map and of the
    state's theta derivatives (mode "tangent")."""
    m = {"adjoint": _REVERSE[reverse], "tangent": 1, "loss": 2}[mode]
    a = C.ARITH_FAST if arith == "fast" else C.ARITH_EXACT
    loss, surv, steps, g_ic, g_th = _run(x0, px0, y0, py0, theta, int(n_turns), float(barrier),
                                         int(checkpoint_every), a, m)
    out = {"loss": loss, "survived": surv.bool(), "steps": steps}
    if m != 2:
        out["grad_ic"] = g_ic
    if m != 2:
        out["grad_theta"] = g_th
    return out
