"""Reverse-mode adjoint of the orbit loss: checked against central finite
differences on short horizons (N = 100) and against the forward-mode
tangent map J^T v on long ones (N = 10^4), through the C ABI and through
torch.autograd."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import TUNES
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from henon_map_cpp_b200 import autograd as AG  # noqa: E402

THETA = [2 * math.pi * TUNES[0], 2 * math.pi * TUNES[1], 16.0, 0.1]


def c5_points(n, seed=5):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, 0.3, n)
    y = rng.uniform(0, 0.3, n)
    px = rng.normal(0, 0.01, n)
    py = rng.normal(0, 0.01, n)
    return [torch.tensor(a, dtype=torch.float64, device="cuda") for a in (x, px, y, py)]


def test_loss_matches_oracle_orbit(gpu):
    pts = c5_points(64)
    th = torch.tensor(THETA, dtype=torch.float64)
    r = AG.per_particle(*pts, th, 300, mode="loss")
    host = [p.cpu().numpy() for p in pts]
    tabs = O.tables(300, *TUNES, "sps", epsilon=16.0)
    w = O.birkhoff_weights(300)
    x, px, y, py = host
    steps = np.zeros(64, np.uint32)
    loss = np.zeros(64)
    for k in range(300):
        x, px, y, py, steps = O.track(x, px, y, py, steps, tabs, 1, 0.1, 10.0)
        loss += w[k] * ((x * x + px * px) + (y * y + py * py))
    alive = steps == 300
    np.testing.assert_array_equal(r["survived"].cpu().numpy(), alive)
    np.testing.assert_array_equal(r["steps"].cpu().numpy(), steps)
    np.testing.assert_allclose(r["loss"].cpu().numpy()[alive], loss[alive], rtol=1e-13)


@pytest.mark.parametrize("reverse", ["inverse", "replay"])
def test_adjoint_matches_central_differences(gpu, reverse):
    n_turns = 100
    pts = c5_points(48, seed=9)
    th = torch.tensor(THETA, dtype=torch.float64)
    r = AG.per_particle(*pts, th, n_turns, checkpoint_every=7, reverse=reverse)
    surv = r["survived"].cpu().numpy()
    assert surv.all()

    def losses(points, theta):
        return AG.per_particle(*points, torch.tensor(theta, dtype=torch.float64), n_turns,
                               mode="loss")["loss"].cpu().numpy()

    # initial conditions: perturb every particle's coordinate c at once
    # (particles are independent, so each loss sees only its own shift)
    for c in range(4):
        h = 1e-6
        up = [p.clone() for p in pts]
        dn = [p.clone() for p in pts]
        up[c] += h
        dn[c] -= h
        fd = (losses(up, THETA) - losses(dn, THETA)) / (2 * h)
        ad = r["grad_ic"][c].cpu().numpy()
        np.testing.assert_allclose(ad, fd, rtol=2e-6, atol=1e-9, err_msg=f"coordinate {c}")
    # parameters (omega_x0, omega_y0, epsilon, mu): per-particle sums
    for j in range(4):
        h = 1e-6 * max(1.0, abs(THETA[j]))
        tu, td = list(THETA), list(THETA)
        tu[j] += h
        td[j] -= h
        fd = (losses(pts, tu) - losses(pts, td)) / (2 * h)
        ad = r["grad_theta"][j].cpu().numpy()
        np.testing.assert_allclose(ad, fd, rtol=2e-5, atol=1e-9, err_msg=f"parameter {j}")


@pytest.mark.parametrize("reverse", ["inverse", "replay"])
def test_adjoint_equals_forward_tangent_long_horizon(gpu, reverse):
    n_turns = 10_000
    pts = c5_points(2048, seed=3)
    th = torch.tensor(THETA, dtype=torch.float64)
    adj = AG.per_particle(*pts, th, n_turns, checkpoint_every=100, reverse=reverse)
    tan = AG.per_particle(*pts, th, n_turns, mode="tangent")
    surv = adj["survived"].cpu().numpy()
    np.testing.assert_array_equal(surv, tan["survived"].cpu().numpy())
    a = adj["grad_ic"].cpu().numpy()[:, surv]
    t = tan["grad_ic"].cpu().numpy()[:, surv]
    rel = np.max(np.abs(a - t), axis=0) / np.max(np.abs(t), axis=0)
    # Regular orbits: 1e-10.  Chaotic ones have gradients ~exp(lambda N);
    # both sides are then accurate to a relative error that grows with
    # |grad|, so the bound is checked on the well-conditioned majority.
    assert surv.sum() > 1000
    assert np.mean(rel < 1e-10) >= 0.95, (np.mean(rel < 1e-10), np.nanmax(rel))
    norm = np.max(np.abs(t), axis=0)
    assert np.all(rel[norm < 1e3] < 1e-10)


def test_reverse_sweeps_agree_and_mu_gradient_at_zero(gpu):
    pts = c5_points(256, seed=2)
    for mu in (0.1, 0.0):
        th = torch.tensor(THETA[:3] + [mu], dtype=torch.float64)
        a = AG.per_particle(*pts, th, 3000, checkpoint_every=100, reverse="inverse")
        b = AG.per_particle(*pts, th, 3000, checkpoint_every=100, reverse="replay")
        s = a["survived"]
        # grad_theta sums 3000 per-turn terms in a different order in the
        # two sweeps (per-turn factors vs. two running sums), so it agrees to
        # a few 1e-12; the initial-condition gradient to ~1e-14.
        for k, tol in (("grad_ic", 1e-12), ("grad_theta", 1e-10)):
            x, y = a[k][:, s].cpu().numpy(), b[k][:, s].cpu().numpy()
            rel = np.abs(x - y) / np.maximum(np.abs(y), 1e-300)
            assert np.median(rel) < tol, (k, mu, np.median(rel))
        # dL/dmu is the octupole's derivative, nonzero also at mu = 0
        assert np.all(b["grad_theta"][3, s].cpu().numpy() != 0.0)


def test_autograd_function(gpu):
    n_turns = 200
    pts = [p.clone().requires_grad_(True) for p in c5_points(256, seed=1)]
    th = torch.tensor(THETA, dtype=torch.float64, requires_grad=True)
    loss = AG.orbit_loss(*pts, th, n_turns, checkpoint_every=20)
    loss.backward()
    r = AG.per_particle(*[p.detach() for p in pts], th.detach(), n_turns, checkpoint_every=20)
    surv = r["survived"]
    count = surv.sum().item()
    torch.testing.assert_close(loss.detach(), r["loss"][surv].sum() / count, rtol=1e-14, atol=0)
    torch.testing.assert_close(pts[0].grad, r["grad_ic"][0] / count, rtol=1e-14, atol=0)
    torch.testing.assert_close(th.grad, r["grad_theta"].sum(dim=1).cpu() / count, rtol=1e-12,
                               atol=0)
    # loss-only path (no gradient requested)
    with torch.no_grad():
        l2 = AG.orbit_loss(*[p.detach() for p in pts], th.detach(), n_turns)
    torch.testing.assert_close(l2, loss.detach(), rtol=0, atol=0)


def test_adjoint_vs_forward_tangent_c5(gpu):
    # The adjoint configuration itself: 65,536 particles, x0, y0 ~ U[0, 0.3],
    # px0, py0 ~ N(0, 0.01^2), eps 16, mu 0.1, N = 10^4, checkpoints every
    # 100.  The reverse sweep's gradients with respect to the initial
    # conditions AND theta = (omega_x0, omega_y0, eps, mu) against forward-
    # mode propagation of the tangent map and of d x / d theta.
    #
    # Conditioning criterion.  Per particle the compared vector is
    #     g = (dL/dx0, dL/dpx0, dL/dy0, dL/dpy0, theta_j dL/dtheta_j),
    # the theta part as derivatives with respect to log theta so that the
    # four parameters share one scale, and rel_i = max|adjoint - tangent| /
    # max|tangent|.  Both methods sum N = 10^4 terms w_k grad A . (d x_k /
    # d input) whose rounding errors grow with the tangent map, so rel_i is
    # bounded by c u N max(1, kappa_i), u = 2^-53, kappa_i = max_c
    # |dL_i/d x0_c| (the propagated tangent map seen through the loss: a
    # regular orbit's grows linearly, kappa up to ~10^3; a chaotic one's
    # exponentially, kappa up to ~10^37 here), and c the cancellation
    # inside the sum (sum of |terms| over |sum|), measured below 10^3 on
    # this set.  Required: every particle within that bound with c = 10^3,
    # and 1e-10 relative on at least 99.9 % of the survivors.
    n_turns = 10_000
    pts = c5_points(65_536, seed=5)
    th = torch.tensor(THETA, dtype=torch.float64)
    adj = AG.per_particle(*pts, th, n_turns, checkpoint_every=100, reverse="inverse")
    tan = AG.per_particle(*pts, th, n_turns, mode="tangent")
    surv = adj["survived"].cpu().numpy()
    np.testing.assert_array_equal(surv, tan["survived"].cpu().numpy())
    assert surv.sum() > 60_000
    scale = np.abs(np.asarray(THETA))[:, None]
    a = np.concatenate([adj["grad_ic"].cpu().numpy()[:, surv],
                        scale * adj["grad_theta"].cpu().numpy()[:, surv]])
    t = np.concatenate([tan["grad_ic"].cpu().numpy()[:, surv],
                        scale * tan["grad_theta"].cpu().numpy()[:, surv]])
    rel = np.max(np.abs(a - t), axis=0) / np.max(np.abs(t), axis=0)
    kappa = np.max(np.abs(t[:4]), axis=0)
    bound = 1e3 * 2.0 ** -53 * n_turns * np.maximum(1.0, kappa)
    stats = (f"survivors {surv.sum()}; rel <= 1e-10 on {np.mean(rel <= 1e-10):.5f} of them; "
             f"max rel / bound {np.max(rel / bound):.3f}; kappa max {kappa.max():.2e}; "
             f"rel quantiles 50/99/99.9 % {np.quantile(rel, [0.5, 0.99, 0.999])}")
    print("\n" + stats)
    assert np.mean(rel <= 1e-10) >= 0.999, stats
    assert np.all(rel <= bound), stats
