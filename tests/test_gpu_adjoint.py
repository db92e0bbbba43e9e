"""Discrete adjoint on the GPU, through the C ABI (grhd_adjoint_*).

* The RHS and RK4-step vector-Jacobian products agree with central
  differences of the operator's own grhd_compute_rhs / grhd_advance_rk4
  (with their accretion rate / integral) on a small torus state.
* The adjoint's forward sweep reproduces the operator's RK4 run and its
  accretion integral (the FP64 forward).
* The gradient of J = integral of the accretion rate with respect to the
  eight torus parameters, from the torch.autograd.Function wrapper, agrees
  with central finite differences (h = 1e-6 relative) to 1e-5.
Central differences whose step crosses a switch of the scheme (limiter,
HLLE or floor branch) measure another one-sided slope, so every
comparison takes the closest of the differences over h in {1e-6, 1e-7}
(and 1e-8 for the single-evaluation VJPs).  The VJP checks weight and
perturb only cells with pressure above 1e-6: con2prim stops at an absolute
residual of 1e-12, so in the atmosphere (pressure 1e-12) its output moves
with the solver's stopping point rather than smoothly, and differences
there measure that, not the derivative of the root.  The torus initial
state has no vertical velocity and is mirror symmetric about z = 0, so
every vertical-velocity slope and every mid-plane slope sits exactly on a
limiter switch; the VJP checks first add 1e-4 relative noise to the
well-conditioned cells (the gradient check keeps the symmetric state: the
torus parameters preserve the symmetry, along which the switches stay
put)."""
import pytest
import torch

pytestmark = pytest.mark.gpu

N = 24
HALF_WIDTH = 12.0


def _workload(steps=1, every=1, accretion_radius=2.5):
    from grdzhadzha_b200 import workloads as W
    return W.adjoint_torus(n=N, half_width=HALF_WIDTH, steps=steps,
                           checkpoint_every=every,
                           accretion_radius=accretion_radius)


def _off_switches(lv, mask, seed):
    """Relative 1e-4 noise on the conserved variables of masked cells, and
    a vertical momentum of 1e-4 D."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    u = lv.interior(slice(0, 5))
    noise = torch.rand(u.shape, generator=g, device="cuda",
                       dtype=torch.float64) * 2 - 1
    u.mul_(1.0 + 1e-4 * noise * mask)
    kick = torch.rand(u[0].shape, generator=g, device="cuda",
                      dtype=torch.float64) * 2 - 1
    u[3].add_(1e-4 * u[0] * kick * mask[0])


def _interior_perturbed(lv, direction, h):
    from grdzhadzha_b200 import LevelBox
    out = LevelBox(lo=lv.lo, hi=lv.hi, ghost=lv.ghost,
                   device=lv.state.device)
    out.state.copy_(lv.state)
    u = out.interior(slice(0, 5))
    u.mul_(1.0 + h * direction)
    return out


def _well_conditioned(lv):
    """1 where the cell's pressure is above 1e-6, else 0 (interior)."""
    from grdzhadzha_b200.operator import PRESSURE
    p = lv.interior(slice(PRESSURE, PRESSURE + 1))
    return (p > 1e-6).to(torch.float64)


def _best(adj, fds):
    return min(fds, key=lambda f: abs(f - adj))


def test_rhs_vjp_matches_operator_differences():
    torch.manual_seed(1)
    op, adj = _workload()
    lv = adj.initial_state()
    mask = _well_conditioned(lv)
    _off_switches(lv, mask, 11)
    lam = torch.randn((5,) + lv.interior_shape, dtype=torch.float64,
                      device="cuda") * mask
    mu = 0.3
    state_bar, spin_bar = adj.rhs_vjp(lv, lam, mu)
    direction = torch.randn_like(lam) * mask

    def J(level):
        rhs = level.new_rhs()
        op.compute_rhs(rhs, level)
        mdot, _ = op.accretion()
        return float((lam * rhs).sum()) + mu * mdot

    u0 = lv.interior(slice(0, 5))
    adj_dir = float((state_bar * direction * u0).sum())
    fds = [(J(_interior_perturbed(lv, direction, h)) -
            J(_interior_perturbed(lv, direction, -h))) / (2 * h)
           for h in (1e-6, 1e-7, 1e-8)]
    fd = _best(adj_dir, fds)
    assert abs(adj_dir - fd) <= 1e-6 * abs(fd), (adj_dir, fds)
    assert spin_bar != 0.0


def test_step_vjp_matches_operator_differences():
    torch.manual_seed(2)
    op, adj = _workload()
    lv = adj.initial_state()
    mask = _well_conditioned(lv)
    _off_switches(lv, mask, 12)
    lam = torch.randn((5,) + lv.interior_shape, dtype=torch.float64,
                      device="cuda") * mask
    mu = 0.7
    state_bar, _ = adj.step_vjp(lv, lam, mu)
    direction = torch.randn_like(lam) * mask
    dt = adj.dt

    def J(level):
        op.accretion(reset=True)
        op.advance_rk4(level, dt=dt)
        _, integral = op.accretion()
        return float((lam * level.interior(slice(0, 5))).sum()) + \
            mu * integral

    u0 = lv.interior(slice(0, 5))
    adj_dir = float((state_bar * direction * u0).sum())
    fds = [(J(_interior_perturbed(lv, direction, h)) -
            J(_interior_perturbed(lv, direction, -h))) / (2 * h)
           for h in (1e-6, 1e-7, 1e-8)]
    fd = _best(adj_dir, fds)
    assert abs(adj_dir - fd) <= 1e-5 * abs(fd), (adj_dir, fds)


def test_forward_sweep_matches_operator_run():
    steps = 6
    op, adj = _workload(steps=steps, every=4)
    J = adj.forward()
    lv = adj.initial_state()
    op.accretion(reset=True)
    for _ in range(steps):
        op.advance_rk4(lv, dt=adj.dt)
    _, integral = op.accretion()
    assert J != 0.0
    assert abs(J - integral) <= 1e-10 * abs(integral)


def test_gradient_matches_central_differences():
    """J through the sphere r = 5, inside the torus body, where it depends
    on every parameter from the first step.  Four steps (two checkpoint
    segments): over longer runs the trajectory crosses limiter, floor and
    HLLE switches within h = 1e-6 of the parameters, J(theta) is only
    piecewise smooth at that scale and central differences stop measuring
    a derivative (at 24^3 they scatter by 1e-4 after 12 steps)."""
    from grdzhadzha_b200.adjoint import THETA_NAMES, AccretionIntegral
    steps, every = 4, 3
    op, adj = _workload(steps=steps, every=every, accretion_radius=5.0)
    theta = torch.tensor(adj.theta(), dtype=torch.float64,
                         requires_grad=True)
    J = AccretionIntegral.apply(theta, adj)
    J.backward()
    grad = theta.grad.tolist()
    base = adj.theta()
    for k, name in enumerate(THETA_NAMES):
        fds = []
        for rel in (1e-6, 1e-7):
            h = rel * max(abs(base[k]), 0.1)
            tp, tm = list(base), list(base)
            tp[k] += h
            tm[k] -= h
            fds.append((adj.forward(tp) - adj.forward(tm)) / (2 * h))
        fd = _best(grad[k], fds)
        assert abs(grad[k] - fd) <= 1e-5 * abs(fd), (name, grad[k], fds)


def test_tangent_linear_sweep_equals_the_adjoint():
    """The adjoint checked without finite differences: the tangent-linear
    sweep (grhd_adjoint_tangent: forward mode along the same taped steps,
    recorded limiter branches and branch decisions) gives dJ = sum_k v_k
    dJ/dtheta_k, which must equal <grad, v> from the backward sweep for
    every direction v.  12 RK4 steps (three checkpoint segments), where
    central differences no longer measure a derivative.

    * J through r = 5 (inside the torus body, where J depends on every
      parameter): each unit direction to 1e-9 of its own component
      (measured 1e-12 .. 1.9e-10, spin the largest) and a random direction
      to 1e-10 of sum_k |g_k v_k|.
    * J through r = 2.5 (the adjoint workload's sphere; over 12 steps only
      atmosphere inflow crosses it, J ~ 1e-8): the components span eight
      decades (spin 2.4e-9 .. mode_2 7e-13) and agree to 1e-7 of the
      gradient's norm (measured 7e-9): the tangents and adjoints carry
      rounding at the scale of the torus region's, ~1e8 times those that
      reach the sphere."""
    import numpy as np
    from grdzhadzha_b200.adjoint import THETA_NAMES
    steps, every = 12, 4
    for R in (5.0, 2.5):
        op, adj = _workload(steps=steps, every=every, accretion_radius=R)
        J0 = adj.forward()
        grad = np.asarray(adj.backward())
        norm = float(np.sqrt((grad ** 2).sum()))
        rows = []
        for k, name in enumerate(THETA_NAMES):
            e = [0.0] * 8
            e[k] = 1.0
            J1, dJ = adj.tangent(e)
            assert abs(J1 - J0) <= 1e-14 * abs(J0), (J1, J0)
            rows.append((name, float(grad[k]), dJ))
            if R == 5.0:
                assert abs(dJ - grad[k]) <= 1e-9 * abs(grad[k]), rows[-1]
            else:
                assert abs(dJ - grad[k]) <= 1e-7 * norm, (rows[-1], norm)
        v = np.random.default_rng(7).uniform(-1.0, 1.0, 8)
        _, dJ = adj.tangent(list(v))
        want = float(np.dot(grad, v))
        print(f"R = {R}: tangent vs adjoint {rows}; random direction "
              f"{dJ} vs {want}")
        if R == 5.0:
            assert abs(dJ - want) <= 1e-10 * float(np.abs(grad * v).sum())
        else:
            assert abs(dJ - want) <= 1e-7 * norm * float(np.linalg.norm(v))
        del adj, op
