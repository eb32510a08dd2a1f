"""The discrete adjoint (pamhd_gpu_adjoint) through the C ABI.

The gradient of a functional of the state after N steps with respect to the
initial state is checked against central finite differences of the forward
map on the forward run's dt schedule (held fixed, as the adjoint linearises
it), along seeded random Gaussian directions:
    max over directions |dJ/dU0 . delta - fd(delta)|  <=  1e-6 max over directions |fd|
with fd the central difference (J(U0 + h delta) - J(U0 - h delta)) / 2h.
The perturbed runs are made both on the GPU and by the CPU oracle (the
reference's arithmetic)."""
import numpy as np
import pytest
import torch

import pamhd_b200 as pg
from pamhd_b200 import autograd as pga
from oracle import pyoracle as po
import states

pytestmark = pytest.mark.gpu

REL = 1e-6


def magnetic_energy(U, mask, volume, mu0=1.0):
    """J = sum over masked cells of B^2 / (2 mu0) * volume, and dJ/dU."""
    B = U[5:8]
    J = float((0.5 / mu0 * (B ** 2).sum(0) * mask).sum() * volume)
    seed = np.zeros_like(U)
    seed[5:8] = B / mu0 * mask * volume
    return J, seed


def ot_case(n, solver=pg.HLLD, cfl=0.4):
    U0 = states.orszag_tang(n)
    cfg = pg.Config(n=(n, n, 1), solver=solver, cell_length=(1 / n, 1 / n, 1.0), adiabatic_index=5 / 3,
                    vacuum_permeability=1.0, time_step_factor=cfl)
    x = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(x, x, indexing="xy")
    mask = ((X >= 0.4) & (X <= 0.6) & (Y >= 0.4) & (Y <= 0.6)).astype(float)[None, :, :]
    return U0, cfg, mask


def conservative(rho, v, U0, gamma=5 / 3):
    """U from (rho, v) at the pressure and field of U0 (the reference's initial-state inputs)."""
    p = (gamma - 1) * (U0[4] - 0.5 * (U0[1:4] ** 2).sum(0) / U0[0] - 0.5 * (U0[5:8] ** 2).sum(0))
    U = U0.copy()
    U[0] = rho
    U[1:4] = rho * v
    U[4] = p / (gamma - 1) + 0.5 * rho * (v ** 2).sum(0) + 0.5 * (U0[5:8] ** 2).sum(0)
    return U


def grad_primitive(g, U0):
    """dJ/drho and dJ/dv at fixed p and B from dJ/dU0 (chain rule through U(rho, v))."""
    rho = U0[0]
    v = U0[1:4] / rho
    g_rho = g[0] + (g[1:4] * v).sum(0) + g[4] * 0.5 * (v ** 2).sum(0)
    g_v = g[1:4] * rho + g[4] * rho * v
    return g_rho, g_v


# Roe on a smooth state with no symmetry: on the Orszag-Tang vortex whole lines of faces hold a
# Roe-averaged transverse field of exactly zero, where the Roe flux is not differentiable (the
# Alfven waves' direction bet2, bet3 is then arbitrary, mhd/roe_athena.hpp:97-105) and a finite
# difference straddles the jump; the other solvers are differentiable there up to kinks the
# adjoint resolves as a central difference does
@pytest.mark.parametrize("solver,case", [(pg.RUSANOV, "ot"), (pg.HLL, "ot"), (pg.HLLD, "ot"), (pg.ROE, "smooth")])
def test_small_grid_against_gpu_and_oracle_perturbed_runs(port, solver, case):
    n, steps, every = 32, 24, 5
    U0, cfg, mask = ot_case(n, solver)
    if case == "smooth":
        U0 = states.smooth_3d((1, n, n), np.random.default_rng(41), amp=0.1)
    vol = 1 / n ** 2
    ctx = pg.Context(cfg)
    ctx.set_state(U0)
    ctx.step(0.0)  # priming: the adjoint starts from primed speeds
    U0p = ctx.get_state()
    # forward with checkpoints + adjoint of J at the end
    ctx.set_state(U0p)
    ctx.step(0.0)
    # the seed needs U_N: one forward pass first
    ctx.steps(steps, 1e300)
    UN = ctx.get_state()
    dts = ctx.dt_history(steps)
    J0, seed = magnetic_energy(UN, mask, vol)
    ctx.set_state(U0p)
    grad, _, dts2 = ctx.adjoint(steps, every, seed, dt_in=dts)
    np.testing.assert_array_equal(dts2, dts)
    rng = np.random.default_rng(20261205)
    ora = port.grid(po.make_cfg((n, n, 1), solver, (1 / n, 1 / n, 1.0), 5 / 3, 1.0, 0.4), threads=8)
    checks = []
    for k in range(4):
        delta = rng.normal(size=U0p.shape) * np.abs(U0p).reshape(8, -1).max(1)[:, None, None, None]
        h = 1e-6
        Js = []
        for sgn in (1, -1):
            ctx.set_state(U0p + sgn * h * delta)
            ctx.steps_dt(dts)
            Js.append(magnetic_energy(ctx.get_state(), mask, vol)[0])
        fd_gpu = (Js[0] - Js[1]) / (2 * h)
        Jo = []
        for sgn in (1, -1):
            ora.set_state(U0p + sgn * h * delta)
            for dt in dts:
                assert ora.step_dt(dt) == 0
            Jo.append(magnetic_energy(ora.get_state(), mask, vol)[0])
        fd_ora = (Jo[0] - Jo[1]) / (2 * h)
        ad = float((grad * delta).sum())
        checks.append((ad, fd_gpu, fd_ora))
    # random directions can nearly cancel: the bar is relative to the largest derivative tested
    scale = max(abs(c[0]) for c in checks)
    for ad, fd_gpu, fd_ora in checks:
        assert abs(ad - fd_gpu) <= REL * scale, (ad, fd_gpu)
        assert abs(ad - fd_ora) <= REL * scale, (ad, fd_ora)


def test_orszag_tang_256_adjoint_config():
    """The configured case: Orszag-Tang 256^2, HLLD, 200 steps, checkpoints every 20 steps;
    J = magnetic energy in [0.4, 0.6]^2 at the last step; gradient with respect to the initial
    density and velocity, checked by central differences (h = 1e-6 of each field's rms) along
    16 seeded Gaussian directions.  CFL 0.25: the reference scheme loses positivity on this
    problem at t = 0.104 whatever the CFL (step 158 at CFL 0.4), and 200 steps at 0.25 end at
    t = 0.084.

    The bar is normwise over the 16 directions: max |ad - fd| <= 1e-6 max |fd|.  The run is close
    to the scheme's positivity limit (random perturbations of 1e-5 of the rms make it fail at
    step 178) and its fluxes have kinks (max, min, |.|, wave-region switches) that a
    perturbation of 1e-6 crosses, so the central difference at h = 1e-6 itself differs from
    the exact directional derivative: by up to 5e-6 relative in the directions where the
    derivative is small, shrinking as h shrinks (direction 5: 4.7e-6 at h = 1e-6, 5e-7 at
    1e-7).  Richardson extrapolation of the differences at h and h/2,
    fd = (4 D(h/2) - D(h)) / 3, removes their smooth O(h^2) part."""
    n, steps, every = 256, 200, 20
    U0, cfg, mask = ot_case(n, cfl=0.25)
    vol = 1 / n ** 2
    ctx = pg.Context(cfg)
    ctx.set_state(U0)
    ctx.step(0.0)
    ctx.steps(steps, 1e300)
    dts = ctx.dt_history(steps)
    J0, seed = magnetic_energy(ctx.get_state(), mask, vol)
    ctx.set_state(U0)
    ctx.step(0.0)
    grad, _, _ = ctx.adjoint(steps, every, seed, dt_in=dts)
    g_rho, g_v = grad_primitive(grad, U0)
    rho0 = U0[0]
    v0 = U0[1:4] / rho0
    rng = np.random.default_rng(20261205)
    rms_rho = np.sqrt((rho0 ** 2).mean())
    rms_v = np.sqrt((v0[:2] ** 2).mean())
    ads, fds = [], []
    for k in range(16):
        d_rho = rng.normal(size=rho0.shape)
        d_v = rng.normal(size=v0.shape)
        d_v[2] = 0.0
        h_rho, h_v = 1e-6 * rms_rho, 1e-6 * rms_v
        D = []
        for frac in (1.0, 0.5):
            Js = []
            for sgn in (1, -1):
                U = conservative(rho0 + sgn * frac * h_rho * d_rho, v0 + sgn * frac * h_v * d_v, U0)
                ctx.set_state(U)
                ctx.step(0.0)
                ctx.steps_dt(dts)
                Js.append(magnetic_energy(ctx.get_state(), mask, vol)[0])
            D.append((Js[0] - Js[1]) / (2 * frac))
        fds.append((4 * D[1] - D[0]) / 3)
        ads.append(float((g_rho * d_rho).sum() * h_rho + (g_v * d_v).sum() * h_v))
    ads, fds = np.array(ads), np.array(fds)
    err = np.abs(ads - fds).max() / np.abs(fds).max()
    assert err <= REL, (err, ads, fds)


def test_inflow_state_gradient():
    """Sensitivity to the state of a VALUE (inflow) side against central differences of runs
    with that state perturbed."""
    n, steps = 24, 12
    b = states.solar_wind_ensemble(nboxes=1, sizes=(n,))[0]
    rng = np.random.default_rng(4)
    U0 = states.ensemble_state(b)
    U0[0] *= 1 + 0.05 * rng.random(U0[0].shape)

    def cfg_for(inflow):
        return pg.Config(n=(n, n, n), solver=pg.HLL, cell_length=(states.EARTH_RADIUS_CELL,) * 3,
                         adiabatic_index=5 / 3, vacuum_permeability=states.MU0_SI, time_step_factor=0.5,
                         bc_lo=(pg.BC_VALUE, pg.BC_COPY, pg.BC_COPY), bc_hi=(pg.BC_COPY,) * 3,
                         value_lo=[inflow, None, None])

    inflow = b["inflow"]
    ctx = pg.Context(cfg_for(inflow))
    ctx.set_state(U0)
    ctx.step(0.0)
    ctx.steps(steps, 1e300)
    dts = ctx.dt_history(steps)
    UN = ctx.get_state()
    w = rng.normal(size=UN.shape) / np.abs(UN).reshape(8, -1).max(1)[:, None, None, None]
    J = lambda U: float((w * U).sum())
    ctx.set_state(U0)
    ctx.step(0.0)
    _, gv, _ = ctx.adjoint(steps, 4, w, dt_in=dts)
    for comp in (0, 1, 4, 6):
        h = 1e-6 * abs(inflow[comp]) if inflow[comp] != 0 else 1e-6 * np.abs(inflow[5:8]).max()
        Js = []
        for sgn in (1, -1):
            v = inflow.copy()
            v[comp] += sgn * h
            c2 = pg.Context(cfg_for(v))
            c2.set_state(U0)
            c2.step(0.0)
            c2.steps_dt(dts)
            Js.append(J(c2.get_state()))
        fd = (Js[0] - Js[1]) / (2 * h)
        assert abs(gv[0, 0, comp] - fd) <= 1e-5 * abs(fd), (comp, gv[0, 0, comp], fd)


def test_autograd_gradcheck():
    """torch.autograd.gradcheck of the wrapped multi-step map on a tiny periodic 3-D grid."""
    rng = np.random.default_rng(6)
    U0 = states.smooth_3d((3, 4, 5), rng, amp=0.1)
    cfg = pg.Config(n=(5, 4, 3), solver=pg.HLLD, cell_length=(0.2, 0.25, 0.3), time_step_factor=0.4)
    ctx = pg.Context(cfg)
    ctx.set_state(U0)
    ctx.step(0.0)
    ctx.steps(3, 1e300)
    dts = ctx.dt_history(3)
    x = torch.tensor(U0, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda u: pga.steps(u, ctx, dts, every=2), (x,), eps=1e-6, atol=1e-7,
                                    rtol=1e-5, fast_mode=True)
