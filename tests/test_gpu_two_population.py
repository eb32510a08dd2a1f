"""The two-population step on the GPU (pamhd_gpu_npop_*, through the C ABI) against the CPU oracle
(oracle/n_solve.hpp, pinned to the reference's own two-population code by
tests/test_two_population_oracle.py).

The device code restates the oracle's operations in the same order and is compiled without FMA
contraction; +, -, *, / and sqrt are correctly rounded on both, so the bar is bit-for-bit
equality of the state and of the next step's limit."""
import numpy as np
import pytest

import pamhd_b200 as pg
from oracle import pyoracle as po
import states

pytestmark = pytest.mark.gpu


def pair(port, shape, L, solver, min_pressure=0.0):
    n = (shape[2], shape[1], shape[0])
    gpu = pg.TwoPopulationContext(n, L, solver, states.GAMMA_53, 1.0, min_pressure)
    ora = port.two_population_grid(n, L, solver, states.GAMMA_53, 1.0, min_pressure)
    return gpu, ora


@pytest.mark.parametrize("shape", [(4, 5, 6), (1, 7, 9), (1, 1, 24)])
def test_rusanov_steps_are_bitwise(port, shape):
    L = (0.1, 0.12, 0.09)
    U0 = states.two_population_random(shape, np.random.default_rng(3))
    gpu, ora = pair(port, shape, L, pg.RUSANOV)
    gpu.set_state(U0)
    ora.set_state(U0)
    dt = 0.0
    for s in range(10):
        mg = gpu.step(dt)
        mo, flag, _, _ = ora.step(dt)
        assert flag == 0
        assert mg == mo, s
        np.testing.assert_array_equal(gpu.get_state(), ora.get_state())
        dt = 0.4 * mo


@pytest.mark.parametrize("solver", [pg.RUSANOV, pg.HLL])
def test_tiled_grid_is_bitwise(port, solver):
    """A grid of 100 x 254 x 48 cells: the face solves run as 32 x 4 tiles marching several z planes
    each (five per block on a 148-SM GPU, the last chunk three), with partial tiles at the +x and +y
    edges; Rusanov three steps, HLL one.  The state is a random 24 x 127 x 50 pattern repeated twice
    along each axis, whose periods fall across the tile edges."""
    L = (0.1, 0.12, 0.09)
    U0 = np.tile(states.two_population_random((24, 127, 50), np.random.default_rng(7)), (1, 2, 2, 2))
    gpu, ora = pair(port, U0.shape[1:], L, solver)
    gpu.set_state(U0)
    ora.set_state(U0)
    dt = 1e-4
    for s in range(3 if solver == pg.RUSANOV else 1):
        mg = gpu.step(dt)
        mo, flag, _, _ = ora.step(dt)
        assert flag == 0
        assert mg == mo, s
        np.testing.assert_array_equal(gpu.get_state(), ora.get_state())
        dt = 0.4 * mo


def test_hll_step_is_bitwise(port):
    """One HLL step (the reference's split HLL does not keep a state positive for long, see
    test_two_population_oracle.py)."""
    shape, L = (4, 5, 6), (0.1, 0.12, 0.09)
    U0 = states.two_population_random(shape, np.random.default_rng(3))
    gpu, ora = pair(port, shape, L, pg.HLL)
    gpu.set_state(U0)
    ora.set_state(U0)
    mg = gpu.step(1e-4)
    mo, flag, _, _ = ora.step(1e-4)
    assert flag == 0 and mg == mo
    np.testing.assert_array_equal(gpu.get_state(), ora.get_state())


def test_min_pressure_floor_is_bitwise(port):
    shape, L = (4, 5, 6), (0.1, 0.12, 0.09)
    U0 = states.two_population_random(shape, np.random.default_rng(4))
    gpu, ora = pair(port, shape, L, pg.RUSANOV, min_pressure=0.45)   # above some cells' pressure
    gpu.set_state(U0)
    ora.set_state(U0)
    for dt in (0.0, 1e-3, 2e-3):
        assert gpu.step(dt) == ora.step(dt)[0]
    np.testing.assert_array_equal(gpu.get_state(), ora.get_state())


def test_device_loop_equals_host_loop(port):
    """run(n, cfl, t_end) on the device (dt = min(cfl max_dt, t_end - t), the loop of
    tests/mhd/two_reference.cpp) equals the same loop driven from the host on the oracle, and stops
    at t_end."""
    shape, L = (6, 6, 6), (0.1, 0.1, 0.1)
    U0 = states.two_population_random(shape, np.random.default_rng(5))
    gpu, ora = pair(port, shape, L, pg.RUSANOV)
    gpu.set_state(U0)
    ora.set_state(U0)
    t, max_dt, steps, t_end = 0.0, 0.0, 0, 0.02
    while t < t_end:
        dt = min(0.5 * max_dt, t_end - t)
        max_dt, flag, _, _ = ora.step(dt)
        assert flag == 0
        t += dt
        steps += 1
    gpu.run(steps + 4, 0.5, t_end)
    gpu.sync()
    tg, ng, _ = gpu.time()
    assert tg == t and ng == steps
    out = np.zeros_like(U0)
    assert gpu.get_state(out=out) is out   # the caller's array, filled in place
    np.testing.assert_array_equal(out, ora.get_state())
    with pytest.raises(ValueError):
        gpu.get_state(out=out[:12])


def test_failure_reports_oracle_face_and_keeps_state(port):
    shape, L = (4, 4, 4), (0.1, 0.1, 0.1)
    U0 = states.two_population_random(shape, np.random.default_rng(6))
    U0[4, 2, 1, 3] = U0[9, 2, 1, 3] = 0.001   # total energy below the field energy
    gpu, ora = pair(port, shape, L, pg.RUSANOV)
    gpu.set_state(U0)
    ora.set_state(U0)
    _, flag, cell, d = ora.step(1e-3)
    assert flag != 0
    with pytest.raises(pg.PhysicsError) as e:
        gpu.step(1e-3)
    assert e.value.flags == flag and tuple(e.value.cell) == cell and e.value.direction == d
    np.testing.assert_array_equal(gpu.get_state(), U0)
