"""The oracle's local time stepping (oracle/substep.hpp), CPU only.

The reference ships no output of a substepped run (its substep configurations,
tests/mhd/config_files/hydrodynamic/substep/, have no golden files), so the restatement is held
to properties of the reference's algorithm: with every exponent 0 it is the plain cell-centred
step bit for bit; with one common exponent k every cell updates once per step with the substep
times 2^k, the plain step again; the periods follow the configured regions, neighbours differ by
at most one exponent, and the totals stay conserved on a periodic grid."""
import numpy as np
import pytest

from oracle import pyoracle as po
import states

SHAPE, N, L = (1, 12, 12), (12, 12, 1), (0.1, 0.1, 1.0)


def regions(shape):
    """The exponents of tests/mhd/config_files/hydrodynamic/substep/100cells/x2.json on the grid
    [-0.5, 0.5]: 0 where y < 0, 1 elsewhere."""
    y = (np.arange(shape[1]) + 0.5) / shape[1] - 0.5
    return np.broadcast_to(np.where(y < 0, 0, 1)[None, :, None], shape).astype(np.int32)


@pytest.mark.parametrize("solver", list(po.SOLVERS))
@pytest.mark.parametrize("k", [0, 1, 2])
def test_common_exponent_is_the_plain_step(port, solver, k):
    U = states.smooth_3d(SHAPE, np.random.default_rng(2))
    cfg = po.make_cfg(N, po.SOLVERS[solver], L, states.GAMMA_53, 1.0, 0.4)
    g, c = port.substep_grid(cfg), port.grid(cfg)
    g.set_state(U)
    c.set_state(U)
    e = np.full(SHAPE, k, np.int32)
    g.set_exponents(e, e)
    for s in range(6):
        cap = 0.0 if s == 0 else 1.0
        dt, steps, periods, flag = g.step(cap)
        dc = c.step(cap)[0]
        assert flag == 0 and dt == dc
        np.testing.assert_array_equal(g.get_state(), c.get_state())


def test_regions_get_their_periods_and_conserve(port):
    U = states.smooth_3d(SHAPE, np.random.default_rng(3))
    cfg = po.make_cfg(N, po.HLLD, L, states.GAMMA_53, 1.0, 0.4)
    g = port.substep_grid(cfg)
    g.set_state(U)
    e = regions(SHAPE)
    g.set_exponents(e, e)
    g.step(0.0)
    for _ in range(5):
        dt, steps, periods, flag = g.step(1.0)
        assert flag == 0 and steps == 2
        np.testing.assert_array_equal(periods, 1 << e)
    out = g.get_state()
    for k in range(8):
        assert abs(out[k].sum() - U[k].sum()) <= 1e-13 * np.abs(U[k]).sum()


def test_neighbours_differ_by_at_most_one_exponent(port):
    U = states.smooth_3d(SHAPE, np.random.default_rng(4))
    cfg = po.make_cfg(N, po.HLL, L, states.GAMMA_53, 1.0, 0.4)
    g = port.substep_grid(cfg)
    g.set_state(U)
    e = np.zeros(SHAPE, np.int32)
    e[0, 8:, 8:] = 3    # a corner three levels above its surroundings
    g.set_exponents(e, e)
    g.step(0.0)
    dt, steps, periods, flag = g.step(1.0)
    ex = np.log2(periods).astype(int)[0]
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            assert np.all(ex - np.roll(np.roll(ex, dy, 0), dx, 1) <= 1)
    assert ex.max() >= 2 and ex[0, 0] == 0
