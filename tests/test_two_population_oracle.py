"""Pins the two-population oracle (oracle/n_solve.hpp) to the reference (CPU only).

  - the restated split solvers (get_flux_N_rusanov, get_flux_N_hll) equal the reference's headers
    compiled here, bit for bit, on the fixtures of tests/golden/two_population.npz (made by
    tests/golden/make_two_population_golden.py) and live where the reference build exists;
  - the restated scheme of tests/mhd/two_reference.cpp reproduces that program's output bit for
    bit and the reference's golden file tests/mhd/2mhd_rusanov.ref within the program's own bar
    (1e-6 relative, values below 1e-25 ignored, two_reference.cpp:703-760); with HLL it fails
    where the program aborts;
  - the restated N_solve grid driven by the reference's headers equals it on the restated
    solvers bit for bit; it conserves the totals on a periodic grid; with one population it is
    the cell-centred Rusanov step to round-off.
"""
import os

import numpy as np
import pytest

from oracle import pyoracle as po
import states

GOLD = os.path.join(os.path.dirname(__file__), "golden", "two_population.npz")


@pytest.fixture(scope="module")
def fix():
    return np.load(GOLD)


def totals(out):
    return np.column_stack([out[:, 0] + out[:, 5], out[:, 1] + out[:, 6], out[:, 2] + out[:, 7],
                            out[:, 3] + out[:, 8], out[:, 4] + out[:, 9], out[:, 10:13]])


@pytest.mark.parametrize("solver", ["rusanov", "hll_athena"])
def test_split_solvers_match_reference_fixture(port, fix, solver):
    fn, fp, s, g = port.face_flux_N(po.SOLVERS[solver], fix["split_neg"], fix["split_pos"],
                                    float(fix["split_area"]), float(fix["split_dt"]))
    np.testing.assert_array_equal(g, fix[f"split_{solver}_flags"])
    np.testing.assert_array_equal(fn, fix[f"split_{solver}_neg"])
    np.testing.assert_array_equal(fp, fix[f"split_{solver}_pos"])
    np.testing.assert_array_equal(s, fix[f"split_{solver}_speed"])


@pytest.mark.parametrize("solver", ["rusanov", "hll_athena"])
def test_split_solvers_match_live_reference(port, ref, solver):
    rng = np.random.default_rng(5)
    a, b = states.nearby_face_states(4000, rng)
    c = states.random_face_states(4000, rng)
    d = states.random_face_states(4000, rng)
    neg, pos = np.vstack([a, c]), np.vstack([b, d])
    for area, dt in ((1.0, 1.0), (0.3, 2e-3)):
        x = port.face_flux_N(po.SOLVERS[solver], neg, pos, area, dt)
        y = ref.face_flux_N(po.SOLVERS[solver], neg, pos, area, dt)
        for u, v in zip(x, y):
            np.testing.assert_array_equal(u, v)


def test_two_reference_scheme_reproduces_program_and_golden(port, fix):
    out, steps = port.reference_2pop_1d(po.RUSANOV)
    tot = totals(out)
    # the program prints 17 significant digits, which round-trip doubles
    np.testing.assert_array_equal(tot, fix["prog_rusanov"])
    gold = fix["gold_rusanov"]
    big = np.maximum(np.abs(tot), np.abs(gold))
    rel = np.where(big > 1e-25, np.abs(tot - gold) / np.where(big == 0, 1, big), 0.0)
    assert rel.max() <= 1e-6
    assert steps > 900


def test_two_reference_scheme_with_hll_fails_where_the_program_aborts(port, fix):
    assert int(fix["prog_hll_aborts"]) == 1
    with pytest.raises(RuntimeError, match="pressure"):
        port.reference_2pop_1d(po.HLL)


def _grid_run(owner, solver, shape, L, U0, steps, cfl=0.4):
    n = (shape[2], shape[1], shape[0])
    g = owner.two_population_grid(n, L, po.SOLVERS[solver], states.GAMMA_53, 1.0, 0.0)
    g.set_state(U0)
    max_dt, flag, _, _ = g.step(0.0)
    assert flag == 0
    traj = []
    for _ in range(steps):
        max_dt, flag, _, _ = g.step(cfl * max_dt)
        assert flag == 0
        traj.append(g.get_state())
    return np.array(traj)


def test_grid_on_reference_headers_is_bitwise(port, ref):
    shape, L = (4, 5, 6), (0.1, 0.12, 0.09)
    U0 = states.two_population_random(shape, np.random.default_rng(3))
    a = _grid_run(port, "rusanov", shape, L, U0, 4)
    b = _grid_run(ref, "rusanov", shape, L, U0, 4)
    np.testing.assert_array_equal(a, b)


def test_grid_hll_step_on_reference_headers_is_bitwise(port, ref):
    """One HLL step: the reference's split HLL leaves the positive side's field flux unscaled by
    area and dt (mhd/N_hll_athena.hpp:224-227), so the field jumps by a physical flux per step and
    the state soon loses positivity, as the reference's own two-population HLL program does; the
    step itself is compared."""
    shape, L = (4, 5, 6), (0.1, 0.12, 0.09)
    U0 = states.two_population_random(shape, np.random.default_rng(3))
    out = []
    for owner in (port, ref):
        g = owner.two_population_grid((6, 5, 4), L, po.HLL, states.GAMMA_53, 1.0, 0.0)
        g.set_state(U0)
        r = g.step(1e-4)
        out.append((r, g.get_state()))
    assert out[0][0] == out[1][0]
    np.testing.assert_array_equal(out[0][1], out[1][1])


def test_grid_conserves_totals(port):
    shape, L = (4, 5, 6), (0.1, 0.12, 0.09)
    U0 = states.two_population_random(shape, np.random.default_rng(4))
    traj = _grid_run(port, "rusanov", shape, L, U0, 6)
    for k in range(13):
        s0, s1 = U0[k].sum(), traj[-1][k].sum()
        assert abs(s1 - s0) <= 1e-12 * np.abs(U0[k]).sum()


def test_one_population_is_the_cell_centred_step(port):
    """With the second population absent, N_solve's Rusanov (split into its two sides) is the
    cell-centred Rusanov step (the cross-check mhd/N_solve.hpp and mhd/solve.hpp share)."""
    shape, L = (4, 5, 6), (0.1, 0.12, 0.09)
    U = states.smooth_3d(shape, np.random.default_rng(6))
    U13 = np.zeros((13,) + shape)
    U13[0:5], U13[10:13] = U[0:5], U[5:8]
    n = (shape[2], shape[1], shape[0])
    g = port.two_population_grid(n, L, po.RUSANOV, states.GAMMA_53, 1.0, 0.0)
    g.set_state(U13)
    c = port.grid(po.make_cfg(n, po.RUSANOV, L, states.GAMMA_53, 1.0, 0.4))
    c.set_state(U)
    for dt in (1e-3, 2e-3, 1.5e-3):
        g.step(dt)
        assert c.step_dt(dt) == 0
    a, b = g.get_state(), c.get_state()
    got = np.concatenate([a[0:5], a[10:13]])
    for k in range(8):
        assert np.abs(got[k] - b[k]).max() <= 1e-13 * max(np.abs(b[k]).max(), 1e-300)
    assert np.abs(a[5:10]).max() == 0.0
