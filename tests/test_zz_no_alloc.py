"""pamhd_gpu_face_flux_noalloc (scratch in a fixed device array, no allocation) against
pamhd_gpu_face_flux (per-call device buffers): identical fluxes, speeds and flags, bit for bit,
on two calls in a row with different faces, solvers and sizes, so that the second call runs on
scratch the first one left behind.  Collected last so it also runs after every other GPU test."""
import numpy as np
import pytest

import pamhd_b200 as pg
import states

pytestmark = pytest.mark.gpu


def faces(n, rng):
    a, b = states.nearby_face_states(n // 2, rng)
    c = states.random_face_states(n - n // 2, rng)
    d = states.random_face_states(n - n // 2, rng)
    e, f = states.edge_case_face_states()
    return np.vstack([e, a, c])[:n], np.vstack([f, b, d])[:n]


def test_noalloc_matches_face_flux_on_two_calls_in_a_row():
    rng = np.random.default_rng(29)
    calls = [
        (pg.HLLD, pg.NOALLOC_MAX_FACES, None, 1.0),
        (pg.HLL, 5001, "bg", 4e-7 * np.pi),
    ]
    for solver, n, bg_kind, mu0 in calls:
        neg, pos = faces(n, rng)
        if mu0 != 1.0:
            scale = np.ones(8)
            scale[5:8] = np.sqrt(mu0)
            neg, pos = neg * scale, pos * scale
        bg = rng.normal(0, 0.3 * np.sqrt(mu0), (n, 3)) if bg_kind else None
        f0, s0, g0 = pg.face_flux(solver, neg, pos, bg, 5 / 3, mu0)
        f1, s1, g1 = pg.face_flux_noalloc(solver, neg, pos, bg, 5 / 3, mu0)
        assert np.array_equal(g1, g0)
        assert np.array_equal(f1.view(np.uint64), f0.view(np.uint64))
        assert np.array_equal(s1.view(np.uint64), s0.view(np.uint64))
        assert (g0 == 0).sum() > n // 2  # most faces are valid states


def test_noalloc_rejects_oversize_and_accepts_empty():
    neg = np.zeros((pg.NOALLOC_MAX_FACES + 1, 8))
    with pytest.raises(pg.PamhdError) as e:
        pg.face_flux_noalloc(pg.HLLD, neg, neg)
    assert e.value.code == pg.ERR_TOO_LARGE
    f, s, g = pg.face_flux_noalloc(pg.HLLD, neg[:0], neg[:0])
    assert f.shape == (0, 8) and s.shape == (0,) and g.shape == (0,)
