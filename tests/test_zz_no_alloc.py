"""pamhd_gpu_face_flux_noalloc (scratch in a fixed device array, no allocation) against
pamhd_gpu_face_flux (per-call device buffers): identical fluxes, speeds and flags, bit for bit,
on two calls in a row with different faces, solvers and sizes, so that the second call runs on
scratch the first one left behind; every solver; no device memory taken by a call once the
device is set up; the caller's current device left as it was.  Collected last so it also runs
after every other GPU test."""
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
        (pg.RUSANOV, 777, "bg", 1.0),
        (pg.ROE, 3000, None, 1.0),
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


def test_noalloc_takes_no_device_memory():
    import torch
    rng = np.random.default_rng(31)
    neg, pos = faces(4096, rng)
    # set-up: the first call on the device (and the kernels' first launches) may take memory
    for solver in (pg.RUSANOV, pg.HLL, pg.HLLD, pg.ROE):
        pg.face_flux_noalloc(solver, neg, pos)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for solver in (pg.RUSANOV, pg.HLL, pg.HLLD, pg.ROE):
        pg.face_flux_noalloc(solver, neg, pos, rng.normal(0, 0.1, (4096, 3)))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)


def test_noalloc_leaves_the_current_device():
    import torch
    count = torch.cuda.device_count()
    torch.cuda.set_device(0)
    rng = np.random.default_rng(37)
    neg, pos = faces(64, rng)
    # a device that does not exist: the CUDA error, and the current device unchanged
    with pytest.raises(pg.PamhdError) as e:
        pg.face_flux_noalloc(pg.HLLD, neg, pos, device=count)
    assert e.value.code == pg.ERR_CUDA
    assert torch.cuda.current_device() == 0
    if count > 1:
        f, s, g = pg.face_flux_noalloc(pg.HLLD, neg, pos, device=1)
        assert torch.cuda.current_device() == 0
        f0, s0, g0 = pg.face_flux(pg.HLLD, neg, pos)
        assert np.array_equal(f.view(np.uint64), f0.view(np.uint64))


def test_noalloc_rejects_oversize_and_accepts_empty():
    neg = np.zeros((pg.NOALLOC_MAX_FACES + 1, 8))
    with pytest.raises(pg.PamhdError) as e:
        pg.face_flux_noalloc(pg.HLLD, neg, neg)
    assert e.value.code == pg.ERR_TOO_LARGE
    f, s, g = pg.face_flux_noalloc(pg.HLLD, neg[:0], neg[:0])
    assert f.shape == (0, 8) and s.shape == (0,) and g.shape == (0,)
    # arrays of mismatched shapes are refused before the C call
    with pytest.raises(ValueError):
        pg.face_flux_noalloc(pg.HLLD, neg[:10], neg[:9])
    with pytest.raises(ValueError):
        pg.face_flux_noalloc(pg.HLLD, neg[:10], neg[:10], np.zeros((9, 3)))
