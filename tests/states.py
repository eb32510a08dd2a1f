"""Seeded MHD states and grids shared by the tests, the fixture generator and
the benchmark inputs (numpy only)."""
from __future__ import annotations

import functools

import numpy as np

GAMMA_53 = 5.0 / 3.0


def energy(rho, v, p, B, gamma, mu0=1.0):
    """Total energy density from primitives (get_total_energy_density, mhd/common.hpp:258)."""
    return p / (gamma - 1) + 0.5 * rho * (v ** 2).sum(axis=0) + 0.5 / mu0 * (B ** 2).sum(axis=0)


def random_face_states(n, rng, gamma=GAMMA_53, spread=1.0):
    """(n, 8) conservative states: rho in [0.1, 3], |v| ~ N(0, spread), B ~ N(0, 1), p in [0.05, 2]."""
    rho = rng.uniform(0.1, 3.0, n)
    v = rng.normal(0.0, spread, (3, n))
    B = rng.normal(0.0, 1.0, (3, n))
    p = rng.uniform(0.05, 2.0, n)
    s = np.zeros((n, 8))
    s[:, 0] = rho
    s[:, 1:4] = (v * rho).T
    s[:, 4] = energy(rho, v, p, B, gamma)
    s[:, 5:8] = B.T
    return s


def nearby_face_states(n, rng, gamma=GAMMA_53, jump=0.05):
    """Pairs of states that differ by a few percent: the smooth-flow regime of a resolved run."""
    a = random_face_states(n, rng, gamma)
    rho = a[:, 0] * (1 + jump * rng.normal(size=n)).clip(0.5, 1.5)
    v = a[:, 1:4] / a[:, 0:1] + jump * rng.normal(size=(n, 3))
    B = a[:, 5:8] + jump * rng.normal(size=(n, 3))
    p_a = (gamma - 1) * (a[:, 4] - 0.5 * (a[:, 1:4] ** 2).sum(1) / a[:, 0] - 0.5 * (a[:, 5:8] ** 2).sum(1))
    p = p_a * (1 + jump * rng.normal(size=n)).clip(0.5, 1.5)
    b = np.zeros_like(a)
    b[:, 0] = rho
    b[:, 1:4] = v * rho[:, None]
    b[:, 4] = energy(rho, v.T, p, B.T, gamma)
    b[:, 5:8] = B
    return a, b


def edge_case_face_states(gamma=GAMMA_53):
    """Hand-made face problems covering the branches of the four solvers."""
    def st(rho, v, p, B):
        v = np.asarray(v, float)
        B = np.asarray(B, float)
        return np.array([rho, *(rho * v), energy(rho, v[:, None], p, B[:, None], gamma)[0], *B])

    cases = [
        # Brio-Wu interface (gamma 2 in the config; here the library gamma)
        (st(1.0, [0, 0, 0], 1.0, [0.75, 1, 0]), st(0.125, [0, 0, 0], 0.1, [0.75, -1, 0])),
        # identical states
        (st(1.0, [0.3, -0.2, 0.1], 0.5, [0.4, 0.2, -0.1]),) * 2,
        # no field at all: fast speed = sound speed
        (st(1.0, [0.1, 0, 0], 1.0, [0, 0, 0]), st(0.5, [-0.1, 0, 0], 0.4, [0, 0, 0])),
        # zero normal field: HLLD double-star states collapse, Roe sign branch
        (st(1.0, [0.0, 0.5, 0], 1.0, [0, 1, 0.5]), st(0.8, [0.0, -0.5, 0], 0.8, [0, -1, 0.2])),
        # purely normal field
        (st(1.0, [0.2, 0, 0], 1.0, [1.0, 0, 0]), st(0.9, [0.1, 0, 0], 0.9, [1.0, 0, 0])),
        # supersonic to +x and to -x (upwind returns)
        (st(1.0, [20.0, 0.1, 0], 1.0, [0.5, 0.2, 0]), st(0.9, [19.0, 0.0, 0], 0.9, [0.5, 0.1, 0])),
        (st(1.0, [-20.0, 0.1, 0], 1.0, [0.5, 0.2, 0]), st(0.9, [-19.0, 0.0, 0], 0.9, [0.5, 0.1, 0])),
        # strong shear
        (st(1.0, [0.0, 5.0, -3.0], 1.0, [0.3, 2.0, 1.0]), st(1.0, [0.0, -5.0, 3.0], 1.0, [0.3, -2.0, -1.0])),
        # strong rarefaction
        (st(1.0, [-2.0, 0, 0], 1.0, [0.5, 0.5, 0]), st(1.0, [2.0, 0, 0], 1.0, [0.5, 0.5, 0])),
        # tiny pressure, strong field
        (st(1.0, [0.1, 0, 0], 1e-4, [3.0, 4.0, 0]), st(1.0, [0.0, 0, 0], 1e-4, [3.0, 3.5, 0])),
    ]
    neg = np.array([c[0] for c in cases])
    pos = np.array([c[-1] for c in cases])
    # invalid inputs: negative density, negative pressure, NaN momentum
    bad_neg = neg[:3].copy()
    bad_pos = pos[:3].copy()
    bad_neg[0, 0] = -1.0
    bad_pos[1, 4] = 0.5 * (bad_pos[1, 1:4] ** 2).sum() / bad_pos[1, 0] + 0.5 * (bad_pos[1, 5:8] ** 2).sum() - 0.01
    bad_neg[2, 1] = np.nan
    return np.vstack([neg, bad_neg]), np.vstack([pos, bad_pos])


def orszag_tang(n, gamma=GAMMA_53):
    """Orszag-Tang vortex on [0,1]^2 with n x n cells (rho 25/(36 pi), p 5/(12 pi), mu0 = 1).
    Returns (8, 1, n, n)."""
    x = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(x, x, indexing="xy")  # arrays indexed [y, x]
    rho = np.full_like(X, 25.0 / (36.0 * np.pi))
    p = np.full_like(X, 5.0 / (12.0 * np.pi))
    v = np.stack([-np.sin(2 * np.pi * Y), np.sin(2 * np.pi * X), np.zeros_like(X)])
    B = np.stack([-np.sin(2 * np.pi * Y), np.sin(4 * np.pi * X), np.zeros_like(X)]) / np.sqrt(4 * np.pi)
    U = np.zeros((8, 1, n, n))
    U[0, 0] = rho
    U[1:4, 0] = v * rho
    U[4, 0] = energy(rho, v, p, B, gamma)
    U[5:8, 0] = B
    return U


def brio_wu(n=1000, gamma=2.0):
    """Brio-Wu shock tube on [0,1] with n cells; returns (8, 1, 1, n) and the two edge states."""
    x = (np.arange(n) + 0.5) / n
    left = x < 0.5
    rho = np.where(left, 1.0, 0.125)
    p = np.where(left, 1.0, 0.1)
    v = np.zeros((3, n))
    B = np.stack([np.full(n, 0.75), np.where(left, 1.0, -1.0), np.zeros(n)])
    U = np.zeros((8, 1, 1, n))
    U[0, 0, 0] = rho
    U[4, 0, 0] = energy(rho, v, p, B, gamma)
    U[5:8, 0, 0] = B
    return U


def smooth_3d(shape, rng, gamma=GAMMA_53, amp=0.1):
    """Smooth periodic 3-D state (8, nz, ny, nx): a few random Fourier modes on a uniform background."""
    nz, ny, nx = shape
    z, y, x = np.meshgrid(np.arange(nz) / nz, np.arange(ny) / ny, np.arange(nx) / nx, indexing="ij")

    def field(base):
        f = np.full(shape, base, float)
        for _ in range(3):
            k = rng.integers(-2, 3, 3)
            ph = rng.uniform(0, 2 * np.pi)
            f += amp * rng.normal() * np.cos(2 * np.pi * (k[0] * x + k[1] * y + k[2] * z) + ph)
        return f

    rho = field(1.0)
    p = field(0.6)
    v = np.stack([field(0.1), field(-0.05), field(0.02)])
    B = np.stack([field(0.5), field(0.3), field(-0.2)])
    U = np.zeros((8,) + tuple(shape))
    U[0] = rho
    U[1:4] = v * rho
    U[4] = energy(rho, v, p, B, gamma)
    U[5:8] = B
    return U


def blast_wave(n, seed=20261203, gamma=GAMMA_53, amp=0.01, kmax=8):
    """Magnetised blast wave on [-0.5, 0.5]^3 with n^3 cells: rho 1, p 0.1 (10 inside r < 0.1),
    B0 = (1, 1, 0)/sqrt(2) plus a divergence-free perturbation dB = curl A built from 48 random-phase
    modes with integer wavenumbers |k| in [1, kmax] (2 pi units), scaled so rms|dB| = amp |B0|.
    The modes are summed by one inverse FFT per component.  Returns (8, n, n, n) float64."""
    rng = np.random.default_rng(seed)
    c = (np.arange(n) + 0.5) / n - 0.5
    modes = []
    for kx in range(-kmax, kmax + 1):
        for ky in range(-kmax, kmax + 1):
            for kz in range(0, kmax + 1):
                k2 = kx * kx + ky * ky + kz * kz
                if 1 <= k2 <= kmax * kmax and (kz > 0 or ky > 0 or (ky == 0 and kx > 0)):
                    modes.append((kx, ky, kz))
    sel = rng.choice(len(modes), size=min(48, len(modes)), replace=False)
    # dB(x) = sum_m -(k x a) sin(k.x + ph), x = cell centres: written as Im of an inverse DFT over
    # the cell index, with the centre offset folded into each mode's phase
    spec = np.zeros((3, n, n, n), dtype=np.complex128)  # indexed [component, kz, ky, kx]
    for m in sel:
        mv = np.array(modes[m], float)
        k = 2 * np.pi * mv
        a = rng.normal(size=3)
        a -= k * (a @ k) / (k @ k)  # transverse amplitude
        ph = rng.uniform(0, 2 * np.pi)
        ph_cell = ph + 2 * np.pi * (mv @ np.full(3, 0.5 / n - 0.5))
        kxa = np.cross(k, a)
        idx = (int(modes[m][2]) % n, int(modes[m][1]) % n, int(modes[m][0]) % n)
        for d in range(3):
            spec[(d,) + idx] += -kxa[d] * np.exp(1j * ph_cell)
    dB = np.fft.ifftn(spec, axes=(1, 2, 3)).imag * float(n) ** 3
    del spec
    rms = np.sqrt((dB ** 2).sum(0).mean())
    B0 = np.array([1.0, 1.0, 0.0]) / np.sqrt(2.0)
    dB *= amp * np.linalg.norm(B0) / rms
    B = B0[:, None, None, None] + dB
    del dB
    rho = np.ones((n, n, n))
    r2 = c[:, None, None] ** 2 + c[None, :, None] ** 2 + c[None, None, :] ** 2
    p = np.where(r2 < 0.01, 10.0, 0.1)
    U = np.zeros((8, n, n, n))
    U[0] = rho
    U[4] = p / (gamma - 1) + 0.5 * (B ** 2).sum(axis=0)
    U[5:8] = B
    return U


PROTON_MASS = 1.672621777e-27   # simulation_options.hpp:61
MU0_SI = 4e-7 * np.pi            # simulation_options.hpp:60
K_BOLTZMANN = 1.380649e-23
EARTH_RADIUS_CELL = 6.371e5      # cell size of the reference's solar-wind box configs (m)


def solar_wind_ensemble(nboxes=64, seed=20261204, sizes=(32, 48, 64, 96, 128), gamma=GAMMA_53):
    """The batched-ensemble configuration: `nboxes` independent cubes with edge drawn uniformly
    from `sizes`, SI units, each with its own seeded solar wind entering through the -x face:
    n ~ U[1, 20] cm^-3, |v_x| ~ U[300, 800] km/s pointing into the box (+x), |B| ~ U[1, 20] nT
    with an isotropic random direction, T log-uniform on [1e4, 1e6] K, p = n k_B T.  The interior
    starts at rest with a quarter of the wind density, the wind temperature and field.
    Returns a list of dicts: n (edge), inflow (8 conservative values), interior (8 conservative
    values of the uniform initial state; ensemble_state() expands it to (8, n, n, n))."""
    rng = np.random.default_rng(seed)
    boxes = []
    for _ in range(nboxes):
        n = int(rng.choice(sizes))
        dens = rng.uniform(1.0, 20.0) * 1e6
        speed = rng.uniform(300.0, 800.0) * 1e3
        bmag = rng.uniform(1.0, 20.0) * 1e-9
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        T = 10 ** rng.uniform(4.0, 6.0)
        rho = dens * PROTON_MASS
        v = np.array([speed, 0.0, 0.0])
        B = bmag * d
        p = dens * K_BOLTZMANN * T
        inflow = np.array([rho, *(rho * v), energy(rho, v[:, None], p, B[:, None], gamma, MU0_SI)[0], *B])
        rho0 = 0.25 * rho
        p0 = 0.25 * dens * K_BOLTZMANN * T
        interior = np.array([rho0, 0.0, 0.0, 0.0,
                             energy(rho0, np.zeros((3, 1)), p0, B[:, None], gamma, MU0_SI)[0], *B])
        boxes.append({"n": n, "inflow": inflow, "interior": interior})
    return boxes


def ensemble_state(box):
    n = box["n"]
    return np.broadcast_to(box["interior"][:, None, None, None], (8, n, n, n)).copy()


def density_advection(n, gamma, vx, proton_mass=1.0):
    """The reference's density-advection test (tests/mhd/config_files/hydrodynamic/
    density_advection/1d/{+x,-x}/rusanov.json): n periodic cells on [0, 1], number density 1.01
    where |x - 0.5| < 0.25 else 1, velocity (vx, 0, 0), pressure 1, no field; conservative state
    as mhd/initialize.hpp builds it (rho = m_p n, mom = rho v, E = p / (gamma - 1) + rho v^2 / 2).
    Returns (8, 1, 1, n)."""
    x = (np.arange(n) + 0.5) / n
    rho = np.where(np.abs(x - 0.5) < 0.25, 1.01, 1.0) * proton_mass
    U = np.zeros((8, 1, 1, n))
    U[0, 0, 0] = rho
    U[1, 0, 0] = rho * vx
    U[4, 0, 0] = 1.0 / (gamma - 1) + 0.5 * rho * vx * vx
    return U


@functools.lru_cache(maxsize=None)
def gauss_legendre_7():
    """Nodes (x >= 0, ascending) and weights of the 7-point Gauss-Legendre rule on [-1, 1], each
    the double nearest to the exact value: Newton iteration on the Legendre polynomial P7 in
    60-digit decimal arithmetic from the Chebyshev-like first guesses cos(pi (i - 1/4) / (7 + 1/2)),
    weights 2 / ((1 - x^2) P7'(x)^2)."""
    import decimal
    import math

    ctx = decimal.Context(prec=60)
    D = decimal.Decimal

    def legendre(x):
        p0, p1 = D(1), x
        for k in range(2, 8):
            p0, p1 = p1, ctx.divide(ctx.subtract(ctx.multiply(D(2 * k - 1) * x, p1), D(k - 1) * p0), D(k))
        # derivative: n (x P_n - P_{n-1}) / (x^2 - 1)
        dp = ctx.divide(D(7) * (x * p1 - p0), x * x - 1)
        return p1, dp

    nodes, weights = [], []
    for i in range(1, 5):
        x = D(repr(math.cos(math.pi * (i - 0.25) / 7.5)))
        for _ in range(100):
            p, dp = legendre(x)
            step = ctx.divide(p, dp)
            x = ctx.subtract(x, step)
            if abs(step) < D(10) ** -55:
                break
        if abs(x) < D(10) ** -50:
            x = D(0)
        _, dp = legendre(x)
        w = ctx.divide(D(2), (1 - x * x) * dp * dp)
        nodes.append(float(x))
        weights.append(float(w))
    order = np.argsort(nodes)
    return [nodes[i] for i in order], [weights[i] for i in order]


def gauss_average(f, a, b):
    """Integral of f over [a, b] by the 7-point Gauss-Legendre rule, in the summation order of
    boost::math::quadrature::gauss<double, 7>::integrate (the rule mhd/initialize.hpp:361-486
    uses): scale * (f(mid) w0 + sum_i (f(mid + scale x_i) + f(mid - scale x_i)) w_i)."""
    x, w = gauss_legendre_7()
    mid = (a + b) * 0.5
    scale = (b - a) * 0.5
    total = f(mid + scale * x[0]) * w[0]
    for i in range(1, 4):
        fp = f(mid + scale * x[i])
        fm = f(mid + scale * -x[i])
        total += (fp + fm) * w[i]
    return scale * total


def staggered_state(n, length, start, number_density, velocity, pressure, field, gamma, mu0,
                    proton_mass=1.0, background=None):
    """Initial cell state and face field of the reference's MHD program (tests/mhd/test.cpp:422-456)
    on a uniform periodic grid: the normal field of every face is its 7-point Gauss-Legendre
    average over the face (initialize_magnetic_field, mhd/initialize.hpp:361-547), in a dimension
    of one cell taken at the grid's middle (get_cell_geom_emulated, grid/amr.hpp:288-310); the
    volume field is the mean of each cell's two faces (update_vol_B); the fluid is set at the
    cell centres (initialize_fluid, mhd/initialize.hpp:77-160: rho = m_p n, mom = rho v, E from
    the pressure, v and the volume field).  The functions take (x, y, z) scalars and return a
    scalar (number density, pressure) or a 3-sequence (velocity, field, background).
    Returns U (8, nz, ny, nx) and faces (3, nz, ny, nx): the field of each cell's -x, -y, -z face;
    with a background field function also bg (3, 3, nz, ny, nx): every component of the
    background field averaged over each cell's -d face the same way (mhd/initialize.hpp:517-530)."""
    n = [int(v) for v in n]
    L = [float(v) for v in length]
    s = [float(v) for v in start]
    mid = [(s[d] + n[d] * L[d] + s[d]) / 2 for d in range(3)]

    def bounds(d, i):
        if n[d] == 1:
            return mid[d], mid[d], mid[d]
        lo = s[d] + i * L[d]
        hi = s[d] + (i + 1) * L[d]
        return lo + L[d] / 2, lo, hi

    faces = np.zeros((3, n[2], n[1], n[0]))
    bg = None if background is None else np.zeros((3, 3, n[2], n[1], n[0]))
    U = np.zeros((8, n[2], n[1], n[0]))

    def face_average(func, comp, d, geo):
        # integrate_face_B of mhd/initialize.hpp:361-486 for the cell's -d face
        a, b = [e for e in range(3) if e != d]   # the two dimensions across the face

        def point(u, v):
            c = [0.0, 0.0, 0.0]
            c[d] = geo[d][1]
            c[a] = u
            c[b] = v
            return func(*c)[comp]

        ua, ea = geo[a][1], geo[a][2]
        ub, eb = geo[b][1], geo[b][2]
        wa, wb = ea - ua, eb - ub
        if wa == 0 and wb == 0:
            return point(ua, ub)
        if wa == 0:
            return gauss_average(lambda v: point(ua, v), ub, eb) / wb
        if wb == 0:
            return gauss_average(lambda u: point(u, ub), ua, ea) / wa
        return gauss_average(lambda v: gauss_average(lambda u: point(u, v), ua, ea), ub, eb) / wa / wb

    for k in range(n[2]):
        for j in range(n[1]):
            for i in range(n[0]):
                geo = [bounds(0, i), bounds(1, j), bounds(2, k)]
                for d in range(3):
                    faces[d, k, j, i] = face_average(field, d, d, geo)
                    if bg is not None:
                        for comp in range(3):
                            bg[d, comp, k, j, i] = face_average(background, comp, d, geo)
    for k in range(n[2]):
        for j in range(n[1]):
            for i in range(n[0]):
                c = [bounds(0, i)[0], bounds(1, j)[0], bounds(2, k)[0]]
                B = [0.5 * (faces[0, k, j, i] + faces[0, k, j, (i + 1) % n[0]]),
                     0.5 * (faces[1, k, j, i] + faces[1, k, (j + 1) % n[1], i]),
                     0.5 * (faces[2, k, j, i] + faces[2, (k + 1) % n[2], j, i])]
                rho = proton_mass * number_density(*c)
                v = velocity(*c)
                p = pressure(*c)
                U[0, k, j, i] = rho
                for e in range(3):
                    U[1 + e, k, j, i] = rho * v[e]
                    U[5 + e, k, j, i] = B[e]
                if rho > 0 and p > 0:
                    kinetic = 0.5 * rho * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
                    magnetic = 0.5 / mu0 * (B[0] * B[0] + B[1] * B[1] + B[2] * B[2])
                    U[4, k, j, i] = p / (gamma - 1) + kinetic + magnetic
    if bg is not None:
        return U, faces, bg
    return U, faces


def alfven_1d(n=100, sign=1):
    """The reference's 1-D Alfven wave (tests/mhd/config_files/magnetohydrodynamic/Alfven_wave/1d/
    {+x,-x}/small_rusanov.json): n x 1 x 1 periodic cells on [0, 1]^3, gamma 5/3, mu0 1, number
    density 1, pressure 0.1, v = sign (0, 0.1 sin 2 pi x, 0.1 cos 2 pi x),
    B = (1, 0.1 sin 2 pi x, 0.1 cos 2 pi x).  Returns U, faces, cell lengths."""
    import math
    tau = 2 * math.pi
    gamma = 1.6666666666666667

    def vel(x, y, z):
        return (0.0, sign * (0.1 * math.sin(tau * x)), sign * (0.1 * math.cos(tau * x)))

    def mag(x, y, z):
        return (1.0, 0.1 * math.sin(tau * x), 0.1 * math.cos(tau * x))

    L = (1.0 / n, 1.0, 1.0)
    U, faces = staggered_state((n, 1, 1), L, (0, 0, 0), lambda x, y, z: 1.0, vel, lambda x, y, z: 0.1,
                               mag, gamma, 1.0)
    return U, faces, L


def alfven_2d(standing=False, background=False):
    """The reference's 2-D Alfven wave on 1 x 10 x 10 level-0 cells (tests/mhd/config_files/
    magnetohydrodynamic/Alfven_wave/2d/x/small_rusanov1.json, travelling; small_rusanov2.json,
    standing): periodic, volume (1, 2/sqrt 3, 2), gamma 5/3, mu0 1, number density 1, pressure
    0.1, with phase = pi (sqrt 3 y + z):
    v = (sin(phase)/1000, -cos(phase)/2000, sqrt 3 cos(phase)/2000), or for the standing wave
    (sin(phase)/1000, sqrt 3/2 - cos(phase)/2000, 0.5 + sqrt 3 cos(phase)/2000);
    B = (sin(phase)/1000, sqrt 3/2 + cos(phase)/2000, 0.5 - sqrt 3 cos(phase)/2000).
    With background=True (small_rusanov_bgB{1,2}.json): B = (sin(phase)/1000, cos(phase)/2000,
    -sqrt 3 cos(phase)/2000) on the constant background field (0, 0.86603, 0.5).
    Returns U, faces, cell lengths (and the background field per face, (3, 3, 10, 10, 1))."""
    import math
    r3 = math.sqrt(3)
    gamma = 1.6666666666666667

    def phase(y, z):
        return math.pi * (r3 * y + z)

    def vel(x, y, z):
        s, c = math.sin(phase(y, z)), math.cos(phase(y, z))
        if standing:
            return (s / 1000, r3 / 2 - c / 2000, 0.5 + r3 * c / 2000)
        return (s / 1000, -c / 2000, r3 * c / 2000)

    def mag(x, y, z):
        s, c = math.sin(phase(y, z)), math.cos(phase(y, z))
        if background:
            return (s / 1000, c / 2000, -r3 * c / 2000)
        return (s / 1000, r3 / 2 + c / 2000, 0.5 - r3 * c / 2000)

    L = (1.0, 2 / r3 / 10, 0.2)
    out = staggered_state((1, 10, 10), L, (0, 0, 0), lambda x, y, z: 1.0, vel, lambda x, y, z: 0.1,
                          mag, gamma, 1.0, background=(lambda x, y, z: (0.0, 0.86603, 0.5)) if background else None)
    if background:
        U, faces, bg = out
        return U, faces, L, bg
    U, faces = out
    return U, faces, L


def face_divergence(faces, L):
    """Discrete divergence of a face field (3, nz, ny, nx) on a periodic grid, per cell."""
    r = lambda a, ax: np.roll(a, -1, axis=ax)
    return ((r(faces[0], 2) - faces[0]) / L[0] + (r(faces[1], 1) - faces[1]) / L[1]
            + (r(faces[2], 0) - faces[2]) / L[2])


def staggered_random(shape, L, rng, amp=0.05, field_amp=0.01, mean_field=(0.3, -0.2, 0.1), gamma=GAMMA_53):
    """A smooth random cell state with a face field of zero discrete divergence: a uniform field
    plus the discrete curl of a random periodic vector potential on the cell edges.  The volume
    field is the mean of each cell's two faces, the total energy recomputed with it at the
    state's pressure.  Returns U (8, nz, ny, nx), faces (3, nz, ny, nx), L."""
    A = rng.normal(size=(3,) + tuple(shape)) * field_amp
    dx, dy, dz = L
    r = lambda a, ax: np.roll(a, -1, axis=ax)
    bx = (r(A[2], 1) - A[2]) / dy - (r(A[1], 0) - A[1]) / dz
    by = (r(A[0], 0) - A[0]) / dz - (r(A[2], 2) - A[2]) / dx
    bz = (r(A[1], 2) - A[1]) / dx - (r(A[0], 1) - A[0]) / dy
    faces = np.stack([bx, by, bz]) + np.asarray(mean_field, dtype=float)[:, None, None, None]
    U = smooth_3d(tuple(shape), rng, gamma=gamma, amp=amp)
    rho = U[0]
    v = U[1:4] / rho
    p = (U[4] - 0.5 * rho * (v ** 2).sum(axis=0) - 0.5 * (U[5:8] ** 2).sum(axis=0)) * (gamma - 1)
    U[5] = 0.5 * (faces[0] + r(faces[0], 2))
    U[6] = 0.5 * (faces[1] + r(faces[1], 1))
    U[7] = 0.5 * (faces[2] + r(faces[2], 0))
    U[4] = energy(rho, v, p, U[5:8], gamma)
    return U, faces, L


def two_population_random(shape, rng, gamma=GAMMA_53, mu0=1.0, amp=0.1):
    """Two fluid populations sharing one field, smooth and periodic: (13, nz, ny, nx) with rho1,
    mom1 xyz, E1, rho2, mom2 xyz, E2, B xyz.  Each population's energy holds its own thermal and
    kinetic energy plus its mass fraction's share of the field energy, so that the total state has
    the total pressure of both."""
    a = smooth_3d(tuple(shape), rng, gamma=gamma, amp=amp)
    b = smooth_3d(tuple(shape), rng, gamma=gamma, amp=amp)
    B = a[5:8]
    rho1, rho2 = a[0], 0.5 * b[0]
    v1, v2 = a[1:4] / a[0], b[1:4] / b[0] + np.array([0.05, -0.02, 0.01])[:, None, None, None]
    p1 = (a[4] - 0.5 * a[0] * (v1 ** 2).sum(axis=0) - 0.5 / mu0 * (B ** 2).sum(axis=0)) * (gamma - 1)
    p2 = 0.5 * p1
    f1, f2 = rho1 / (rho1 + rho2), rho2 / (rho1 + rho2)
    pb = 0.5 / mu0 * (B ** 2).sum(axis=0)
    U = np.zeros((13,) + tuple(shape))
    U[0], U[1:4], U[4] = rho1, rho1 * v1, p1 / (gamma - 1) + 0.5 * rho1 * (v1 ** 2).sum(axis=0) + f1 * pb
    U[5], U[6:9], U[9] = rho2, rho2 * v2, p2 / (gamma - 1) + 0.5 * rho2 * (v2 ** 2).sum(axis=0) + f2 * pb
    U[10:13] = B
    return U
