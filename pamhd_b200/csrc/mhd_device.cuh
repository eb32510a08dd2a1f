/*
FP64 device physics of the finite-volume MHD step (sm_100a).

The four Riemann solvers of the reference (mhd/rusanov.hpp:67,
mhd/hll_athena.hpp:65, mhd/hlld_athena.hpp:62, mhd/roe_athena.hpp:575) and
the MHD primitives they use (mhd/common.hpp), written for the GPU:

  - Each cell's derived quantities (1/rho, velocity, thermal pressure,
    magnetic pressure and the fast magnetosonic speed along each axis) are
    computed once per cell and shared by the six faces of the cell.  The
    reference recomputes them in every solver call.
  - Divisions by the same denominator are done once as a reciprocal, and
    the compiler contracts a*b+c into FMA.  Results therefore differ from
    the reference by round-off (the parity tests hold them to 1e-12).
  - Branches (supersonic upwinding, HLLD degeneracy thresholds, region
    selection, Roe's positivity check) are the reference's, with its
    epsilon thresholds.
  - Where the reference throws std::domain_error, the device code raises a
    PAMHD_FLAG_* bit for that face instead (include/pamhd_gpu.h).

Conventions: a face is solved in its own frame, x = face normal; Side holds
one cell's state rotated into that frame (get_rotated_vector,
mhd/common.hpp:612).  Flux order: rho, mom x/y/z, E, B x/y/z.
*/
#ifndef PAMHD_B200_MHD_DEVICE_CUH
#define PAMHD_B200_MHD_DEVICE_CUH

#include <cstdint>

#include "../../include/pamhd_gpu.h"

namespace pamhd_b200 {

constexpr double DBL_EPS = 2.220446049250313080847e-16;  // numeric_limits<double>::epsilon()
constexpr double DBL_MIN_NORMAL = 2.2250738585072013831e-308;

__device__ __forceinline__ bool is_normal(const double x)
{
	const double a = fabs(x);
	return a >= DBL_MIN_NORMAL and a <= 1.7976931348623157e308;
}

__device__ __forceinline__ bool is_finite(const double x)
{
	return fabs(x) <= 1.7976931348623157e308;
}

// physical constants of one run
struct Gas {
	double gamma;     // adiabatic index
	double mu0;       // vacuum permeability
	double inv_mu0;   // 1 / mu0
	double sqrt_mu0;
	double inv_sqrt_mu0;
};

/*
Derived quantities of one cell (mhd/common.hpp:79 get_pressure,
:327 get_sound_speed, :381 get_alfven_speed, :418
get_fast_magnetosonic_speed), computed once per cell.  cf[d] is the fast
magnetosonic speed along axis d.  bad holds the PAMHD_FLAG_* bits the
reference would raise for any face touching this cell, in its order of
checks: density, then pressure, then wave speed.
*/
struct Derived {
	double rinv, vx, vy, vz, p, cf[3];
	uint32_t bad;
};

/*
Reciprocal of a non-zero normal double by Newton-Raphson iteration
(r <- r + r (1 - x r), quadratic convergence) from the hardware estimate of
PTX rcp.approx.ftz.f64; two iterations bring the estimate's relative error
below 2^-52, so the result is within one unit in the last place of 1/x.
Used where the operand is a normal, non-zero number by construction.
*/
__device__ __forceinline__ double recip(const double x)
{
	double r;
	asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
	double e = __fma_rn(-x, r, 1.0);
	r = __fma_rn(r, e, r);
	e = __fma_rn(-x, r, 1.0);
	return __fma_rn(r, e, r);
}

/*
Reciprocal square root of a positive normal double: Newton-Raphson
iteration for f(r) = 1/r^2 - x, r <- r + (r/2)(1 - x r^2) (quadratic
convergence), from the hardware estimate of PTX rsqrt.approx.ftz.f64; two
iterations.  sqrt(x) is then x * rsqrt(x), within a few units in the last
place, which the 1e-12 parity bar leaves ample room for.
*/
__device__ __forceinline__ double rsqrt_nr(const double x)
{
	double r;
	asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
	double e = __fma_rn(__dmul_rn(-x, r), r, 1.0);
	r = __fma_rn(__dmul_rn(0.5, r), e, r);
	e = __fma_rn(__dmul_rn(-x, r), r, 1.0);
	return __fma_rn(__dmul_rn(0.5, r), e, r);
}

/*
Square root of a non-negative double as x * rsqrt_nr(x) (0, +inf and NaN
pass through as themselves).
*/
__device__ __forceinline__ double sqrt_nr(const double x)
{
	return (x > 0.0 and x <= 1.7976931348623157e308) ? __dmul_rn(x, rsqrt_nr(x)) : x;
}


/*
Every operation below is an explicitly rounded intrinsic, so that every
inlined copy of this function computes the same bits for the same cell
(the halo of one tile is the interior of the next).
*/
template <bool NEED_X, bool NEED_Y, bool NEED_Z, bool NR_SQRT = false>
__device__ __forceinline__ Derived derive(
	const double rho, const double mx, const double my, const double mz,
	const double E, const double bx, const double by, const double bz, const Gas& g
) {
	Derived d;
	d.rinv = recip(rho);
	d.vx = __dmul_rn(mx, d.rinv);
	d.vy = __dmul_rn(my, d.rinv);
	d.vz = __dmul_rn(mz, d.rinv);
	const double b2 = __fma_rn(bz, bz, __fma_rn(by, by, __dmul_rn(bx, bx)));
	const double m2 = __fma_rn(mz, mz, __fma_rn(my, my, __dmul_rn(mx, mx)));
	const double kinetic = __dmul_rn(__dmul_rn(0.5, d.rinv), m2);
	const double magnetic = __dmul_rn(__dmul_rn(0.5, g.inv_mu0), b2);
	d.p = __dmul_rn(__dsub_rn(__dsub_rn(E, kinetic), magnetic), g.gamma - 1.0);
	d.bad = 0;
	if (not (rho > 0.0 and is_normal(rho))) {
		d.bad = PAMHD_FLAG_DENSITY;
	} else if (not (d.p > 0.0 and is_normal(d.p))) {
		d.bad = PAMHD_FLAG_PRESSURE;
	}
	const double cs2 = __dmul_rn(__dmul_rn(g.gamma, d.p), d.rinv);
	if (b2 > 0.0) {
		const double va2 = __dmul_rn(__dmul_rn(b2, g.inv_mu0), d.rinv);
		const double sum2 = __dadd_rn(cs2, va2);
		const double inv_b2 = recip(b2);
		const double prod = __dmul_rn(__dmul_rn(2.0, cs2), va2);
		const double base = __fma_rn(va2, va2, __dmul_rn(cs2, cs2));
		const double comp[3] = {bx, by, bz};
		const bool need[3] = {NEED_X, NEED_Y, NEED_Z};
		bool wave_ok = is_normal(sum2) and is_finite(b2);
		#pragma unroll
		for (int a = 0; a < 3; a++) {
			if (not need[a]) {
				d.cf[a] = 0.0;
				continue;
			}
			const double cos2 = __dmul_rn(__dmul_rn(comp[a], comp[a]), inv_b2);
			const double to_sqrt = __fma_rn(prod, __fma_rn(-2.0, cos2, 1.0), base);
			wave_ok = wave_ok and to_sqrt > 0.0 and is_normal(to_sqrt);
			d.cf[a] = NR_SQRT
				? sqrt_nr(__dmul_rn(0.5, __dadd_rn(sum2, sqrt_nr(fmax(to_sqrt, 0.0)))))
				: __dsqrt_rn(__dmul_rn(0.5, __dadd_rn(sum2, __dsqrt_rn(fmax(to_sqrt, 0.0)))));
		}
		if (d.bad == 0 and not wave_ok) d.bad = PAMHD_FLAG_WAVE_SPEED;
	} else {
		const double cs = NR_SQRT ? sqrt_nr(fmax(cs2, 0.0)) : __dsqrt_rn(fmax(cs2, 0.0));
		d.cf[0] = d.cf[1] = d.cf[2] = cs;
		if (d.bad == 0 and not is_finite(b2)) d.bad = PAMHD_FLAG_WAVE_SPEED;
	}
	return d;
}

// one cell seen from a face, rotated into the face frame
struct Side {
	double rho, m0, m1, m2, E, b0, b1, b2;
	double rinv, v0, v1, v2, p, cf;
	uint32_t bad;
};

/*
Rotation into the frame of a face normal to axis `axis` (0, 1, 2):
get_rotated_vector(v, axis + 1), mhd/common.hpp:612-648:
  x: (v0, v1, v2)   y: (v1, v2, v0)   z: (v2, v0, v1)
*/
template <int AXIS>
__device__ __forceinline__ void rotate(const double a, const double b, const double c,
                                       double& r0, double& r1, double& r2)
{
	if (AXIS == 0) { r0 = a; r1 = b; r2 = c; }
	if (AXIS == 1) { r0 = b; r1 = c; r2 = a; }
	if (AXIS == 2) { r0 = c; r1 = a; r2 = b; }
}

// and back: get_rotated_vector(r, -(axis + 1))
template <int AXIS>
__device__ __forceinline__ void unrotate(const double r0, const double r1, const double r2,
                                         double& a, double& b, double& c)
{
	if (AXIS == 0) { a = r0; b = r1; c = r2; }
	if (AXIS == 1) { a = r2; b = r0; c = r1; }
	if (AXIS == 2) { a = r1; b = r2; c = r0; }
}

// a cell's state (8 values, xyz frame) and derived quantities seen from a face normal to axis A
template <int A>
__device__ __forceinline__ Side side_of(const double U[8], const Derived& d)
{
	Side s;
	s.rho = U[0];
	rotate<A>(U[1], U[2], U[3], s.m0, s.m1, s.m2);
	s.E = U[4];
	rotate<A>(U[5], U[6], U[7], s.b0, s.b1, s.b2);
	s.rinv = d.rinv;
	s.p = d.p;
	s.cf = d.cf[A];
	s.v0 = s.m0 * s.rinv;
	s.v1 = s.m1 * s.rinv;
	s.v2 = s.m2 * s.rinv;
	s.bad = d.bad;
	return s;
}

/*
Arithmetic of the face solvers (Rusanov, HLL, HLLD).  Ar<false>: plain expressions, as written
(the files built with -fmad=false round every operation on its own).
Ar<true>: every operation an explicitly rounded intrinsic, a fused
multiply-add where the formula has a product added, so that every kernel
of the cell-centred step (single grid, batched, persistent) computes the
same bits for the same face, whatever other code it is inlined beside.
In both, fma(a, b, c) is a b + c and x - y z is written fma(-y, z, x),
which negates exactly, so Ar<false> keeps the written operation order.
*/
template <bool X> struct Ar {
	static __device__ __forceinline__ double mul(const double a, const double b) { return X ? __dmul_rn(a, b) : a * b; }
	static __device__ __forceinline__ double add(const double a, const double b) { return X ? __dadd_rn(a, b) : a + b; }
	static __device__ __forceinline__ double sub(const double a, const double b) { return X ? __dsub_rn(a, b) : a - b; }
	static __device__ __forceinline__ double fma(const double a, const double b, const double c)
	{
		return X ? __fma_rn(a, b, c) : a * b + c;
	}
};

/*
Ideal-MHD flux along the face normal, mhd/common.hpp:146-244, with the
background field zero (every configuration of the fused step).  pb is the
magnetic pressure B^2 / (2 mu0).
*/
template <bool X = false>
__device__ __forceinline__ void physical_flux(const Side& s, const double pb, const Gas& g, double F[8])
{
	if constexpr (X) {
		using A = Ar<true>;
		F[0] = s.m0;
		F[1] = A::add(A::fma(s.m0, s.v0, -A::mul(g.inv_mu0, A::mul(s.b0, s.b0))), A::add(s.p, pb));
		F[2] = A::fma(s.m1, s.v0, -A::mul(g.inv_mu0, A::mul(s.b0, s.b1)));
		F[3] = A::fma(s.m2, s.v0, -A::mul(g.inv_mu0, A::mul(s.b0, s.b2)));
		const double vb = A::fma(s.v2, s.b2, A::fma(s.v1, s.b1, A::mul(s.v0, s.b0)));
		F[4] = A::fma(s.v0, A::add(A::add(s.E, s.p), pb), -A::mul(A::mul(s.b0, vb), g.inv_mu0));
		F[5] = 0.0;
		F[6] = A::fma(s.v0, s.b1, -A::mul(s.b0, s.v1));
		F[7] = A::fma(s.v0, s.b2, -A::mul(s.b0, s.v2));
		return;
	}
	F[0] = s.m0;
	F[1] = s.m0 * s.v0 - g.inv_mu0 * (s.b0 * s.b0) + (s.p + pb);
	F[2] = s.m1 * s.v0 - g.inv_mu0 * (s.b0 * s.b1);
	F[3] = s.m2 * s.v0 - g.inv_mu0 * (s.b0 * s.b2);
	const double vb = s.v0 * s.b0 + s.v1 * s.b1 + s.v2 * s.b2;
	F[4] = s.v0 * (s.E + s.p + pb) - s.b0 * vb * g.inv_mu0;
	F[5] = 0.0;
	F[6] = s.v0 * s.b1 - s.b0 * s.v1;
	F[7] = s.v0 * s.b2 - s.b0 * s.v2;
}

/*
The same with a background face field bg (in the face frame), for the
solver-level entry point: mhd/common.hpp:174-241 splits the field into the
cell's own part B and the background part.
*/
__device__ __forceinline__ void physical_flux_bg(
	const Side& s, const double bg0, const double bg1, const double bg2, const Gas& g, double F[8]
) {
	const double t0 = s.b0 + bg0, t1 = s.b1 + bg1, t2 = s.b2 + bg2;
	const double p_bg = 0.5 * g.inv_mu0 * (bg0 * bg0 + bg1 * bg1 + bg2 * bg2);
	const double p_b1 = 0.5 * g.inv_mu0 * (s.b0 * s.b0 + s.b1 * s.b1 + s.b2 * s.b2);
	const double p_tot = 0.5 * g.inv_mu0 * (t0 * t0 + t1 * t1 + t2 * t2);
	F[0] = s.m0;
	F[1] = s.m0 * s.v0 - g.inv_mu0 * (t0 * t0 - bg0 * bg0) + (s.p + p_tot - p_bg);
	F[2] = s.m1 * s.v0 - g.inv_mu0 * (t0 * t1 - bg0 * bg1);
	F[3] = s.m2 * s.v0 - g.inv_mu0 * (t0 * t2 - bg0 * bg2);
	const double vb = s.v0 * s.b0 + s.v1 * s.b1 + s.v2 * s.b2;
	F[4] = s.v0 * (s.E + s.p + p_b1) - s.b0 * vb * g.inv_mu0
		+ g.inv_mu0 * (s.b1 * (s.v0 * bg1 - s.v1 * bg0) + s.b2 * (s.v0 * bg2 - s.v2 * bg0));
	F[5] = 0.0;
	F[6] = s.v0 * t1 - t0 * s.v1;
	F[7] = s.v0 * t2 - t0 * s.v2;
}

template <bool X = false>
__device__ __forceinline__ double magnetic_pressure(const Side& s, const Gas& g)
{
	if constexpr (X) {
		using A = Ar<true>;
		return A::mul(A::mul(0.5, g.inv_mu0), A::fma(s.b2, s.b2, A::fma(s.b1, s.b1, A::mul(s.b0, s.b0))));
	}
	return 0.5 * g.inv_mu0 * (s.b0 * s.b0 + s.b1 * s.b1 + s.b2 * s.b2);
}

/*
Rusanov (local Lax-Friedrichs), mhd/rusanov.hpp:67-179:
F = (F_L + F_R)/2 - s/2 (U_R - U_L), s = max(|u_L|, |u_R|) + max(c_f,L, c_f,R).
The field's normal component is diffused like the rest (the reference
does not zero it).
*/
template <bool BG, bool EX = false>
__device__ __forceinline__ double flux_rusanov(const Side& L, const Side& R, const Gas& g, double F[8],
                                               uint32_t& flag, const double* bg = nullptr)
{
	using A = Ar<EX and not BG>;
	const double fast = fmax(L.cf, R.cf);
	const double s = A::add(fmax(fabs(L.v0), fabs(R.v0)), fast);
	double FL[8], FR[8];
	if (BG) {
		physical_flux_bg(L, bg[0], bg[1], bg[2], g, FL);
		physical_flux_bg(R, bg[0], bg[1], bg[2], g, FR);
	} else {
		physical_flux<EX>(L, magnetic_pressure<EX>(L, g), g, FL);
		physical_flux<EX>(R, magnetic_pressure<EX>(R, g), g, FR);
	}
	const double h = A::mul(0.5, s);
	const double UL[8] = {L.rho, L.m0, L.m1, L.m2, L.E, L.b0, L.b1, L.b2};
	const double UR[8] = {R.rho, R.m0, R.m1, R.m2, R.E, R.b0, R.b1, R.b2};
	#pragma unroll
	for (int v = 0; v < 8; v++) {
		F[v] = A::fma(-A::sub(UR[v], UL[v]), h, A::mul(0.5, A::add(FL[v], FR[v])));
	}
	if (flag == 0 and (not is_finite(F[0]) or not is_finite(s))) flag = PAMHD_FLAG_FLUX;
	return s;
}

/*
HLL with Davis wave-speed estimates, mhd/hll_athena.hpp:65-275:
S_L = min(u_L, u_R) - max c_f, S_R = max(u_L, u_R) + max c_f,
bm = min(S_L, 0), bp = max(S_R, 0); a degenerate fan (bp - bm not a
positive normal number) gives zero flux and zero speed.
*/
template <bool BG, bool EX = false>
__device__ __forceinline__ double flux_hll(const Side& L, const Side& R, const Gas& g, double F[8],
                                           uint32_t& /*flag*/, const double* bg = nullptr)
{
	using A = Ar<EX and not BG>;
	const double fast = fmax(L.cf, R.cf);
	const bool order = L.v0 <= R.v0;
	const double s_neg = A::sub(order ? L.v0 : R.v0, fast);
	const double s_pos = A::add(order ? R.v0 : L.v0, fast);
	const double bm = fmin(s_neg, 0.0), bp = fmax(s_pos, 0.0);
	const double width = A::sub(bp, bm);
	if (not (is_normal(width) and width > 0.0)) {
		#pragma unroll
		for (int v = 0; v < 8; v++) F[v] = 0.0;
		return 0.0;
	}
	double FL[8], FR[8];
	if (BG) {
		physical_flux_bg(L, bg[0], bg[1], bg[2], g, FL);
		physical_flux_bg(R, bg[0], bg[1], bg[2], g, FR);
	} else {
		physical_flux<EX>(L, magnetic_pressure<EX>(L, g), g, FL);
		physical_flux<EX>(R, magnetic_pressure<EX>(R, g), g, FR);
	}
	const double UL[8] = {L.rho, L.m0, L.m1, L.m2, L.E, L.b0, L.b1, L.b2};
	const double UR[8] = {R.rho, R.m0, R.m1, R.m2, R.E, R.b0, R.b1, R.b2};
	const double w = A::mul(A::mul(0.5, A::add(bp, bm)), recip(width));
	#pragma unroll
	for (int v = 0; v < 8; v++) {
		const double a = (v == 5) ? 0.0 : A::fma(-bm, UL[v], FL[v]);
		const double b = (v == 5) ? 0.0 : A::fma(-bp, UR[v], FR[v]);
		F[v] = A::fma(A::sub(a, b), w, A::mul(0.5, A::add(a, b)));
	}
	return fmax(fabs(bp), fabs(bm));
}

// transverse velocity and field of one side's star state (Miyoshi & Kusano eqns 44-47); the
// degeneracy test is a select, so the function is one basic block
struct Star_T {
	double w1, w2, b1, b2;
};

template <bool EX>
__device__ __forceinline__ Star_T star_transverse(const Side& X, const double rho_sd, const double sd,
                                                  const double sm, const double s_mid, const double bx,
                                                  const double bx2_mu, const double thr, const Gas& g)
{
	using A = Ar<EX>;
	const double tmp = A::fma(rho_sd, sm, -bx2_mu);
	const double it = recip(tmp);
	const bool keep = fabs(tmp) < thr;
	const double t1 = A::mul(A::mul(A::mul(bx, A::sub(s_mid, X.v0)), g.inv_mu0), it);
	const double t2 = A::mul(A::fma(rho_sd, sd, -bx2_mu), it);
	Star_T t;
	t.w1 = keep ? X.v1 : A::fma(-X.b1, t1, X.v1);
	t.w2 = keep ? X.v2 : A::fma(-X.b2, t1, X.v2);
	t.b1 = keep ? X.b1 : A::mul(X.b1, t2);
	t.b2 = keep ? X.b2 : A::mul(X.b2, t2);
	return t;
}

/*
HLLD of Miyoshi & Kusano (J. Comput. Phys. 208, 2005), as
mhd/hlld_athena.hpp:62-559; the background field is ignored there (:77)
and here.  Past the supersonic cases every region's ingredients are
computed in one straight run (both sides' transverse star states, the
double-star state) and the reference's region choice (:475-552) selects
among them, so that the compiler can overlap the two sides' dependency
chains; values of regions not taken are discarded by selects, never
multiplied in.
The side the flux is taken from comes from pick(left): a caller that holds
the sides' records in shared memory reads that side again instead of
selecting all of its fields between the two sides held in registers.
*/
struct Held_Sides {
	const Side& L;
	const Side& R;
	__device__ __forceinline__ Side operator()(const bool left) const { return left ? L : R; }
};

template <bool EX, class PICK>
__device__ __forceinline__ double flux_hlld(const Side& L, const Side& R, const Gas& g, double F[8],
                                            uint32_t& /*flag*/, const PICK& pick)
{
	using A = Ar<EX>;
	const double fast = fmax(L.cf, R.cf);
	const bool order = L.v0 <= R.v0;
	const double s_neg = A::sub(order ? L.v0 : R.v0, fast);  // eqn 67
	const double s_pos = A::add(order ? R.v0 : L.v0, fast);
	const double pbL = magnetic_pressure<EX>(L, g), pbR = magnetic_pressure<EX>(R, g);

	if (s_neg >= 0.0) {
		physical_flux<EX>(L, pbL, g, F);
		return fabs(s_pos);
	}
	if (s_pos <= 0.0) {
		physical_flux<EX>(R, pbR, g, F);
		return fabs(s_neg);
	}
	const double speed = fmax(fabs(s_neg), fabs(s_pos));

	const double bx = A::mul(0.5, A::add(L.b0, R.b0));
	const double bx2_mu = A::mul(A::mul(bx, bx), g.inv_mu0);
	const double sdL = A::sub(s_neg, L.v0), sdR = A::sub(s_pos, R.v0);       // < 0 and > 0 here
	const double ptL = A::add(L.p, pbL), ptR = A::add(R.p, pbR);
	const double rsdL = A::mul(L.rho, sdL), rsdR = A::mul(R.rho, sdR);
	// eqn 38; the denominator is sdR rho_R - sdL rho_L > 0
	const double s_mid = A::mul(A::add(A::sub(A::fma(sdR, R.m0, -A::mul(sdL, L.m0)), ptR), ptL),
	                            recip(A::sub(rsdR, rsdL)));
	const double smL = A::sub(s_neg, s_mid), smR = A::sub(s_pos, s_mid);     // < 0 and > 0 for physical states
	const double ismL = recip(smL), ismR = recip(smR);
	// eqn 43, and the square roots of the star densities with their reciprocals
	const double rsL = A::mul(rsdL, ismL), rsR = A::mul(rsdR, ismR);
	const double irL = rsqrt_nr(rsL), irR = rsqrt_nr(rsR);
	const double sqL = A::mul(rsL, irL), sqR = A::mul(rsR, irR);
	// eqn 51
	const double abx = A::mul(fabs(bx), g.inv_sqrt_mu0);
	const double ssL = A::fma(-abx, irL, s_mid), ssR = A::fma(abx, irR, s_mid);
	const double ptst = A::fma(rsdL, A::sub(s_mid, L.v0), ptL);
	const double thr = A::mul(DBL_EPS, ptst);
	// transverse star velocity and field of both sides, eqns 44-47
	const Star_T tl = star_transverse<EX>(L, rsdL, sdL, smL, s_mid, bx, bx2_mu, thr, g);
	const Star_T tr = star_transverse<EX>(R, rsdR, sdR, smR, s_mid, bx, bx2_mu, thr, g);

	// region order of hlld_athena.hpp:475-552: S*_L >= 0, S_M >= 0, S*_R > 0, else
	const bool left = s_mid >= 0.0;
	const bool star_l = ssL >= 0.0;
	const bool star_r = not star_l and not left and not (ssR > 0.0);
	const bool dbl = not star_l and not star_r;
	const bool useL = star_l or (dbl and left);   // the side the flux is taken from
	const Side S = pick(useL);
	const Star_T& ts = useL ? tl : tr;
	const double sd = useL ? sdL : sdR, ism = useL ? ismL : ismR, rs = useL ? rsL : rsR;
	const double pt = useL ? ptL : ptR, s_out = useL ? s_neg : s_pos;

	// that side's full star state, eqn 48 for the energy
	const double vb_star = A::fma(ts.w2, ts.b2, A::fma(ts.w1, ts.b1, A::mul(s_mid, bx)));
	const double vb = A::fma(S.v2, S.b2, A::fma(S.v1, S.b1, A::mul(S.v0, S.b0)));
	double us[8];
	us[0] = rs; us[1] = A::mul(rs, s_mid); us[2] = A::mul(rs, ts.w1); us[3] = A::mul(rs, ts.w2);
	{
		double e = A::fma(sd, S.E, -A::mul(pt, S.v0));
		e = A::fma(ptst, s_mid, e);
		e = A::fma(A::mul(bx, g.inv_mu0), A::sub(vb, vb_star), e);
		us[4] = A::mul(e, ism);
	}
	us[5] = bx; us[6] = ts.b1; us[7] = ts.b2;
	const double U0[8] = {S.rho, S.m0, S.m1, S.m2, S.E, S.b0, S.b1, S.b2};
	physical_flux<EX>(S, useL ? pbL : pbR, g, F);

	// double-star state, eqns 59-63 (the star state itself when Bx ~ 0)
	const double inv_sum = recip(A::add(sqL, sqR));
	const double sgn = (bx > 0.0) ? 1.0 : -1.0;
	const double cv = A::mul(sgn, g.inv_sqrt_mu0);
	const double v1 = A::mul(inv_sum, A::fma(cv, A::sub(tr.b1, tl.b1), A::fma(sqR, tr.w1, A::mul(sqL, tl.w1))));
	const double v2 = A::mul(inv_sum, A::fma(cv, A::sub(tr.b2, tl.b2), A::fma(sqR, tr.w2, A::mul(sqL, tl.w2))));
	const double wb = A::mul(A::mul(A::mul(sgn, sqL), sqR), g.sqrt_mu0);
	const double b1 = A::mul(inv_sum, A::fma(wb, A::sub(tr.w1, tl.w1), A::fma(sqR, tl.b1, A::mul(sqL, tr.b1))));
	const double b2 = A::mul(inv_sum, A::fma(wb, A::sub(tr.w2, tl.w2), A::fma(sqR, tl.b2, A::mul(sqL, tr.b2))));
	const double vb2 = A::fma(v2, b2, A::fma(v1, b1, A::mul(s_mid, bx)));
	const double e2 = left
		? A::sub(us[4], A::mul(A::mul(A::mul(sqL, sgn), A::sub(vb_star, vb2)), g.inv_sqrt_mu0))
		: A::add(us[4], A::mul(A::mul(A::mul(sqR, sgn), A::sub(vb_star, vb2)), g.inv_sqrt_mu0));
	const bool two = dbl and not (A::mul(A::mul(0.5, bx), bx) < thr);
	double u2[8];
	u2[0] = us[0]; u2[1] = us[1];
	u2[2] = two ? A::mul(rs, v1) : us[2];
	u2[3] = two ? A::mul(rs, v2) : us[3];
	u2[4] = two ? e2 : us[4];
	u2[5] = us[5];
	u2[6] = two ? b1 : us[6];
	u2[7] = two ? b2 : us[7];

	// single star: F + s_out (U* - U); double star: F + s_in U** - (s_in - s_out) U* - s_out U
	const double s_in = left ? ssL : ssR;
	const double c2 = dbl ? s_in : 0.0;
	const double c1 = dbl ? A::sub(s_in, s_out) : -s_out;
	#pragma unroll
	for (int v = 0; v < 8; v++) {
		if (v == 5) continue;
		F[v] = A::fma(-U0[v], s_out, A::fma(-us[v], c1, A::fma(u2[v], c2, F[v])));
	}
	F[5] = 0.0;
	return speed;
}

/*
Roe solver for adiabatic MHD, after Athena's esys_roe_adb_mhd and fluxes
(mhd/roe_athena.hpp:56-559; eigensystem eqns B17-B29 of Stone et al.,
ApJS 178, 2008), in units where the field is B / sqrt(mu0).  The signal
speed is the one of mhd/roe_athena.hpp:763-815.
*/
__device__ __forceinline__ double flux_roe(const Side& L, const Side& R, const Gas& g, double F[8],
                                           uint32_t& flag)
{
	const double gm1 = g.gamma - 1.0, gm2 = g.gamma - 2.0;
	const double ism = g.inv_sqrt_mu0;
	const double bxi = 0.5 * (L.b0 + R.b0) * ism;
	const double byl = L.b1 * ism, bzl = L.b2 * ism, byr = R.b1 * ism, bzr = R.b2 * ism;
	// pressure with mu0 = 1, as the reference's get_primitive call (roe_athena.hpp:706-721)
	const double pl = (L.E - 0.5 * L.rinv * (L.m0 * L.m0 + L.m1 * L.m1 + L.m2 * L.m2)
		- 0.5 * (L.b0 * L.b0 + L.b1 * L.b1 + L.b2 * L.b2)) * gm1;
	const double pr = (R.E - 0.5 * R.rinv * (R.m0 * R.m0 + R.m1 * R.m1 + R.m2 * R.m2)
		- 0.5 * (R.b0 * R.b0 + R.b1 * R.b1 + R.b2 * R.b2)) * gm1;

	const double sdl = sqrt(L.rho), sdr = sqrt(R.rho);
	const double isd = 1.0 / (sdl + sdr);
	const double droe = sdl * sdr;
	const double v1 = (sdl * L.v0 + sdr * R.v0) * isd;
	const double v2 = (sdl * L.v1 + sdr * R.v1) * isd;
	const double v3 = (sdl * L.v2 + sdr * R.v2) * isd;
	const double b2 = (sdr * byl + sdl * byr) * isd;
	const double b3 = (sdr * bzl + sdl * bzr) * isd;
	const double dby = byl - byr, dbz = bzl - bzr;
	const double x = 0.5 * (dby * dby + dbz * dbz) * (isd * isd);
	const double y = 0.5 * (L.rho + R.rho) / droe;
	const double pbl = 0.5 * (bxi * bxi + byl * byl + bzl * bzl);
	const double pbr = 0.5 * (bxi * bxi + byr * byr + bzr * bzr);
	const double h = ((L.E + pl + pbl) / sdl + (R.E + pr + pbr) / sdr) * isd;
	const double b1 = bxi;

	// eigensystem (B17-B29)
	const double di = 1.0 / droe;
	const double vsq = v1 * v1 + v2 * v2 + v3 * v3;
	const double btsq = b2 * b2 + b3 * b3;
	const double ystar = gm1 - gm2 * y;
	const double bt_starsq = ystar * btsq;
	const double vaxsq = b1 * b1 * di;
	const double hp = h - (vaxsq + btsq * di);
	const double twid_asq = fmax(gm1 * (hp - 0.5 * vsq) - gm2 * x, DBL_EPS);
	const double ct2 = bt_starsq * di;
	const double tsum = vaxsq + ct2 + twid_asq;
	const double tdif = vaxsq + ct2 - twid_asq;
	const double cf2_cs2 = sqrt(tdif * tdif + 4.0 * twid_asq * ct2);
	const double cfsq = 0.5 * (tsum + cf2_cs2);
	const double cf = sqrt(cfsq);
	const double cssq = twid_asq * vaxsq / cfsq;
	const double cs = sqrt(cssq);
	const double bt = sqrt(btsq);
	const double bt_star = sqrt(bt_starsq);
	double bet2 = 1.0, bet3 = 0.0;
	if (bt != 0.0) {
		const double ibt = 1.0 / bt;
		bet2 = b2 * ibt;
		bet3 = b3 * ibt;
	}
	const double iys = 1.0 / sqrt(ystar);
	const double bet2_star = bet2 * iys, bet3_star = bet3 * iys;
	const double bet_starsq = bet2_star * bet2_star + bet3_star * bet3_star;
	const double vbet = v2 * bet2_star + v3 * bet3_star;
	double alpha_f, alpha_s;
	if ((cfsq - cssq) == 0.0) {
		alpha_f = 1.0; alpha_s = 0.0;
	} else if ((twid_asq - cssq) <= 0.0) {
		alpha_f = 0.0; alpha_s = 1.0;
	} else if ((cfsq - twid_asq) <= 0.0) {
		alpha_f = 1.0; alpha_s = 0.0;
	} else {
		const double id = 1.0 / (cfsq - cssq);
		alpha_f = sqrt((twid_asq - cssq) * id);
		alpha_s = sqrt((cfsq - twid_asq) * id);
	}
	const double sqrtd = sqrt(droe);
	const double isqrtd = 1.0 / sqrtd;
	const double sg = (b1 > 0.0) ? 1.0 : -1.0;
	const double twid_a = sqrt(twid_asq);
	const double qf = cf * alpha_f * sg, qs = cs * alpha_s * sg;
	const double af_prime = twid_a * alpha_f * isqrtd, as_prime = twid_a * alpha_s * isqrtd;
	const double afpbb = af_prime * bt_star * bet_starsq, aspbb = as_prime * bt_star * bet_starsq;
	const double vax = sqrt(vaxsq);
	double ev[7] = {v1 - cf, v1 - vax, v1 - cs, v1, v1 + cs, v1 + vax, v1 + cf};

	// left and right conserved states in units B / sqrt(mu0); flux of each
	const double Ul[7] = {L.rho, L.m0, L.m1, L.m2, L.E, byl, bzl};
	const double Ur[7] = {R.rho, R.m0, R.m1, R.m2, R.E, byr, bzr};
	double Fl[7], Fr[7];
	{
		Fl[0] = L.m0;
		Fl[1] = L.m0 * L.v0 + pl - 0.5 * (bxi * bxi - byl * byl - bzl * bzl);
		Fl[2] = L.m0 * L.v1 - bxi * byl;
		Fl[3] = L.m0 * L.v2 - bxi * bzl;
		Fl[4] = (L.E + pl) * L.v0 + pbl * L.v0 - bxi * (bxi * L.v0 + byl * L.v1 + bzl * L.v2);
		Fl[5] = byl * L.v0 - bxi * L.v1;
		Fl[6] = bzl * L.v0 - bxi * L.v2;
		Fr[0] = R.m0;
		Fr[1] = R.m0 * R.v0 + pr - 0.5 * (bxi * bxi - byr * byr - bzr * bzr);
		Fr[2] = R.m0 * R.v1 - bxi * byr;
		Fr[3] = R.m0 * R.v2 - bxi * bzr;
		Fr[4] = (R.E + pr) * R.v0 + pbr * R.v0 - bxi * (bxi * R.v0 + byr * R.v1 + bzr * R.v2);
		Fr[5] = byr * R.v0 - bxi * R.v1;
		Fr[6] = bzr * R.v0 - bxi * R.v2;
	}

	double Fo[7];
	if (ev[0] >= 0.0) {
		#pragma unroll
		for (int r = 0; r < 7; r++) Fo[r] = Fl[r];
	} else if (ev[6] <= 0.0) {
		#pragma unroll
		for (int r = 0; r < 7; r++) Fo[r] = Fr[r];
	} else {
		// right eigenvectors as columns, R[row][wave]
		double Rm[7][7];
		Rm[0][0] = alpha_f; Rm[0][1] = 0.0; Rm[0][2] = alpha_s; Rm[0][3] = 1.0;
		Rm[0][4] = alpha_s; Rm[0][5] = 0.0; Rm[0][6] = alpha_f;
		Rm[1][0] = alpha_f * ev[0]; Rm[1][1] = 0.0; Rm[1][2] = alpha_s * ev[2]; Rm[1][3] = v1;
		Rm[1][4] = alpha_s * ev[4]; Rm[1][5] = 0.0; Rm[1][6] = alpha_f * ev[6];
		{
			const double qa = alpha_f * v2, qb = alpha_s * v2, qc = qs * bet2_star, qd = qf * bet2_star;
			Rm[2][0] = qa + qc; Rm[2][1] = -bet3; Rm[2][2] = qb - qd; Rm[2][3] = v2;
			Rm[2][4] = qb + qd; Rm[2][5] = bet3; Rm[2][6] = qa - qc;
		}
		{
			const double qa = alpha_f * v3, qb = alpha_s * v3, qc = qs * bet3_star, qd = qf * bet3_star;
			Rm[3][0] = qa + qc; Rm[3][1] = bet2; Rm[3][2] = qb - qd; Rm[3][3] = v3;
			Rm[3][4] = qb + qd; Rm[3][5] = -bet2; Rm[3][6] = qa - qc;
		}
		Rm[4][0] = alpha_f * (hp - v1 * cf) + qs * vbet + aspbb;
		Rm[4][1] = -(v2 * bet3 - v3 * bet2);
		Rm[4][2] = alpha_s * (hp - v1 * cs) - qf * vbet - afpbb;
		Rm[4][3] = 0.5 * vsq + gm2 * x / gm1;
		Rm[4][4] = alpha_s * (hp + v1 * cs) + qf * vbet - afpbb;
		Rm[4][5] = -Rm[4][1];
		Rm[4][6] = alpha_f * (hp + v1 * cf) - qs * vbet + aspbb;
		Rm[5][0] = as_prime * bet2_star; Rm[5][1] = -bet3 * sg * isqrtd; Rm[5][2] = -af_prime * bet2_star;
		Rm[5][3] = 0.0; Rm[5][4] = Rm[5][2]; Rm[5][5] = Rm[5][1]; Rm[5][6] = Rm[5][0];
		Rm[6][0] = as_prime * bet3_star; Rm[6][1] = bet2 * sg * isqrtd; Rm[6][2] = -af_prime * bet3_star;
		Rm[6][3] = 0.0; Rm[6][4] = Rm[6][2]; Rm[6][5] = Rm[6][1]; Rm[6][6] = Rm[6][0];

		// left eigenvectors as rows
		double norm = 0.5 / twid_asq;
		const double cff = norm * alpha_f * cf, css = norm * alpha_s * cs;
		const double qfn = qf * norm, qsn = qs * norm;
		const double af = norm * af_prime * droe, as = norm * as_prime * droe;
		const double afpb = norm * af_prime * bt_star, aspb = norm * as_prime * bt_star;
		norm *= gm1;
		const double af_n = alpha_f * norm, as_n = alpha_s * norm;
		const double ibs = 1.0 / bet_starsq;
		const double q2_star = bet2_star * ibs, q3_star = bet3_star * ibs;
		const double vqstr = v2 * q2_star + v3 * q3_star;
		norm *= 2.0;
		double Lm[7][7];
		Lm[0][0] = af_n * (vsq - hp) + cff * (cf + v1) - qsn * vqstr - aspb;
		Lm[0][1] = -af_n * v1 - cff;
		Lm[0][2] = -af_n * v2 + qsn * q2_star;
		Lm[0][3] = -af_n * v3 + qsn * q3_star;
		Lm[0][4] = af_n;
		Lm[0][5] = as * q2_star - af_n * b2;
		Lm[0][6] = as * q3_star - af_n * b3;
		Lm[1][0] = 0.5 * (v2 * bet3 - v3 * bet2); Lm[1][1] = 0.0; Lm[1][2] = -0.5 * bet3;
		Lm[1][3] = 0.5 * bet2; Lm[1][4] = 0.0; Lm[1][5] = -0.5 * sqrtd * bet3 * sg;
		Lm[1][6] = 0.5 * sqrtd * bet2 * sg;
		Lm[2][0] = as_n * (vsq - hp) + css * (cs + v1) + qfn * vqstr + afpb;
		Lm[2][1] = -as_n * v1 - css;
		Lm[2][2] = -as_n * v2 - qfn * q2_star;
		Lm[2][3] = -as_n * v3 - qfn * q3_star;
		Lm[2][4] = as_n;
		Lm[2][5] = -af * q2_star - as_n * b2;
		Lm[2][6] = -af * q3_star - as_n * b3;
		Lm[3][0] = 1.0 - norm * (0.5 * vsq - gm2 * x / gm1);
		Lm[3][1] = norm * v1; Lm[3][2] = norm * v2; Lm[3][3] = norm * v3;
		Lm[3][4] = -norm; Lm[3][5] = norm * b2; Lm[3][6] = norm * b3;
		Lm[4][0] = as_n * (vsq - hp) + css * (cs - v1) - qfn * vqstr + afpb;
		Lm[4][1] = -as_n * v1 + css;
		Lm[4][2] = -as_n * v2 + qfn * q2_star;
		Lm[4][3] = -as_n * v3 + qfn * q3_star;
		Lm[4][4] = as_n;
		Lm[4][5] = Lm[2][5];
		Lm[4][6] = Lm[2][6];
		Lm[5][0] = -Lm[1][0]; Lm[5][1] = 0.0; Lm[5][2] = -Lm[1][2]; Lm[5][3] = -Lm[1][3];
		Lm[5][4] = 0.0; Lm[5][5] = Lm[1][5]; Lm[5][6] = Lm[1][6];
		Lm[6][0] = af_n * (vsq - hp) + cff * (cf - v1) + qsn * vqstr - aspb;
		Lm[6][1] = -af_n * v1 + cff;
		Lm[6][2] = -af_n * v2 - qsn * q2_star;
		Lm[6][3] = -af_n * v3 - qsn * q3_star;
		Lm[6][4] = af_n;
		Lm[6][5] = Lm[0][5];
		Lm[6][6] = Lm[0][6];

		double a[7], dU[7];
		#pragma unroll
		for (int m = 0; m < 7; m++) dU[m] = Ur[m] - Ul[m];
		#pragma unroll
		for (int n = 0; n < 7; n++) {
			double s = 0.0;
			#pragma unroll
			for (int m = 0; m < 7; m++) s += Lm[n][m] * dU[m];
			a[n] = s;
		}
		// positivity of the intermediate states
		double u[7];
		uint32_t roe_fail = 0;
		#pragma unroll
		for (int m = 0; m < 7; m++) u[m] = Ul[m];
		#pragma unroll
		for (int n = 0; n < 6; n++) {
			#pragma unroll
			for (int m = 0; m < 7; m++) u[m] += a[n] * Rm[m][n];
			// the reference throws at the first failing intermediate state
			if (ev[n + 1] > ev[n] and roe_fail == 0) {
				if (u[0] <= 0.0) {
					roe_fail = PAMHD_FLAG_ROE_DENSITY;
				} else {
					const double pi = u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0]
						- 0.5 * (u[5] * u[5] + u[6] * u[6] + bxi * bxi);
					if (pi < 0.0) roe_fail = PAMHD_FLAG_ROE_PRESSURE;
				}
			}
		}
		if (flag == 0) flag = roe_fail;
		#pragma unroll
		for (int r = 0; r < 7; r++) Fo[r] = 0.5 * (Fl[r] + Fr[r]);
		#pragma unroll
		for (int m = 0; m < 7; m++) {
			const double c = 0.5 * a[m] * fabs(ev[m]);
			#pragma unroll
			for (int r = 0; r < 7; r++) Fo[r] -= c * Rm[r][m];
		}
	}
	F[0] = Fo[0]; F[1] = Fo[1]; F[2] = Fo[2]; F[3] = Fo[3]; F[4] = Fo[4];
	F[5] = 0.0;
	F[6] = Fo[5] * g.sqrt_mu0;
	F[7] = Fo[6] * g.sqrt_mu0;

	// signal speed (roe_athena.hpp:763-815)
	const double fast = fmax(L.cf, R.cf);
	const bool order = L.v0 <= R.v0;
	const double s_neg = (order ? L.v0 : R.v0) - fast;
	const double s_pos = (order ? R.v0 : L.v0) + fast;
	if (s_neg >= 0.0) return fabs(s_pos);
	if (s_pos <= 0.0) return fabs(s_neg);
	return fmax(fabs(s_neg), fabs(s_pos));
}

template <bool EX = false>
__device__ __forceinline__ double flux_hlld(const Side& L, const Side& R, const Gas& g, double F[8],
                                            uint32_t& flag)
{
	return flux_hlld<EX>(L, R, g, F, flag, Held_Sides{L, R});
}

// pick: see flux_hlld (the other solvers use the sides held); EX: Ar<true> arithmetic for HLLD
template <int SOLVER, bool EX = false, class PICK>
__device__ __forceinline__ double solve_face(const Side& L, const Side& R, const Gas& g, double F[8],
                                             uint32_t& flag, const PICK& pick)
{
	flag = L.bad | R.bad;
	if (flag & PAMHD_FLAG_DENSITY) flag = PAMHD_FLAG_DENSITY;
	else if (flag & PAMHD_FLAG_PRESSURE) flag = PAMHD_FLAG_PRESSURE;
	if (SOLVER == PAMHD_RUSANOV) return flux_rusanov<false, EX>(L, R, g, F, flag);
	if (SOLVER == PAMHD_HLL_ATHENA) return flux_hll<false, EX>(L, R, g, F, flag);
	if (SOLVER == PAMHD_HLLD_ATHENA) return flux_hlld<EX>(L, R, g, F, flag, pick);
	return flux_roe(L, R, g, F, flag);
}

template <int SOLVER, bool EX = false>
__device__ __forceinline__ double solve_face(const Side& L, const Side& R, const Gas& g, double F[8],
                                             uint32_t& flag)
{
	return solve_face<SOLVER, EX>(L, R, g, F, flag, Held_Sides{L, R});
}

} // namespace pamhd_b200

#endif
