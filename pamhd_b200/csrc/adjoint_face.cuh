/*
Discrete adjoint of one face: the vector-Jacobian product of the face
flux F(U_L, U_R) of each Riemann solver.

Given the cotangent phi = dJ/dF of a face's flux (face frame, x = normal),
face_vjp<SOLVER> returns gL = (dF/dU_L)^T phi and gR = (dF/dU_R)^T phi,
with U the conservative states (rho, mom, E, B) in the face frame.  The
flux is the one of the fused step (mhd_device.cuh): the cell's derived
quantities (1/rho, velocity, pressure, fast speed along the normal) are
recomputed from U here, and their adjoints are propagated back to U, so
the product is exact for the function the forward step evaluates (up to
round-off).  Branches (supersonic upwinding, HLLD degeneracy and region
choice, the max of the fast speeds) follow the forward evaluation: the
product is that of the branch taken.  The timestep is a constant of the
linearisation (the adjoint runs on a frozen dt schedule).

Reverse mode is written out by hand: the forward pass keeps every
intermediate in registers, then the statements are differentiated in
reverse order; a variable's adjoint is named a_<variable>.

__host__ __device__ so that the CPU tests can check it against finite
differences of the oracle without a GPU.
*/
#ifndef PAMHD_B200_ADJOINT_FACE_CUH
#define PAMHD_B200_ADJOINT_FACE_CUH

#ifndef __CUDACC__
#include <cmath>
#define __host__
#define __device__
#define __forceinline__ inline
using std::fabs;
using std::fmax;
using std::sqrt;
#endif

namespace pamhd_b200 {
namespace adjoint {

struct Gas_Adj {
	double gamma, inv_mu0, inv_sqrt_mu0, sqrt_mu0;
};

/*
1 / x.  On the device: Newton-Raphson iteration r <- r + r (1 - x r) from
the estimate of PTX rcp.approx.ftz.f64, two iterations (within one unit in
the last place for normal non-zero x); on the host, IEEE division.  Each
denominator of the products below is inverted once and multiplied in.
*/
__host__ __device__ __forceinline__ double rcp(const double x)
{
#ifdef __CUDA_ARCH__
	double r;
	asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
	double e = fma(-x, r, 1.0);
	r = fma(r, e, r);
	e = fma(-x, r, 1.0);
	return fma(r, e, r);
#else
	return 1.0 / x;
#endif
}

// forward intermediates of one cell seen from a face
struct Side_Fwd {
	double rho, m0, m1, m2, E, b0, b1, b2;
	double r, v0, v1, v2, b2s, m2s, ke, pb, p, cs2, va2, sum2, cos2, base, prod, ts, q, h, cf;
	double ib2s, iq, icf;  // 1 / b2s, 1 / q (0 when q is 0), 1 / cf
	bool has_field;
};

// adjoints of a side's derived quantities gathered before the reverse of derive()
struct Side_Adj {
	double rho, m0, m1, m2, E, b0, b1, b2;  // direct dependence on U
	double v0, v1, v2, p, pb, cf;           // through the derived quantities
};

__host__ __device__ __forceinline__ void side_forward(const double* U, const Gas_Adj& g, Side_Fwd& s)
{
	s.rho = U[0]; s.m0 = U[1]; s.m1 = U[2]; s.m2 = U[3]; s.E = U[4]; s.b0 = U[5]; s.b1 = U[6]; s.b2 = U[7];
	s.r = rcp(s.rho);
	s.v0 = s.m0 * s.r;
	s.v1 = s.m1 * s.r;
	s.v2 = s.m2 * s.r;
	s.b2s = s.b0 * s.b0 + s.b1 * s.b1 + s.b2 * s.b2;
	s.m2s = s.m0 * s.m0 + s.m1 * s.m1 + s.m2 * s.m2;
	s.ke = 0.5 * s.r * s.m2s;
	s.pb = 0.5 * g.inv_mu0 * s.b2s;
	s.p = (s.E - s.ke - s.pb) * (g.gamma - 1.0);
	s.cs2 = g.gamma * s.p * s.r;
	s.has_field = s.b2s > 0.0;
	if (s.has_field) {
		s.va2 = s.b2s * g.inv_mu0 * s.r;
		s.sum2 = s.cs2 + s.va2;
		s.ib2s = rcp(s.b2s);
		s.cos2 = s.b0 * s.b0 * s.ib2s;
		s.base = s.cs2 * s.cs2 + s.va2 * s.va2;
		s.prod = 2.0 * s.cs2 * s.va2;
		s.ts = s.base + s.prod * (1.0 - 2.0 * s.cos2);
		s.q = sqrt(fmax(s.ts, 0.0));
		s.iq = s.q > 0.0 ? rcp(s.q) : 0.0;
		s.h = 0.5 * (s.sum2 + s.q);
		s.cf = sqrt(s.h);
	} else {
		s.va2 = s.sum2 = s.cos2 = s.base = s.prod = s.ts = s.q = s.ib2s = s.iq = 0.0;
		s.h = s.cs2;
		s.cf = sqrt(fmax(s.cs2, 0.0));
	}
	s.icf = s.cf > 0.0 ? rcp(s.cf) : 0.0;
}

__host__ __device__ __forceinline__ void side_adj_zero(Side_Adj& a)
{
	a.rho = a.m0 = a.m1 = a.m2 = a.E = a.b0 = a.b1 = a.b2 = 0.0;
	a.v0 = a.v1 = a.v2 = a.p = a.pb = a.cf = 0.0;
}

// reverse of side_forward: g[8] receives dJ/dU of the side
__host__ __device__ __forceinline__ void side_reverse(const Side_Fwd& s, const Side_Adj& a, const Gas_Adj& g,
                                                      double* out)
{
	double a_rho = a.rho, a_m0 = a.m0, a_m1 = a.m1, a_m2 = a.m2, a_E = a.E;
	double a_b0 = a.b0, a_b1 = a.b1, a_b2 = a.b2;
	double a_p = a.p, a_pb = a.pb, a_r = 0.0, a_b2s = 0.0, a_cs2 = 0.0;
	if (s.has_field) {
		// cf = sqrt(h), h = (sum2 + q)/2, q = sqrt(ts), ts = base + prod (1 - 2 cos2)
		const double a_h = a.cf * 0.5 * s.icf;
		const double a_sum2 = 0.5 * a_h;
		const double a_q = 0.5 * a_h;
		const double a_ts = a_q * 0.5 * s.iq;
		const double a_base = a_ts;
		const double a_prod = a_ts * (1.0 - 2.0 * s.cos2);
		const double a_cos2 = -2.0 * s.prod * a_ts;
		// prod = 2 cs2 va2, base = cs2^2 + va2^2, sum2 = cs2 + va2
		a_cs2 += 2.0 * s.va2 * a_prod + 2.0 * s.cs2 * a_base + a_sum2;
		const double a_va2 = 2.0 * s.cs2 * a_prod + 2.0 * s.va2 * a_base + a_sum2;
		// cos2 = b0^2 / b2s
		a_b0 += 2.0 * s.b0 * s.ib2s * a_cos2;
		a_b2s += -s.cos2 * s.ib2s * a_cos2;
		// va2 = b2s / mu0 * r
		a_b2s += g.inv_mu0 * s.r * a_va2;
		a_r += s.b2s * g.inv_mu0 * a_va2;
	} else {
		a_cs2 += s.cs2 > 0.0 ? a.cf * 0.5 * s.icf : 0.0;
	}
	// cs2 = gamma p r
	a_p += g.gamma * s.r * a_cs2;
	a_r += g.gamma * s.p * a_cs2;
	// p = (E - ke - pb)(gamma - 1)
	const double gm1 = g.gamma - 1.0;
	a_E += gm1 * a_p;
	const double a_ke = -gm1 * a_p;
	a_pb += -gm1 * a_p;
	// pb = b2s / (2 mu0), ke = r m2s / 2
	a_b2s += 0.5 * g.inv_mu0 * a_pb;
	a_r += 0.5 * s.m2s * a_ke;
	const double a_m2s = 0.5 * s.r * a_ke;
	a_m0 += 2.0 * s.m0 * a_m2s;
	a_m1 += 2.0 * s.m1 * a_m2s;
	a_m2 += 2.0 * s.m2 * a_m2s;
	a_b0 += 2.0 * s.b0 * a_b2s;
	a_b1 += 2.0 * s.b1 * a_b2s;
	a_b2 += 2.0 * s.b2 * a_b2s;
	// v = m r
	a_m0 += s.r * a.v0;
	a_m1 += s.r * a.v1;
	a_m2 += s.r * a.v2;
	a_r += s.m0 * a.v0 + s.m1 * a.v1 + s.m2 * a.v2;
	// r = 1 / rho
	a_rho += -s.r * s.r * a_r;
	out[0] = a_rho; out[1] = a_m0; out[2] = a_m1; out[3] = a_m2;
	out[4] = a_E; out[5] = a_b0; out[6] = a_b1; out[7] = a_b2;
}

/*
Physical flux (background field zero) and its reverse: F = flux(U, v, p, pb)
(mhd/common.hpp:146-244).
*/
__host__ __device__ __forceinline__ void phys_forward(const Side_Fwd& s, const Gas_Adj& g, double* F)
{
	const double vb = s.v0 * s.b0 + s.v1 * s.b1 + s.v2 * s.b2;
	F[0] = s.m0;
	F[1] = s.m0 * s.v0 - g.inv_mu0 * s.b0 * s.b0 + s.p + s.pb;
	F[2] = s.m1 * s.v0 - g.inv_mu0 * s.b0 * s.b1;
	F[3] = s.m2 * s.v0 - g.inv_mu0 * s.b0 * s.b2;
	F[4] = s.v0 * (s.E + s.p + s.pb) - g.inv_mu0 * s.b0 * vb;
	F[5] = 0.0;
	F[6] = s.v0 * s.b1 - s.b0 * s.v1;
	F[7] = s.v0 * s.b2 - s.b0 * s.v2;
}

__host__ __device__ __forceinline__ void phys_reverse(const Side_Fwd& s, const Gas_Adj& g, const double* aF,
                                                      Side_Adj& a)
{
	const double vb = s.v0 * s.b0 + s.v1 * s.b1 + s.v2 * s.b2;
	const double im = g.inv_mu0;
	// F0 = m0
	a.m0 += aF[0];
	// F1 = m0 v0 - im b0^2 + p + pb
	a.m0 += s.v0 * aF[1];
	a.v0 += s.m0 * aF[1];
	a.b0 += -2.0 * im * s.b0 * aF[1];
	a.p += aF[1];
	a.pb += aF[1];
	// F2 = m1 v0 - im b0 b1, F3 = m2 v0 - im b0 b2
	a.m1 += s.v0 * aF[2];
	a.m2 += s.v0 * aF[3];
	a.v0 += s.m1 * aF[2] + s.m2 * aF[3];
	a.b0 += -im * (s.b1 * aF[2] + s.b2 * aF[3]);
	a.b1 += -im * s.b0 * aF[2];
	a.b2 += -im * s.b0 * aF[3];
	// F4 = v0 (E + p + pb) - im b0 vb, vb = v.b
	a.v0 += (s.E + s.p + s.pb) * aF[4];
	a.E += s.v0 * aF[4];
	a.p += s.v0 * aF[4];
	a.pb += s.v0 * aF[4];
	a.b0 += -im * vb * aF[4];
	const double a_vb = -im * s.b0 * aF[4];
	a.v0 += s.b0 * a_vb;
	a.v1 += s.b1 * a_vb;
	a.v2 += s.b2 * a_vb;
	a.b0 += s.v0 * a_vb;
	a.b1 += s.v1 * a_vb;
	a.b2 += s.v2 * a_vb;
	// F6 = v0 b1 - b0 v1, F7 = v0 b2 - b0 v2
	a.v0 += s.b1 * aF[6] + s.b2 * aF[7];
	a.b1 += s.v0 * aF[6];
	a.b2 += s.v0 * aF[7];
	a.b0 += -s.v1 * aF[6] - s.v2 * aF[7];
	a.v1 += -s.b0 * aF[6];
	a.v2 += -s.b0 * aF[7];
}

/*
Kinks.  At a tie of max(a, b) / min(a, b) (equal to within round-off:
symmetric data give exact-arithmetic ties that rounding breaks by an ulp),
or at |x| with x = 0, the flux has no derivative; the adjoint then uses the average of the one-sided
derivatives (half to each argument, 0 for |0|), which is what a central
difference across the kink measures.  Ties are common, not exceptional, in
symmetric data such as the Orszag-Tang vortex.
*/
__host__ __device__ __forceinline__ void max_rev(const double a, const double b, const double g, double& ga, double& gb)
{
	// arguments equal to within round-off are ties of the exact-arithmetic flux
	const double tie = 1e-12 * fmax(fabs(a), fabs(b));
	if (a > b + tie) ga += g;
	else if (b > a + tie) gb += g;
	else { ga += 0.5 * g; gb += 0.5 * g; }
}

__host__ __device__ __forceinline__ double abs_rev(const double x, const double g)
{
	return x > 0.0 ? g : (x < 0.0 ? -g : 0.0);
}

__host__ __device__ __forceinline__ void state_of(const Side_Fwd& s, double* U)
{
	U[0] = s.rho; U[1] = s.m0; U[2] = s.m1; U[3] = s.m2; U[4] = s.E; U[5] = s.b0; U[6] = s.b1; U[7] = s.b2;
}

__host__ __device__ __forceinline__ void add_state(Side_Adj& a, const double* aU)
{
	a.rho += aU[0]; a.m0 += aU[1]; a.m1 += aU[2]; a.m2 += aU[3];
	a.E += aU[4]; a.b0 += aU[5]; a.b1 += aU[6]; a.b2 += aU[7];
}

// ---------------------------------------------------------------- Rusanov

// F = (FL + FR)/2 - s/2 (UR - UL), s = max(|vL0|, |vR0|) + max(cfL, cfR)
__host__ __device__ __forceinline__ void rusanov_vjp(const double* UL, const double* UR, const Gas_Adj& g,
                                                     const double* phi, double* gL, double* gR, double* F = nullptr)
{
	Side_Fwd L, R;
	side_forward(UL, g, L);
	side_forward(UR, g, R);
	const double aL = fabs(L.v0), aR = fabs(R.v0);
	const double s = fmax(aL, aR) + fmax(L.cf, R.cf);
	if (F != nullptr) {
		double FL[8], FR[8];
		phys_forward(L, g, FL);
		phys_forward(R, g, FR);
		for (int v = 0; v < 8; v++) F[v] = 0.5 * (FL[v] + FR[v]) - 0.5 * s * (UR[v] - UL[v]);
	}
	Side_Adj AL, AR;
	side_adj_zero(AL);
	side_adj_zero(AR);
	double aFh[8], a_s = 0.0;
	for (int v = 0; v < 8; v++) {
		aFh[v] = 0.5 * phi[v];
		a_s += -0.5 * (UR[v] - UL[v]) * phi[v];
	}
	double dUR[8], dUL[8];
	for (int v = 0; v < 8; v++) {
		dUR[v] = -0.5 * s * phi[v];
		dUL[v] = 0.5 * s * phi[v];
	}
	add_state(AL, dUL);
	add_state(AR, dUR);
	phys_reverse(L, g, aFh, AL);
	phys_reverse(R, g, aFh, AR);
	// s = max(|vL0|, |vR0|) + max(cfL, cfR)
	double a_aL = 0.0, a_aR = 0.0;
	max_rev(aL, aR, a_s, a_aL, a_aR);
	AL.v0 += abs_rev(L.v0, a_aL);
	AR.v0 += abs_rev(R.v0, a_aR);
	max_rev(L.cf, R.cf, a_s, AL.cf, AR.cf);
	side_reverse(L, AL, g, gL);
	side_reverse(R, AR, g, gR);
}

// ---------------------------------------------------------------- HLL

/*
bm = min(S_L, 0), bp = max(S_R, 0), a = FL - bm UL, b = FR - bp UR (field
normal component zero), F = (a + b)/2 + (a - b) w, w = (bp + bm)/(2 (bp - bm)).
*/
__host__ __device__ __forceinline__ void hll_vjp(const double* UL, const double* UR, const Gas_Adj& g,
                                                 const double* phi, double* gL, double* gR, double* F = nullptr)
{
	Side_Fwd L, R;
	side_forward(UL, g, L);
	side_forward(UR, g, R);
	const bool left_fast = L.cf >= R.cf;
	const double fast = left_fast ? L.cf : R.cf;
	const bool order = L.v0 <= R.v0;
	const double s_neg = (order ? L.v0 : R.v0) - fast;
	const double s_pos = (order ? R.v0 : L.v0) + fast;
	const bool bm_on = s_neg < 0.0, bp_on = s_pos > 0.0;
	const double bm = bm_on ? s_neg : 0.0, bp = bp_on ? s_pos : 0.0;
	const double width = bp - bm;
	Side_Adj AL, AR;
	side_adj_zero(AL);
	side_adj_zero(AR);
	if (not (width > 0.0)) {
		for (int v = 0; v < 8; v++) {
			gL[v] = gR[v] = 0.0;
			if (F != nullptr) F[v] = 0.0;
		}
		return;
	}
	double FL[8], FR[8];
	phys_forward(L, g, FL);
	phys_forward(R, g, FR);
	const double iwidth = rcp(width);
	const double w = 0.5 * (bp + bm) * iwidth;
	double a[8], b[8];
	for (int v = 0; v < 8; v++) {
		a[v] = v == 5 ? 0.0 : FL[v] - bm * UL[v];
		b[v] = v == 5 ? 0.0 : FR[v] - bp * UR[v];
		if (F != nullptr) F[v] = 0.5 * (a[v] + b[v]) + (a[v] - b[v]) * w;
	}
	// reverse
	double a_w = 0.0, aa[8], ab[8];
	for (int v = 0; v < 8; v++) {
		aa[v] = (0.5 + w) * phi[v];
		ab[v] = (0.5 - w) * phi[v];
		a_w += (a[v] - b[v]) * phi[v];
	}
	aa[5] = ab[5] = 0.0;
	// w = (bp + bm) / (2 width), width = bp - bm
	const double a_width = -w * iwidth * a_w;
	double a_bp = 0.5 * iwidth * a_w + a_width;
	double a_bm = 0.5 * iwidth * a_w - a_width;
	double dUL[8], dUR[8];
	for (int v = 0; v < 8; v++) {
		a_bm += -UL[v] * aa[v];
		a_bp += -UR[v] * ab[v];
		dUL[v] = -bm * aa[v];
		dUR[v] = -bp * ab[v];
	}
	add_state(AL, dUL);
	add_state(AR, dUR);
	phys_reverse(L, g, aa, AL);
	phys_reverse(R, g, ab, AR);
	// bm = min(s_neg, 0), bp = max(s_pos, 0)
	const double a_sneg = s_neg < 0.0 ? a_bm : (s_neg == 0.0 ? 0.5 * a_bm : 0.0);
	const double a_spos = s_pos > 0.0 ? a_bp : (s_pos == 0.0 ? 0.5 * a_bp : 0.0);
	// s_neg = min(vL0, vR0) - fast, s_pos = max(vL0, vR0) + fast
	max_rev(L.v0, R.v0, a_spos, AL.v0, AR.v0);
	max_rev(R.v0, L.v0, a_sneg, AL.v0, AR.v0);
	max_rev(L.cf, R.cf, -a_sneg + a_spos, AL.cf, AR.cf);
	side_reverse(L, AL, g, gL);
	side_reverse(R, AR, g, gR);
}

// ---------------------------------------------------------------- HLLD

// one side's star state (eqns 44-48) and everything its reverse needs
struct Star {
	double sd, sm, rs, tmp, t1, t2, w1, w2, sb1, sb2, vb, vb_old, num_e, Es;
	double ism, itmp;  // 1 / sm, 1 / tmp (0 when degenerate)
	bool degenerate;
};

__host__ __device__ __forceinline__ void hlld_vjp(const double* UL, const double* UR, const Gas_Adj& g,
                                                  const double* phi, double* gL, double* gR, double* F = nullptr)
{
	constexpr double eps = 2.220446049250313080847e-16;
	Side_Fwd L, R;
	side_forward(UL, g, L);
	side_forward(UR, g, R);
	Side_Adj AL, AR;
	side_adj_zero(AL);
	side_adj_zero(AR);
	const bool left_fast = L.cf >= R.cf;
	const double fast = left_fast ? L.cf : R.cf;
	const bool order = L.v0 <= R.v0;
	const double s_neg = (order ? L.v0 : R.v0) - fast;
	const double s_pos = (order ? R.v0 : L.v0) + fast;
	const double im = g.inv_mu0;

	// supersonic: the upwind physical flux
	if (s_neg >= 0.0 or s_pos <= 0.0) {
		const bool up_left = s_neg >= 0.0;
		const Side_Fwd& S = up_left ? L : R;
		Side_Adj& A = up_left ? AL : AR;
		if (F != nullptr) phys_forward(S, g, F);
		phys_reverse(S, g, phi, A);
		side_reverse(L, AL, g, gL);
		side_reverse(R, AR, g, gR);
		return;
	}

	const double bx = 0.5 * (L.b0 + R.b0);
	const double bx2m = bx * bx * im;
	const double ptL = L.p + L.pb, ptR = R.p + R.pb;
	Star sL, sR;
	sL.sd = s_neg - L.v0;
	sR.sd = s_pos - R.v0;
	const double num = sR.sd * R.m0 - sL.sd * L.m0 - ptR + ptL;
	const double den = sR.sd * R.rho - sL.sd * L.rho;
	const double iden = rcp(den);
	const double s_mid = num * iden;
	sL.sm = s_neg - s_mid;
	sR.sm = s_pos - s_mid;
	sL.ism = rcp(sL.sm);
	sR.ism = rcp(sR.sm);
	sL.rs = L.rho * sL.sd * sL.ism;
	sR.rs = R.rho * sR.sd * sR.ism;
	const double sqL = sqrt(sL.rs), sqR = sqrt(sR.rs);
	const double isqL = rcp(sqL), isqR = rcp(sqR);
	const double abx = fabs(bx) * g.inv_sqrt_mu0;
	const double ssL = s_mid - abx * isqL, ssR = s_mid + abx * isqR;
	const double ptst = ptL + L.rho * sL.sd * (s_mid - L.v0);
	const double thr = eps * ptst;

	auto star_fwd = [&](const Side_Fwd& S, Star& st, const double pt) {
		st.tmp = S.rho * st.sd * st.sm - bx2m;
		st.degenerate = fabs(st.tmp) < thr;
		if (st.degenerate) {
			st.t1 = st.t2 = st.itmp = 0.0;
			st.w1 = S.v1; st.w2 = S.v2; st.sb1 = S.b1; st.sb2 = S.b2;
		} else {
			st.itmp = rcp(st.tmp);
			st.t1 = bx * (s_mid - S.v0) * im * st.itmp;
			st.t2 = (S.rho * st.sd * st.sd - bx2m) * st.itmp;
			st.w1 = S.v1 - S.b1 * st.t1;
			st.w2 = S.v2 - S.b2 * st.t1;
			st.sb1 = S.b1 * st.t2;
			st.sb2 = S.b2 * st.t2;
		}
		st.vb = s_mid * bx + st.w1 * st.sb1 + st.w2 * st.sb2;
		st.vb_old = S.v0 * S.b0 + S.v1 * S.b1 + S.v2 * S.b2;
		st.num_e = st.sd * S.E - pt * S.v0 + ptst * s_mid + bx * im * (st.vb_old - st.vb);
		st.Es = st.num_e * st.ism;
	};
	star_fwd(L, sL, ptL);
	star_fwd(R, sR, ptR);
	const double uL[8] = {sL.rs, sL.rs * s_mid, sL.rs * sL.w1, sL.rs * sL.w2, sL.Es, bx, sL.sb1, sL.sb2};
	const double uR[8] = {sR.rs, sR.rs * s_mid, sR.rs * sR.w1, sR.rs * sR.w2, sR.Es, bx, sR.sb1, sR.sb2};

	// adjoints of the fan quantities
	double a_sneg = 0.0, a_spos = 0.0, a_smid = 0.0, a_bx = 0.0, a_ssL = 0.0, a_ssR = 0.0;
	double a_uL[8] = {0, 0, 0, 0, 0, 0, 0, 0}, a_uR[8] = {0, 0, 0, 0, 0, 0, 0, 0};
	double a_sqL = 0.0, a_sqR = 0.0, a_ptst = 0.0;
	double a_w1L = 0.0, a_w2L = 0.0, a_sb1L = 0.0, a_sb2L = 0.0, a_vbL = 0.0;
	double a_w1R = 0.0, a_w2R = 0.0, a_sb1R = 0.0, a_sb2R = 0.0, a_vbR = 0.0;

	const bool left = s_mid >= 0.0;
	if (ssL >= 0.0 or (not left and not (ssR > 0.0))) {
		// outer regions: F = FS + s (u* - US), field normal component zero
		const bool useL = ssL >= 0.0;
		const Side_Fwd& S = useL ? L : R;
		Side_Adj& A = useL ? AL : AR;
		const double* us = useL ? uL : uR;
		double* a_us = useL ? a_uL : a_uR;
		const double s = useL ? s_neg : s_pos;
		double US[8];
		state_of(S, US);
		if (F != nullptr) {
			phys_forward(S, g, F);
			for (int v = 0; v < 8; v++) F[v] += s * (us[v] - US[v]);
			F[5] = 0.0;
		}
		double ph[8];
		for (int v = 0; v < 8; v++) ph[v] = v == 5 ? 0.0 : phi[v];
		double a_s = 0.0, dU[8];
		for (int v = 0; v < 8; v++) {
			a_s += (us[v] - US[v]) * ph[v];
			a_us[v] += s * ph[v];
			dU[v] = -s * ph[v];
		}
		add_state(A, dU);
		phys_reverse(S, g, ph, A);
		if (useL) a_sneg += a_s; else a_spos += a_s;
	} else {
		// inner regions: F = FS + u** ss - u* (ss - s) - US s
		const Side_Fwd& S = left ? L : R;
		Side_Adj& A = left ? AL : AR;
		const double* us = left ? uL : uR;
		double* a_us = left ? a_uL : a_uR;
		const double s = left ? s_neg : s_pos;
		const double ss = left ? ssL : ssR;
		double US[8];
		state_of(S, US);
		const bool dstar = not (0.5 * bx * bx < thr);
		double u2[8];
		double isum = 0.0, sgn = 1.0, cv = 0.0, v1 = 0.0, v2 = 0.0, wb = 0.0, bb1 = 0.0, bb2 = 0.0, vb2 = 0.0;
		double n1 = 0.0, n2 = 0.0, k1 = 0.0, k2 = 0.0;
		if (not dstar) {
			for (int v = 0; v < 8; v++) u2[v] = us[v];
		} else {
			isum = rcp(sqL + sqR);
			sgn = bx > 0.0 ? 1.0 : -1.0;
			cv = sgn * g.inv_sqrt_mu0;
			n1 = (sqL * sL.w1 + sqR * sR.w1) + cv * (sR.sb1 - sL.sb1);
			n2 = (sqL * sL.w2 + sqR * sR.w2) + cv * (sR.sb2 - sL.sb2);
			v1 = isum * n1;
			v2 = isum * n2;
			wb = sgn * sqL * sqR * g.sqrt_mu0;
			k1 = (sqL * sR.sb1 + sqR * sL.sb1) + wb * (sR.w1 - sL.w1);
			k2 = (sqL * sR.sb2 + sqR * sL.sb2) + wb * (sR.w2 - sL.w2);
			bb1 = isum * k1;
			bb2 = isum * k2;
			vb2 = s_mid * bx + v1 * bb1 + v2 * bb2;
			const double rs = us[0];
			u2[0] = rs;
			u2[1] = us[1];
			u2[2] = rs * v1;
			u2[3] = rs * v2;
			u2[4] = left ? uL[4] - sqL * sgn * (sL.vb - vb2) * g.inv_sqrt_mu0
			             : uR[4] + sqR * sgn * (sR.vb - vb2) * g.inv_sqrt_mu0;
			u2[5] = bx;
			u2[6] = bb1;
			u2[7] = bb2;
		}
		if (F != nullptr) {
			phys_forward(S, g, F);
			for (int v = 0; v < 8; v++) F[v] = F[v] + u2[v] * ss - us[v] * (ss - s) - US[v] * s;
			F[5] = 0.0;
		}
		double ph[8];
		for (int v = 0; v < 8; v++) ph[v] = v == 5 ? 0.0 : phi[v];
		double a_u2[8], a_ss = 0.0, a_s = 0.0, dU[8];
		for (int v = 0; v < 8; v++) {
			a_u2[v] = ss * ph[v];
			a_us[v] += -(ss - s) * ph[v];
			dU[v] = -s * ph[v];
			a_ss += (u2[v] - us[v]) * ph[v];
			a_s += (us[v] - US[v]) * ph[v];
		}
		add_state(A, dU);
		phys_reverse(S, g, ph, A);
		if (left) { a_ssL += a_ss; a_sneg += a_s; } else { a_ssR += a_ss; a_spos += a_s; }
		if (not dstar) {
			for (int v = 0; v < 8; v++) a_us[v] += a_u2[v];
		} else {
			const double rs = us[0];
			// u2 = [rs, us1, rs v1, rs v2, E2, bx, bb1, bb2]
			a_us[0] += a_u2[0] + v1 * a_u2[2] + v2 * a_u2[3];
			a_us[1] += a_u2[1];
			double a_v1 = rs * a_u2[2], a_v2 = rs * a_u2[3];
			a_bx += a_u2[5];
			double a_bb1 = a_u2[6], a_bb2 = a_u2[7];
			double a_vb2 = 0.0, a_sq = 0.0, a_sgnvb = 0.0;
			// E2 = E* -/+ sq sgn (vb* - vb2) / sqrt(mu0)
			const double sq = left ? sqL : sqR;
			const double vbs = left ? sL.vb : sR.vb;
			const double pm = left ? -1.0 : 1.0;
			a_us[4] += a_u2[4];
			a_sq = pm * sgn * (vbs - vb2) * g.inv_sqrt_mu0 * a_u2[4];
			a_sgnvb = pm * sq * sgn * g.inv_sqrt_mu0 * a_u2[4];
			if (left) a_vbL += a_sgnvb; else a_vbR += a_sgnvb;
			a_vb2 += -a_sgnvb;
			if (left) a_sqL += a_sq; else a_sqR += a_sq;
			// vb2 = s_mid bx + v1 bb1 + v2 bb2
			a_smid += bx * a_vb2;
			a_bx += s_mid * a_vb2;
			a_v1 += bb1 * a_vb2;
			a_v2 += bb2 * a_vb2;
			a_bb1 += v1 * a_vb2;
			a_bb2 += v2 * a_vb2;
			// bb = isum k, v = isum n
			double a_isum = k1 * a_bb1 + k2 * a_bb2 + n1 * a_v1 + n2 * a_v2;
			const double a_k1 = isum * a_bb1, a_k2 = isum * a_bb2;
			const double a_n1 = isum * a_v1, a_n2 = isum * a_v2;
			// k = (sqL sbR + sqR sbL) + wb (wR - wL)
			a_sqL += sR.sb1 * a_k1 + sR.sb2 * a_k2;
			a_sqR += sL.sb1 * a_k1 + sL.sb2 * a_k2;
			a_sb1R += sqL * a_k1;
			a_sb2R += sqL * a_k2;
			a_sb1L += sqR * a_k1;
			a_sb2L += sqR * a_k2;
			const double a_wb = (sR.w1 - sL.w1) * a_k1 + (sR.w2 - sL.w2) * a_k2;
			a_w1R += wb * a_k1;
			a_w2R += wb * a_k2;
			a_w1L += -wb * a_k1;
			a_w2L += -wb * a_k2;
			// wb = sgn sqL sqR sqrt(mu0)
			a_sqL += sgn * sqR * g.sqrt_mu0 * a_wb;
			a_sqR += sgn * sqL * g.sqrt_mu0 * a_wb;
			// n = (sqL wL + sqR wR) + cv (sbR - sbL)
			a_sqL += sL.w1 * a_n1 + sL.w2 * a_n2;
			a_sqR += sR.w1 * a_n1 + sR.w2 * a_n2;
			a_w1L += sqL * a_n1;
			a_w2L += sqL * a_n2;
			a_w1R += sqR * a_n1;
			a_w2R += sqR * a_n2;
			a_sb1R += cv * a_n1;
			a_sb2R += cv * a_n2;
			a_sb1L += -cv * a_n1;
			a_sb2L += -cv * a_n2;
			// isum = 1 / (sqL + sqR)
			const double a_sumsq = -isum * isum * a_isum;
			a_sqL += a_sumsq;
			a_sqR += a_sumsq;
		}
	}

	// star states: u* = [rs, rs s_mid, rs w1, rs w2, E*, bx, sb1, sb2]
	auto star_rev = [&](const Side_Fwd& S, Side_Adj& A, const Star& st, const double pt, const double* a_u,
	                    double& a_w1, double& a_w2, double& a_sb1, double& a_sb2, double& a_vb, double& a_sd,
	                    double& a_sm, double& a_rs, double& a_pt) {
		a_rs += a_u[0] + s_mid * a_u[1] + st.w1 * a_u[2] + st.w2 * a_u[3];
		a_smid += st.rs * a_u[1];
		a_w1 += st.rs * a_u[2];
		a_w2 += st.rs * a_u[3];
		a_bx += a_u[5];
		a_sb1 += a_u[6];
		a_sb2 += a_u[7];
		// E* = num_e / sm
		const double a_num_e = a_u[4] * st.ism;
		a_sm += -st.Es * st.ism * a_u[4];
		// num_e = sd E - pt v0 + ptst s_mid + bx/mu0 (vb_old - vb)
		a_sd += S.E * a_num_e;
		A.E += st.sd * a_num_e;
		a_pt += -S.v0 * a_num_e;
		A.v0 += -pt * a_num_e;
		a_ptst += s_mid * a_num_e;
		a_smid += ptst * a_num_e;
		a_bx += im * (st.vb_old - st.vb) * a_num_e;
		const double a_vb_old = bx * im * a_num_e;
		a_vb += -bx * im * a_num_e;
		// vb_old = v . b
		A.v0 += S.b0 * a_vb_old; A.v1 += S.b1 * a_vb_old; A.v2 += S.b2 * a_vb_old;
		A.b0 += S.v0 * a_vb_old; A.b1 += S.v1 * a_vb_old; A.b2 += S.v2 * a_vb_old;
		// vb = s_mid bx + w1 sb1 + w2 sb2
		a_smid += bx * a_vb;
		a_bx += s_mid * a_vb;
		a_w1 += st.sb1 * a_vb;
		a_w2 += st.sb2 * a_vb;
		a_sb1 += st.w1 * a_vb;
		a_sb2 += st.w2 * a_vb;
		if (st.degenerate) {
			A.v1 += a_w1; A.v2 += a_w2; A.b1 += a_sb1; A.b2 += a_sb2;
		} else {
			// w = v - b t1, sb = b t2
			A.v1 += a_w1; A.v2 += a_w2;
			A.b1 += -st.t1 * a_w1 + st.t2 * a_sb1;
			A.b2 += -st.t1 * a_w2 + st.t2 * a_sb2;
			const double a_t1 = -S.b1 * a_w1 - S.b2 * a_w2;
			const double a_t2 = S.b1 * a_sb1 + S.b2 * a_sb2;
			// t1 = bx (s_mid - v0) / mu0 / tmp, t2 = (rho sd^2 - bx2m) / tmp
			const double a_tmp = -(st.t1 * a_t1 + st.t2 * a_t2) * st.itmp;
			const double c1 = im * st.itmp * a_t1, c2 = st.itmp * a_t2;
			a_bx += (s_mid - S.v0) * c1;
			a_smid += bx * c1;
			A.v0 += -bx * c1;
			A.rho += st.sd * st.sd * c2;
			a_sd += 2.0 * S.rho * st.sd * c2;
			double a_bx2m = -c2;
			// tmp = rho sd sm - bx2m
			A.rho += st.sd * st.sm * a_tmp;
			a_sd += S.rho * st.sm * a_tmp;
			a_sm += S.rho * st.sd * a_tmp;
			a_bx2m += -a_tmp;
			a_bx += 2.0 * bx * im * a_bx2m;
		}
	};
	double a_sdL = 0.0, a_smL = 0.0, a_rsL = 0.0, a_ptL = 0.0;
	double a_sdR = 0.0, a_smR = 0.0, a_rsR = 0.0, a_ptR = 0.0;
	star_rev(R, AR, sR, ptR, a_uR, a_w1R, a_w2R, a_sb1R, a_sb2R, a_vbR, a_sdR, a_smR, a_rsR, a_ptR);
	star_rev(L, AL, sL, ptL, a_uL, a_w1L, a_w2L, a_sb1L, a_sb2L, a_vbL, a_sdL, a_smL, a_rsL, a_ptL);

	// ptst = ptL + rhoL sdL (s_mid - vL0)
	a_ptL += a_ptst;
	AL.rho += sL.sd * (s_mid - L.v0) * a_ptst;
	a_sdL += L.rho * (s_mid - L.v0) * a_ptst;
	a_smid += L.rho * sL.sd * a_ptst;
	AL.v0 += -L.rho * sL.sd * a_ptst;
	// ssL = s_mid - abx / sqL, ssR = s_mid + abx / sqR, abx = |bx| / sqrt(mu0)
	a_smid += a_ssL + a_ssR;
	const double a_abx = -a_ssL * isqL + a_ssR * isqR;
	a_sqL += abx * isqL * isqL * a_ssL;
	a_sqR += -abx * isqR * isqR * a_ssR;
	a_bx += abs_rev(bx, g.inv_sqrt_mu0 * a_abx);
	// sq = sqrt(rs)
	a_rsL += 0.5 * isqL * a_sqL;
	a_rsR += 0.5 * isqR * a_sqR;
	// rs = rho sd / sm
	AL.rho += sL.sd * sL.ism * a_rsL;
	a_sdL += L.rho * sL.ism * a_rsL;
	a_smL += -sL.rs * sL.ism * a_rsL;
	AR.rho += sR.sd * sR.ism * a_rsR;
	a_sdR += R.rho * sR.ism * a_rsR;
	a_smR += -sR.rs * sR.ism * a_rsR;
	// sm = s - s_mid
	a_sneg += a_smL;
	a_spos += a_smR;
	a_smid += -a_smL - a_smR;
	// s_mid = num / den
	const double a_num = a_smid * iden;
	const double a_den = -s_mid * iden * a_smid;
	// num = sdR mR0 - sdL mL0 - ptR + ptL, den = sdR rhoR - sdL rhoL
	a_sdR += R.m0 * a_num + R.rho * a_den;
	a_sdL += -L.m0 * a_num - L.rho * a_den;
	AR.m0 += sR.sd * a_num;
	AL.m0 += -sL.sd * a_num;
	a_ptR += -a_num;
	a_ptL += a_num;
	AR.rho += sR.sd * a_den;
	AL.rho += -sL.sd * a_den;
	// sd = s - v0
	a_sneg += a_sdL;
	AL.v0 += -a_sdL;
	a_spos += a_sdR;
	AR.v0 += -a_sdR;
	// pt = p + pb
	AL.p += a_ptL; AL.pb += a_ptL;
	AR.p += a_ptR; AR.pb += a_ptR;
	// bx = (bL0 + bR0) / 2
	AL.b0 += 0.5 * a_bx;
	AR.b0 += 0.5 * a_bx;
	// s_neg = min(vL0, vR0) - fast, s_pos = max(vL0, vR0) + fast, fast = max(cfL, cfR)
	max_rev(L.v0, R.v0, a_spos, AL.v0, AR.v0);
	max_rev(R.v0, L.v0, a_sneg, AL.v0, AR.v0);
	max_rev(L.cf, R.cf, -a_sneg + a_spos, AL.cf, AR.cf);
	side_reverse(L, AL, g, gL);
	side_reverse(R, AR, g, gR);
}

// ---------------------------------------------------------------- Roe

/*
Roe solver for adiabatic MHD (flux_roe of mhd_device.cuh: Athena's
esys_roe_adb_mhd and fluxes, mhd/roe_athena.hpp:56-559, the eigensystem of
eqns B17-B29 of Stone et al., ApJS 178, 2008), in units where the field is
B / sqrt(mu0).  Forward, then reverse: through the flux of the upwind side
(supersonic fans) or through F = (F_L + F_R)/2 - sum_m a_m |ev_m| R_m / 2,
a = L (U_R - U_L), back through the 7 x 7 right and left eigenvectors, the
eigenvalues and the Roe averages to the two states.  Kinks: |ev_m| at 0
(abs_rev), the floor of twid_asq (max_rev), the branches of alpha_f and
alpha_s and of the transverse field direction (bt = 0) taken as evaluated.
The positivity check of the intermediate states only raises flags: it has
no derivative.
*/
__host__ __device__ __forceinline__ void roe_vjp(const double* UL, const double* UR, const Gas_Adj& g,
                                                 const double* phi, double* gL, double* gR, double* F = nullptr)
{
	constexpr double eps = 2.220446049250313080847e-16;
	Side_Fwd L, R;
	side_forward(UL, g, L);
	side_forward(UR, g, R);
	Side_Adj AL, AR;
	side_adj_zero(AL);
	side_adj_zero(AR);
	const double gm1 = g.gamma - 1.0, gm2 = g.gamma - 2.0, igm1 = rcp(gm1);
	const double ism = g.inv_sqrt_mu0;

	// ---- forward: Roe averages (roe_athena.hpp:575-760)
	const double bxi = 0.5 * (L.b0 + R.b0) * ism;
	const double byl = L.b1 * ism, bzl = L.b2 * ism, byr = R.b1 * ism, bzr = R.b2 * ism;
	// pressure with mu0 = 1, as the reference's get_primitive call
	const double pl = (L.E - 0.5 * L.r * L.m2s - 0.5 * L.b2s) * gm1;
	const double pr = (R.E - 0.5 * R.r * R.m2s - 0.5 * R.b2s) * gm1;
	const double sdl = sqrt(L.rho), sdr = sqrt(R.rho);
	const double isdl = rcp(sdl), isdr = rcp(sdr);
	const double isd = rcp(sdl + sdr);
	const double droe = sdl * sdr;
	const double di = rcp(droe);
	const double v1 = (sdl * L.v0 + sdr * R.v0) * isd;
	const double v2 = (sdl * L.v1 + sdr * R.v1) * isd;
	const double v3 = (sdl * L.v2 + sdr * R.v2) * isd;
	const double b2 = (sdr * byl + sdl * byr) * isd;
	const double b3 = (sdr * bzl + sdl * bzr) * isd;
	const double dby = byl - byr, dbz = bzl - bzr;
	const double x = 0.5 * (dby * dby + dbz * dbz) * (isd * isd);
	const double y = 0.5 * (L.rho + R.rho) * di;
	const double pbl = 0.5 * (bxi * bxi + byl * byl + bzl * bzl);
	const double pbr = 0.5 * (bxi * bxi + byr * byr + bzr * bzr);
	const double hl = (L.E + pl + pbl) * isdl, hr = (R.E + pr + pbr) * isdr;
	const double h = (hl + hr) * isd;
	const double b1 = bxi;
	// eigensystem (B17-B29)
	const double vsq = v1 * v1 + v2 * v2 + v3 * v3;
	const double btsq = b2 * b2 + b3 * b3;
	const double ystar = gm1 - gm2 * y;
	const double bt_starsq = ystar * btsq;
	const double vaxsq = b1 * b1 * di;
	const double hp = h - (vaxsq + btsq * di);
	const double twid_raw = gm1 * (hp - 0.5 * vsq) - gm2 * x;
	const double twid_asq = fmax(twid_raw, eps);
	const double ct2 = bt_starsq * di;
	const double tsum = vaxsq + ct2 + twid_asq;
	const double tdif = vaxsq + ct2 - twid_asq;
	const double cf2_cs2 = sqrt(tdif * tdif + 4.0 * twid_asq * ct2);
	const double cfsq = 0.5 * (tsum + cf2_cs2);
	const double cf = sqrt(cfsq);
	const double icfsq = rcp(cfsq);
	const double cssq = twid_asq * vaxsq * icfsq;
	const double cs = sqrt(cssq);
	const double bt = sqrt(btsq);
	const double bt_star = sqrt(bt_starsq);
	const bool has_bt = bt != 0.0;
	const double ibt = has_bt ? rcp(bt) : 0.0;
	const double bet2 = has_bt ? b2 * ibt : 1.0, bet3 = has_bt ? b3 * ibt : 0.0;
	const double iys = rcp(sqrt(ystar));
	const double bet2_star = bet2 * iys, bet3_star = bet3 * iys;
	const double bet_starsq = bet2_star * bet2_star + bet3_star * bet3_star;
	const double vbet = v2 * bet2_star + v3 * bet3_star;
	int acase;
	double alpha_f, alpha_s, aid = 0.0, ra = 0.0, rb = 0.0;
	if ((cfsq - cssq) == 0.0) {
		acase = 0; alpha_f = 1.0; alpha_s = 0.0;
	} else if ((twid_asq - cssq) <= 0.0) {
		acase = 1; alpha_f = 0.0; alpha_s = 1.0;
	} else if ((cfsq - twid_asq) <= 0.0) {
		acase = 2; alpha_f = 1.0; alpha_s = 0.0;
	} else {
		acase = 3;
		aid = rcp(cfsq - cssq);
		ra = (twid_asq - cssq) * aid;
		rb = (cfsq - twid_asq) * aid;
		alpha_f = sqrt(ra);
		alpha_s = sqrt(rb);
	}
	const double sqrtd = sqrt(droe);
	const double isqrtd = rcp(sqrtd);
	const double sg = (b1 > 0.0) ? 1.0 : -1.0;
	const double twid_a = sqrt(twid_asq);
	const double qf = cf * alpha_f * sg, qs = cs * alpha_s * sg;
	const double af_prime = twid_a * alpha_f * isqrtd, as_prime = twid_a * alpha_s * isqrtd;
	const double afpbb = af_prime * bt_star * bet_starsq, aspbb = as_prime * bt_star * bet_starsq;
	const double vax = sqrt(vaxsq);
	const double ev[7] = {v1 - cf, v1 - vax, v1 - cs, v1, v1 + cs, v1 + vax, v1 + cf};

	// both states and their fluxes in units B / sqrt(mu0)
	const double Ul[7] = {L.rho, L.m0, L.m1, L.m2, L.E, byl, bzl};
	const double Ur[7] = {R.rho, R.m0, R.m1, R.m2, R.E, byr, bzr};
	auto flux7 = [&](const Side_Fwd& S, const double p, const double pb, const double by, const double bz,
	                 double* Fs) {
		Fs[0] = S.m0;
		Fs[1] = S.m0 * S.v0 + p - 0.5 * (bxi * bxi - by * by - bz * bz);
		Fs[2] = S.m0 * S.v1 - bxi * by;
		Fs[3] = S.m0 * S.v2 - bxi * bz;
		Fs[4] = (S.E + p) * S.v0 + pb * S.v0 - bxi * (bxi * S.v0 + by * S.v1 + bz * S.v2);
		Fs[5] = by * S.v0 - bxi * S.v1;
		Fs[6] = bz * S.v0 - bxi * S.v2;
	};
	double Fl[7], Fr[7];
	flux7(L, pl, pbl, byl, bzl, Fl);
	flux7(R, pr, pbr, byr, bzr, Fr);

	// adjoint of the 7-component flux
	const double aFo[7] = {phi[0], phi[1], phi[2], phi[3], phi[4], phi[6] * g.sqrt_mu0, phi[7] * g.sqrt_mu0};
	double aFl[7] = {0, 0, 0, 0, 0, 0, 0}, aFr[7] = {0, 0, 0, 0, 0, 0, 0};
	double aUl[7] = {0, 0, 0, 0, 0, 0, 0}, aUr[7] = {0, 0, 0, 0, 0, 0, 0};
	// adjoints of the averages and of the eigensystem's scalars
	double a_v1 = 0, a_v2 = 0, a_v3 = 0, a_b2 = 0, a_b3 = 0, a_x = 0, a_hp = 0, a_vsq = 0, a_cf = 0, a_cs = 0;
	double a_af = 0, a_as = 0, a_qf = 0, a_qs = 0, a_bet2 = 0, a_bet3 = 0, a_b2s = 0, a_b3s = 0, a_vbet = 0;
	double a_afp = 0, a_asp = 0, a_afpbb = 0, a_aspbb = 0, a_isqrtd = 0, a_sqrtd = 0, a_droe = 0, a_vax = 0;
	double a_bt_star = 0, a_bsq = 0, a_twid = 0;
	double Fo[7];

	if (ev[0] >= 0.0) {
		for (int r = 0; r < 7; r++) { Fo[r] = Fl[r]; aFl[r] = aFo[r]; }
	} else if (ev[6] <= 0.0) {
		for (int r = 0; r < 7; r++) { Fo[r] = Fr[r]; aFr[r] = aFo[r]; }
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
		const double wv = v2 * bet3 - v3 * bet2;
		Rm[4][0] = alpha_f * (hp - v1 * cf) + qs * vbet + aspbb;
		Rm[4][1] = -wv;
		Rm[4][2] = alpha_s * (hp - v1 * cs) - qf * vbet - afpbb;
		Rm[4][3] = 0.5 * vsq + gm2 * x * igm1;
		Rm[4][4] = alpha_s * (hp + v1 * cs) + qf * vbet - afpbb;
		Rm[4][5] = wv;
		Rm[4][6] = alpha_f * (hp + v1 * cf) - qs * vbet + aspbb;
		Rm[5][0] = as_prime * bet2_star; Rm[5][1] = -bet3 * sg * isqrtd; Rm[5][2] = -af_prime * bet2_star;
		Rm[5][3] = 0.0; Rm[5][4] = Rm[5][2]; Rm[5][5] = Rm[5][1]; Rm[5][6] = Rm[5][0];
		Rm[6][0] = as_prime * bet3_star; Rm[6][1] = bet2 * sg * isqrtd; Rm[6][2] = -af_prime * bet3_star;
		Rm[6][3] = 0.0; Rm[6][4] = Rm[6][2]; Rm[6][5] = Rm[6][1]; Rm[6][6] = Rm[6][0];

		// left eigenvectors as rows
		const double itw = rcp(twid_asq);
		const double norm0 = 0.5 * itw;
		const double cff = norm0 * alpha_f * cf, css = norm0 * alpha_s * cs;
		const double qfn = qf * norm0, qsn = qs * norm0;
		const double afd = norm0 * af_prime * droe, asd = norm0 * as_prime * droe;
		const double afpb = norm0 * af_prime * bt_star, aspb = norm0 * as_prime * bt_star;
		const double norm1 = norm0 * gm1;
		const double af_n = alpha_f * norm1, as_n = alpha_s * norm1;
		const double ibs = rcp(bet_starsq);
		const double q2s = bet2_star * ibs, q3s = bet3_star * ibs;
		const double vqstr = v2 * q2s + v3 * q3s;
		const double norm2 = norm1 * 2.0;
		double Lm[7][7];
		Lm[0][0] = af_n * (vsq - hp) + cff * (cf + v1) - qsn * vqstr - aspb;
		Lm[0][1] = -af_n * v1 - cff;
		Lm[0][2] = -af_n * v2 + qsn * q2s;
		Lm[0][3] = -af_n * v3 + qsn * q3s;
		Lm[0][4] = af_n;
		Lm[0][5] = asd * q2s - af_n * b2;
		Lm[0][6] = asd * q3s - af_n * b3;
		Lm[1][0] = 0.5 * wv; Lm[1][1] = 0.0; Lm[1][2] = -0.5 * bet3;
		Lm[1][3] = 0.5 * bet2; Lm[1][4] = 0.0; Lm[1][5] = -0.5 * sqrtd * bet3 * sg;
		Lm[1][6] = 0.5 * sqrtd * bet2 * sg;
		Lm[2][0] = as_n * (vsq - hp) + css * (cs + v1) + qfn * vqstr + afpb;
		Lm[2][1] = -as_n * v1 - css;
		Lm[2][2] = -as_n * v2 - qfn * q2s;
		Lm[2][3] = -as_n * v3 - qfn * q3s;
		Lm[2][4] = as_n;
		Lm[2][5] = -afd * q2s - as_n * b2;
		Lm[2][6] = -afd * q3s - as_n * b3;
		Lm[3][0] = 1.0 - norm2 * (0.5 * vsq - gm2 * x * igm1);
		Lm[3][1] = norm2 * v1; Lm[3][2] = norm2 * v2; Lm[3][3] = norm2 * v3;
		Lm[3][4] = -norm2; Lm[3][5] = norm2 * b2; Lm[3][6] = norm2 * b3;
		Lm[4][0] = as_n * (vsq - hp) + css * (cs - v1) - qfn * vqstr + afpb;
		Lm[4][1] = -as_n * v1 + css;
		Lm[4][2] = -as_n * v2 + qfn * q2s;
		Lm[4][3] = -as_n * v3 + qfn * q3s;
		Lm[4][4] = as_n;
		Lm[4][5] = Lm[2][5];
		Lm[4][6] = Lm[2][6];
		Lm[5][0] = -Lm[1][0]; Lm[5][1] = 0.0; Lm[5][2] = -Lm[1][2]; Lm[5][3] = -Lm[1][3];
		Lm[5][4] = 0.0; Lm[5][5] = Lm[1][5]; Lm[5][6] = Lm[1][6];
		Lm[6][0] = af_n * (vsq - hp) + cff * (cf - v1) + qsn * vqstr - aspb;
		Lm[6][1] = -af_n * v1 + cff;
		Lm[6][2] = -af_n * v2 - qsn * q2s;
		Lm[6][3] = -af_n * v3 - qsn * q3s;
		Lm[6][4] = af_n;
		Lm[6][5] = Lm[0][5];
		Lm[6][6] = Lm[0][6];

		double a[7], dU[7];
		for (int m = 0; m < 7; m++) dU[m] = Ur[m] - Ul[m];
		for (int n = 0; n < 7; n++) {
			double t = 0.0;
			for (int m = 0; m < 7; m++) t += Lm[n][m] * dU[m];
			a[n] = t;
		}
		double c[7];
		for (int r = 0; r < 7; r++) Fo[r] = 0.5 * (Fl[r] + Fr[r]);
		for (int m = 0; m < 7; m++) {
			c[m] = 0.5 * a[m] * fabs(ev[m]);
			for (int r = 0; r < 7; r++) Fo[r] -= c[m] * Rm[r][m];
		}

		// ---- reverse of the projection: Fo = (Fl + Fr)/2 - sum_m c_m R[:, m], c_m = a_m |ev_m| / 2
		double aR[7][7], aL[7][7], a_a[7], a_ev[7];
		for (int r = 0; r < 7; r++) {
			aFl[r] += 0.5 * aFo[r];
			aFr[r] += 0.5 * aFo[r];
		}
		for (int m = 0; m < 7; m++) {
			double a_c = 0.0;
			for (int r = 0; r < 7; r++) {
				a_c -= aFo[r] * Rm[r][m];
				aR[r][m] = -c[m] * aFo[r];
			}
			a_a[m] = 0.5 * fabs(ev[m]) * a_c;
			a_ev[m] = abs_rev(ev[m], 0.5 * a[m] * a_c);
		}
		// a = L dU
		for (int m = 0; m < 7; m++) {
			double t = 0.0;
			for (int n = 0; n < 7; n++) {
				aL[n][m] = a_a[n] * dU[m];
				t += Lm[n][m] * a_a[n];
			}
			aUr[m] += t;
			aUl[m] -= t;
		}
		// entries of L defined as others
		aL[2][5] += aL[4][5]; aL[2][6] += aL[4][6];
		aL[0][5] += aL[6][5]; aL[0][6] += aL[6][6];
		aL[1][0] -= aL[5][0]; aL[1][2] -= aL[5][2]; aL[1][3] -= aL[5][3];
		aL[1][5] += aL[5][5]; aL[1][6] += aL[5][6];
		double a_af_n = 0, a_as_n = 0, a_cff = 0, a_css = 0, a_qsn = 0, a_qfn = 0, a_vqstr = 0;
		double a_aspb = 0, a_afpb = 0, a_asd = 0, a_afd = 0, a_q2s = 0, a_q3s = 0, a_norm2 = 0, a_wv = 0;
		// rows 0 and 6 (fast waves), 2 and 4 (slow waves): X (vsq - hp) + Y (c +/- v1) +/- Q vqstr +/- P
		auto wave_row0 = [&](const double* A, const double sgn_c, const double sgn_q, const double sgn_p,
		                     const double n_, const double cc, const double c_, const double qn, const double* row,
		                     double& a_n_, double& a_cc, double& a_c_, double& a_qn, double& a_p) {
			a_n_ += (vsq - hp) * A[0];
			a_vsq += n_ * A[0];
			a_hp -= n_ * A[0];
			a_cc += (c_ + sgn_c * v1) * A[0];
			a_c_ += cc * A[0];
			a_v1 += sgn_c * cc * A[0];
			a_qn += sgn_q * vqstr * A[0];
			a_vqstr += sgn_q * qn * A[0];
			a_p += sgn_p * A[0];
			(void)row;
		};
		// row 0: af_n (vsq - hp) + cff (cf + v1) - qsn vqstr - aspb
		wave_row0(aL[0], 1.0, -1.0, -1.0, af_n, cff, cf, qsn, Lm[0], a_af_n, a_cff, a_cf, a_qsn, a_aspb);
		// row 6: af_n (vsq - hp) + cff (cf - v1) + qsn vqstr - aspb
		wave_row0(aL[6], -1.0, 1.0, -1.0, af_n, cff, cf, qsn, Lm[6], a_af_n, a_cff, a_cf, a_qsn, a_aspb);
		// row 2: as_n (vsq - hp) + css (cs + v1) + qfn vqstr + afpb
		wave_row0(aL[2], 1.0, 1.0, 1.0, as_n, css, cs, qfn, Lm[2], a_as_n, a_css, a_cs, a_qfn, a_afpb);
		// row 4: as_n (vsq - hp) + css (cs - v1) - qfn vqstr + afpb
		wave_row0(aL[4], -1.0, -1.0, 1.0, as_n, css, cs, qfn, Lm[4], a_as_n, a_css, a_cs, a_qfn, a_afpb);
		// columns 1..4 of rows 0, 6: -af_n v -/+ ..., row 0: -cff, +qsn q; row 6: +cff, -qsn q
		a_af_n += -v1 * aL[0][1] - v2 * aL[0][2] - v3 * aL[0][3] + aL[0][4];
		a_af_n += -v1 * aL[6][1] - v2 * aL[6][2] - v3 * aL[6][3] + aL[6][4];
		a_v1 += -af_n * (aL[0][1] + aL[6][1]);
		a_v2 += -af_n * (aL[0][2] + aL[6][2]);
		a_v3 += -af_n * (aL[0][3] + aL[6][3]);
		a_cff += -aL[0][1] + aL[6][1];
		a_qsn += q2s * (aL[0][2] - aL[6][2]) + q3s * (aL[0][3] - aL[6][3]);
		a_q2s += qsn * (aL[0][2] - aL[6][2]);
		a_q3s += qsn * (aL[0][3] - aL[6][3]);
		// rows 2, 4: -as_n v -/+ ..., row 2: -css, -qfn q; row 4: +css, +qfn q
		a_as_n += -v1 * aL[2][1] - v2 * aL[2][2] - v3 * aL[2][3] + aL[2][4];
		a_as_n += -v1 * aL[4][1] - v2 * aL[4][2] - v3 * aL[4][3] + aL[4][4];
		a_v1 += -as_n * (aL[2][1] + aL[4][1]);
		a_v2 += -as_n * (aL[2][2] + aL[4][2]);
		a_v3 += -as_n * (aL[2][3] + aL[4][3]);
		a_css += -aL[2][1] + aL[4][1];
		a_qfn += q2s * (-aL[2][2] + aL[4][2]) + q3s * (-aL[2][3] + aL[4][3]);
		a_q2s += qfn * (-aL[2][2] + aL[4][2]);
		a_q3s += qfn * (-aL[2][3] + aL[4][3]);
		// columns 5, 6: row 0 asd q - af_n b, row 2 -afd q - as_n b
		a_asd += q2s * aL[0][5] + q3s * aL[0][6];
		a_q2s += asd * aL[0][5] - afd * aL[2][5];
		a_q3s += asd * aL[0][6] - afd * aL[2][6];
		a_af_n += -b2 * aL[0][5] - b3 * aL[0][6];
		a_b2 += -af_n * aL[0][5] - as_n * aL[2][5];
		a_b3 += -af_n * aL[0][6] - as_n * aL[2][6];
		a_afd += -q2s * aL[2][5] - q3s * aL[2][6];
		a_as_n += -b2 * aL[2][5] - b3 * aL[2][6];
		// row 1: 0.5 wv, -0.5 bet3, 0.5 bet2, -0.5 sqrtd bet3 sg, 0.5 sqrtd bet2 sg
		a_wv += 0.5 * aL[1][0];
		a_bet3 += -0.5 * aL[1][2] - 0.5 * sqrtd * sg * aL[1][5];
		a_bet2 += 0.5 * aL[1][3] + 0.5 * sqrtd * sg * aL[1][6];
		a_sqrtd += 0.5 * sg * (-bet3 * aL[1][5] + bet2 * aL[1][6]);
		// row 3: 1 - norm2 (vsq / 2 - gm2 x / gm1), norm2 (v1, v2, v3, -1, b2, b3)
		a_norm2 += -(0.5 * vsq - gm2 * x * igm1) * aL[3][0]
		           + v1 * aL[3][1] + v2 * aL[3][2] + v3 * aL[3][3] - aL[3][4] + b2 * aL[3][5] + b3 * aL[3][6];
		a_vsq += -0.5 * norm2 * aL[3][0];
		a_x += norm2 * gm2 * igm1 * aL[3][0];
		a_v1 += norm2 * aL[3][1];
		a_v2 += norm2 * aL[3][2];
		a_v3 += norm2 * aL[3][3];
		a_b2 += norm2 * aL[3][5];
		a_b3 += norm2 * aL[3][6];
		// the left eigenvectors' scalars
		double a_norm1 = 2.0 * a_norm2, a_norm0 = 0.0;
		a_v2 += q2s * a_vqstr;
		a_v3 += q3s * a_vqstr;
		a_q2s += v2 * a_vqstr;
		a_q3s += v3 * a_vqstr;
		const double a_ibs = bet2_star * a_q2s + bet3_star * a_q3s;
		a_b2s += ibs * a_q2s;
		a_b3s += ibs * a_q3s;
		a_bsq += -ibs * ibs * a_ibs;
		a_af += norm1 * a_af_n;
		a_as += norm1 * a_as_n;
		a_norm1 += alpha_f * a_af_n + alpha_s * a_as_n;
		a_norm0 += gm1 * a_norm1;
		a_norm0 += af_prime * bt_star * a_afpb + as_prime * bt_star * a_aspb;
		a_afp += norm0 * bt_star * a_afpb;
		a_asp += norm0 * bt_star * a_aspb;
		a_bt_star += norm0 * (af_prime * a_afpb + as_prime * a_aspb);
		a_norm0 += af_prime * droe * a_afd + as_prime * droe * a_asd;
		a_afp += norm0 * droe * a_afd;
		a_asp += norm0 * droe * a_asd;
		a_droe += norm0 * (af_prime * a_afd + as_prime * a_asd);
		a_qf += norm0 * a_qfn;
		a_qs += norm0 * a_qsn;
		a_norm0 += qf * a_qfn + qs * a_qsn;
		a_norm0 += alpha_f * cf * a_cff + alpha_s * cs * a_css;
		a_af += norm0 * cf * a_cff;
		a_cf += norm0 * alpha_f * a_cff;
		a_as += norm0 * cs * a_css;
		a_cs += norm0 * alpha_s * a_css;
		a_twid += -0.5 * itw * itw * a_norm0;

		// ---- reverse of the right eigenvectors
		a_af += aR[0][0] + aR[0][6];
		a_as += aR[0][2] + aR[0][4];
		a_af += ev[0] * aR[1][0] + ev[6] * aR[1][6];
		a_as += ev[2] * aR[1][2] + ev[4] * aR[1][4];
		a_ev[0] += alpha_f * aR[1][0];
		a_ev[6] += alpha_f * aR[1][6];
		a_ev[2] += alpha_s * aR[1][2];
		a_ev[4] += alpha_s * aR[1][4];
		a_v1 += aR[1][3];
		{
			// row 2: qa + qc, -bet3, qb - qd, v2, qb + qd, bet3, qa - qc
			const double a_qa = aR[2][0] + aR[2][6], a_qc = aR[2][0] - aR[2][6];
			const double a_qb = aR[2][2] + aR[2][4], a_qd = -aR[2][2] + aR[2][4];
			a_bet3 += -aR[2][1] + aR[2][5];
			a_v2 += aR[2][3] + alpha_f * a_qa + alpha_s * a_qb;
			a_af += v2 * a_qa;
			a_as += v2 * a_qb;
			a_qs += bet2_star * a_qc;
			a_qf += bet2_star * a_qd;
			a_b2s += qs * a_qc + qf * a_qd;
		}
		{
			// row 3: qa + qc, bet2, qb - qd, v3, qb + qd, -bet2, qa - qc
			const double a_qa = aR[3][0] + aR[3][6], a_qc = aR[3][0] - aR[3][6];
			const double a_qb = aR[3][2] + aR[3][4], a_qd = -aR[3][2] + aR[3][4];
			a_bet2 += aR[3][1] - aR[3][5];
			a_v3 += aR[3][3] + alpha_f * a_qa + alpha_s * a_qb;
			a_af += v3 * a_qa;
			a_as += v3 * a_qb;
			a_qs += bet3_star * a_qc;
			a_qf += bet3_star * a_qd;
			a_b3s += qs * a_qc + qf * a_qd;
		}
		// row 4
		a_af += (hp - v1 * cf) * aR[4][0] + (hp + v1 * cf) * aR[4][6];
		a_as += (hp - v1 * cs) * aR[4][2] + (hp + v1 * cs) * aR[4][4];
		a_hp += alpha_f * (aR[4][0] + aR[4][6]) + alpha_s * (aR[4][2] + aR[4][4]);
		a_v1 += alpha_f * cf * (-aR[4][0] + aR[4][6]) + alpha_s * cs * (-aR[4][2] + aR[4][4]);
		a_cf += alpha_f * v1 * (-aR[4][0] + aR[4][6]);
		a_cs += alpha_s * v1 * (-aR[4][2] + aR[4][4]);
		a_qs += vbet * (aR[4][0] - aR[4][6]);
		a_qf += vbet * (-aR[4][2] + aR[4][4]);
		a_vbet += qs * (aR[4][0] - aR[4][6]) + qf * (-aR[4][2] + aR[4][4]);
		a_aspbb += aR[4][0] + aR[4][6];
		a_afpbb += -aR[4][2] - aR[4][4];
		a_wv += -aR[4][1] + aR[4][5];
		a_vsq += 0.5 * aR[4][3];
		a_x += gm2 * igm1 * aR[4][3];
		// rows 5 and 6
		a_asp += bet2_star * (aR[5][0] + aR[5][6]) + bet3_star * (aR[6][0] + aR[6][6]);
		a_afp += -bet2_star * (aR[5][2] + aR[5][4]) - bet3_star * (aR[6][2] + aR[6][4]);
		a_b2s += as_prime * (aR[5][0] + aR[5][6]) - af_prime * (aR[5][2] + aR[5][4]);
		a_b3s += as_prime * (aR[6][0] + aR[6][6]) - af_prime * (aR[6][2] + aR[6][4]);
		a_bet3 += -sg * isqrtd * (aR[5][1] + aR[5][5]);
		a_bet2 += sg * isqrtd * (aR[6][1] + aR[6][5]);
		a_isqrtd += sg * (-bet3 * (aR[5][1] + aR[5][5]) + bet2 * (aR[6][1] + aR[6][5]));
		// wv = v2 bet3 - v3 bet2
		a_v2 += bet3 * a_wv;
		a_v3 += -bet2 * a_wv;
		a_bet3 += v2 * a_wv;
		a_bet2 += -v3 * a_wv;
		// eigenvalues
		for (int m = 0; m < 7; m++) a_v1 += a_ev[m];
		a_cf += -a_ev[0] + a_ev[6];
		a_vax += -a_ev[1] + a_ev[5];
		a_cs += -a_ev[2] + a_ev[4];
	}
	if (F != nullptr) {
		F[0] = Fo[0]; F[1] = Fo[1]; F[2] = Fo[2]; F[3] = Fo[3]; F[4] = Fo[4];
		F[5] = 0.0;
		F[6] = Fo[5] * g.sqrt_mu0;
		F[7] = Fo[6] * g.sqrt_mu0;
	}

	// ---- reverse of the eigensystem's scalars (zero outside the middle branch)
	double a_vaxsq = vax > 0.0 ? 0.5 * rcp(vax) * a_vax : 0.0;
	a_afp += bt_star * bet_starsq * a_afpbb;
	a_asp += bt_star * bet_starsq * a_aspbb;
	a_bt_star += bet_starsq * (af_prime * a_afpbb + as_prime * a_aspbb);
	a_bsq += bt_star * (af_prime * a_afpbb + as_prime * a_aspbb);
	double a_twid_a = alpha_f * isqrtd * a_afp + alpha_s * isqrtd * a_asp;
	a_af += twid_a * isqrtd * a_afp;
	a_as += twid_a * isqrtd * a_asp;
	a_isqrtd += twid_a * (alpha_f * a_afp + alpha_s * a_asp);
	a_cf += alpha_f * sg * a_qf;
	a_af += cf * sg * a_qf;
	a_cs += alpha_s * sg * a_qs;
	a_as += cs * sg * a_qs;
	a_twid += twid_a > 0.0 ? 0.5 * rcp(twid_a) * a_twid_a : 0.0;
	a_sqrtd += -isqrtd * isqrtd * a_isqrtd;
	a_droe += 0.5 * isqrtd * a_sqrtd;
	double a_cfsq = 0.0, a_cssq = 0.0;
	if (acase == 3) {
		const double a_ra = alpha_f > 0.0 ? 0.5 * rcp(alpha_f) * a_af : 0.0;
		const double a_rb = alpha_s > 0.0 ? 0.5 * rcp(alpha_s) * a_as : 0.0;
		a_twid += aid * (a_ra - a_rb);
		a_cssq += -aid * a_ra;
		a_cfsq += aid * a_rb;
		const double a_aid = (twid_asq - cssq) * a_ra + (cfsq - twid_asq) * a_rb;
		a_cfsq += -aid * aid * a_aid;
		a_cssq += aid * aid * a_aid;
	}
	// vbet = v2 bet2* + v3 bet3*, bet_starsq = bet2*^2 + bet3*^2, bet* = bet iys
	a_v2 += bet2_star * a_vbet;
	a_v3 += bet3_star * a_vbet;
	a_b2s += v2 * a_vbet + 2.0 * bet2_star * a_bsq;
	a_b3s += v3 * a_vbet + 2.0 * bet3_star * a_bsq;
	a_bet2 += iys * a_b2s;
	a_bet3 += iys * a_b3s;
	const double a_iys = bet2 * a_b2s + bet3 * a_b3s;
	double a_ystar = -0.5 * iys * iys * iys * a_iys;
	double a_btsq = 0.0;
	if (has_bt) {
		a_b2 += ibt * a_bet2;
		a_b3 += ibt * a_bet3;
		const double a_bt = -ibt * ibt * (b2 * a_bet2 + b3 * a_bet3);
		a_btsq += 0.5 * ibt * a_bt;
	}
	double a_bt_starsq = bt_star > 0.0 ? 0.5 * rcp(bt_star) * a_bt_star : 0.0;
	a_cssq += cs > 0.0 ? 0.5 * rcp(cs) * a_cs : 0.0;
	a_twid += vaxsq * icfsq * a_cssq;
	a_vaxsq += twid_asq * icfsq * a_cssq;
	a_cfsq += -cssq * icfsq * a_cssq;
	a_cfsq += cf > 0.0 ? 0.5 * rcp(cf) * a_cf : 0.0;
	const double a_tsum = 0.5 * a_cfsq, a_cf2 = 0.5 * a_cfsq;
	const double a_q = cf2_cs2 > 0.0 ? 0.5 * rcp(cf2_cs2) * a_cf2 : 0.0;
	const double a_tdif = 2.0 * tdif * a_q;
	a_twid += 4.0 * ct2 * a_q + a_tsum - a_tdif;
	double a_ct2 = 4.0 * twid_asq * a_q + a_tsum + a_tdif;
	a_vaxsq += a_tsum + a_tdif;
	a_bt_starsq += di * a_ct2;
	double a_di = bt_starsq * a_ct2;
	// twid_asq = max(twid_raw, eps)
	double a_raw = 0.0, a_floor = 0.0;
	max_rev(twid_raw, eps, a_twid, a_raw, a_floor);
	a_hp += gm1 * a_raw;
	a_vsq += -0.5 * gm1 * a_raw;
	a_x += -gm2 * a_raw;
	// hp = h - (vaxsq + btsq di)
	double a_h = a_hp;
	a_vaxsq += -a_hp;
	a_btsq += -di * a_hp;
	a_di += -btsq * a_hp;
	// vaxsq = b1^2 di
	double a_bxi = 2.0 * b1 * di * a_vaxsq;
	a_di += b1 * b1 * a_vaxsq;
	// bt_starsq = ystar btsq, ystar = gm1 - gm2 y
	a_ystar += btsq * a_bt_starsq;
	a_btsq += ystar * a_bt_starsq;
	const double a_y = -gm2 * a_ystar;
	a_b2 += 2.0 * b2 * a_btsq;
	a_b3 += 2.0 * b3 * a_btsq;
	a_v1 += 2.0 * v1 * a_vsq;
	a_v2 += 2.0 * v2 * a_vsq;
	a_v3 += 2.0 * v3 * a_vsq;

	// ---- reverse of the Roe averages
	double a_sdl = 0.0, a_sdr = 0.0, a_isd = 0.0;
	double a_byl = 0.0, a_bzl = 0.0, a_byr = 0.0, a_bzr = 0.0, a_pl = 0.0, a_pr = 0.0, a_pbl = 0.0, a_pbr = 0.0;
	// h = (hl + hr) isd, hl = (E + p + pb) / sd
	const double a_hl = isd * a_h, a_hr = isd * a_h;
	a_isd += (hl + hr) * a_h;
	AL.E += isdl * a_hl; a_pl += isdl * a_hl; a_pbl += isdl * a_hl;
	AR.E += isdr * a_hr; a_pr += isdr * a_hr; a_pbr += isdr * a_hr;
	a_sdl += -isdl * isdl * (L.E + pl + pbl) * a_hl;
	a_sdr += -isdr * isdr * (R.E + pr + pbr) * a_hr;
	// y = (rhoL + rhoR) di / 2
	AL.rho += 0.5 * di * a_y;
	AR.rho += 0.5 * di * a_y;
	a_di += 0.5 * (L.rho + R.rho) * a_y;
	// x = (dby^2 + dbz^2) isd^2 / 2
	const double a_dby = dby * isd * isd * a_x, a_dbz = dbz * isd * isd * a_x;
	a_isd += (dby * dby + dbz * dbz) * isd * a_x;
	a_byl += a_dby; a_byr -= a_dby;
	a_bzl += a_dbz; a_bzr -= a_dbz;
	// b2 = (sdr byl + sdl byr) isd, b3 likewise
	a_sdr += (byl * a_b2 + bzl * a_b3) * isd;
	a_sdl += (byr * a_b2 + bzr * a_b3) * isd;
	a_byl += sdr * isd * a_b2;
	a_byr += sdl * isd * a_b2;
	a_bzl += sdr * isd * a_b3;
	a_bzr += sdl * isd * a_b3;
	a_isd += (sdr * byl + sdl * byr) * a_b2 + (sdr * bzl + sdl * bzr) * a_b3;
	// v = (sdl vL + sdr vR) isd
	a_sdl += (L.v0 * a_v1 + L.v1 * a_v2 + L.v2 * a_v3) * isd;
	a_sdr += (R.v0 * a_v1 + R.v1 * a_v2 + R.v2 * a_v3) * isd;
	AL.v0 += sdl * isd * a_v1; AL.v1 += sdl * isd * a_v2; AL.v2 += sdl * isd * a_v3;
	AR.v0 += sdr * isd * a_v1; AR.v1 += sdr * isd * a_v2; AR.v2 += sdr * isd * a_v3;
	a_isd += (sdl * L.v0 + sdr * R.v0) * a_v1 + (sdl * L.v1 + sdr * R.v1) * a_v2 + (sdl * L.v2 + sdr * R.v2) * a_v3;
	// di = 1 / droe, droe = sdl sdr, isd = 1 / (sdl + sdr)
	a_droe += -di * di * a_di;
	a_sdl += sdr * a_droe;
	a_sdr += sdl * a_droe;
	const double a_sum = -isd * isd * a_isd;
	a_sdl += a_sum;
	a_sdr += a_sum;

	// ---- reverse of both fluxes and states
	auto flux7_rev = [&](const Side_Fwd& S, Side_Adj& A, const double p, const double pb, const double by,
	                     const double bz, const double* aFs, const double* aUs, double& a_p, double& a_pb,
	                     double& a_by, double& a_bz) {
		const double vbx = bxi * S.v0 + by * S.v1 + bz * S.v2;
		A.m0 += aFs[0] + S.v0 * aFs[1] + S.v1 * aFs[2] + S.v2 * aFs[3];
		A.v0 += S.m0 * aFs[1] + (S.E + p + pb) * aFs[4] - bxi * bxi * aFs[4] + by * aFs[5] + bz * aFs[6];
		A.v1 += S.m0 * aFs[2] - bxi * by * aFs[4] - bxi * aFs[5];
		A.v2 += S.m0 * aFs[3] - bxi * bz * aFs[4] - bxi * aFs[6];
		a_p += aFs[1] + S.v0 * aFs[4];
		a_pb += S.v0 * aFs[4];
		A.E += S.v0 * aFs[4];
		a_bxi += -bxi * aFs[1] - by * aFs[2] - bz * aFs[3] - (vbx + bxi * S.v0) * aFs[4] - S.v1 * aFs[5] - S.v2 * aFs[6];
		a_by += by * aFs[1] - bxi * aFs[2] - bxi * S.v1 * aFs[4] + S.v0 * aFs[5];
		a_bz += bz * aFs[1] - bxi * aFs[3] - bxi * S.v2 * aFs[4] + S.v0 * aFs[6];
		// the state [rho, m, E, by, bz]
		A.rho += aUs[0];
		A.m0 += aUs[1]; A.m1 += aUs[2]; A.m2 += aUs[3];
		A.E += aUs[4];
		a_by += aUs[5];
		a_bz += aUs[6];
	};
	flux7_rev(L, AL, pl, pbl, byl, bzl, aFl, aUl, a_pl, a_pbl, a_byl, a_bzl);
	flux7_rev(R, AR, pr, pbr, byr, bzr, aFr, aUr, a_pr, a_pbr, a_byr, a_bzr);
	// pb = (bxi^2 + by^2 + bz^2) / 2
	a_bxi += bxi * (a_pbl + a_pbr);
	a_byl += byl * a_pbl; a_bzl += bzl * a_pbl;
	a_byr += byr * a_pbr; a_bzr += bzr * a_pbr;
	// sd = sqrt(rho)
	AL.rho += 0.5 * isdl * a_sdl;
	AR.rho += 0.5 * isdr * a_sdr;
	// p = (E - r m2s / 2 - b2s / 2)(gamma - 1), with r = 1 / rho
	auto pres_rev = [&](const Side_Fwd& S, Side_Adj& A, const double a_p) {
		A.E += gm1 * a_p;
		A.rho += 0.5 * S.m2s * gm1 * S.r * S.r * a_p;
		const double c = -S.r * gm1 * a_p;
		A.m0 += c * S.m0; A.m1 += c * S.m1; A.m2 += c * S.m2;
		const double d = -gm1 * a_p;
		A.b0 += d * S.b0; A.b1 += d * S.b1; A.b2 += d * S.b2;
	};
	pres_rev(L, AL, a_pl);
	pres_rev(R, AR, a_pr);
	// bxi = (bL0 + bR0) / (2 sqrt(mu0)), by = b1 / sqrt(mu0), bz = b2 / sqrt(mu0)
	AL.b0 += 0.5 * ism * a_bxi;
	AR.b0 += 0.5 * ism * a_bxi;
	AL.b1 += ism * a_byl; AL.b2 += ism * a_bzl;
	AR.b1 += ism * a_byr; AR.b2 += ism * a_bzr;
	side_reverse(L, AL, g, gL);
	side_reverse(R, AR, g, gR);
}

template <int SOLVER>
__host__ __device__ __forceinline__ void face_vjp(const double* UL, const double* UR, const Gas_Adj& g,
                                                  const double* phi, double* gL, double* gR, double* F = nullptr)
{
	if (SOLVER == 0) rusanov_vjp(UL, UR, g, phi, gL, gR, F);
	else if (SOLVER == 2) hll_vjp(UL, UR, g, phi, gL, gR, F);
	else if (SOLVER == 3) hlld_vjp(UL, UR, g, phi, gL, gR, F);
	else roe_vjp(UL, UR, g, phi, gL, gR, F);
}

}} // namespaces

#endif
