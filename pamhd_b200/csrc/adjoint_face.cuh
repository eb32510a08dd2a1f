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

template <int SOLVER>
__host__ __device__ __forceinline__ void face_vjp(const double* UL, const double* UR, const Gas_Adj& g,
                                                  const double* phi, double* gL, double* gR, double* F = nullptr)
{
	if (SOLVER == 0) rusanov_vjp(UL, UR, g, phi, gL, gR, F);
	else if (SOLVER == 2) hll_vjp(UL, UR, g, phi, gL, gR, F);
	else hlld_vjp(UL, UR, g, phi, gL, gR, F);
}

}} // namespaces

#endif
