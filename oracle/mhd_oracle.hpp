/*
CPU oracle for PAMHD's finite-volume MHD step.

TEST INFRASTRUCTURE - this is the checker, not the product.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may build, load or
call anything under oracle/.  The product (pamhd_b200/csrc, include/) never
includes or links it.

What it restates, in plain C++ and in the reference's operation order
(expression by expression, so that a build with -ffp-contract=off gives the
same bits as the reference headers built the same way):
  L1  mhd/common.hpp          get_pressure :79, get_velocity :121,
                              get_flux :146, get_total_energy_density :258,
                              get_sound_speed :327, get_alfven_speed :381,
                              get_fast_magnetosonic_speed :418,
                              get_rotated_vector :612, apply_fluxes :707
      common_functions.hpp    add :52, mul :84, dot :136 (sum order)
  L2  mhd/rusanov.hpp:67, mhd/hll_athena.hpp:65, mhd/hlld_athena.hpp:62,
      mhd/roe_athena.hpp:56 (eigensystem), :341 (fluxes), :575 (wrapper)
  L3  the cell-centred ("Mode C") step of mhd/solve.hpp on a uniform grid,
      written out in Mode_C_Grid below with its own citations.

Parity pin: tests/test_oracle_pin.py compares these solvers bit for bit with
the reference's own headers compiled by oracle/Makefile (oracle/_ref), and
with the committed fixtures in tests/golden made from them; the 1-D scheme
(reference_1d) is compared with the reference's golden files
tests/mhd/mhd_rusanov.ref and mhd_hll_athena.ref and with the compiled
tests/mhd/reference.cpp.

Errors: where the reference throws std::domain_error, the oracle throws
Domain_Error carrying the matching PAMHD_FLAG_* bit of include/pamhd_gpu.h.
*/
#ifndef PAMHD_ORACLE_HPP
#define PAMHD_ORACLE_HPP

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../include/pamhd_gpu.h"

namespace oracle {

using Vec3 = std::array<double, 3>;

// conservative state, in the order of detail::MHD (mhd/variables.hpp:240)
struct MHD {
	double rho = 0;
	Vec3 mom{0, 0, 0};
	double nrj = 0;
	Vec3 mag{0, 0, 0};
};

struct Face_Flux {
	MHD flux;
	double speed = 0;
};

struct Domain_Error : std::domain_error {
	uint32_t flag;
	Domain_Error(uint32_t f, const std::string& what) : std::domain_error(what), flag(f) {}
};

// ---------------------------------------------------------------- L1

// mhd/common.hpp:79-115
inline double get_pressure(
	const double rho, const Vec3& mom, const double nrj, const Vec3& mag,
	const double gamma, const double mu0
) {
	if (rho <= 0) {
		throw Domain_Error(PAMHD_FLAG_DENSITY, "Non-positive mass density given to get_pressure");
	}
	const double
		kinetic = 0.5 / rho * (mom[0] * mom[0] + mom[1] * mom[1] + mom[2] * mom[2]),
		magnetic = 0.5 / mu0 * (mag[0] * mag[0] + mag[1] * mag[1] + mag[2] * mag[2]);
	return (nrj - kinetic - magnetic) * (gamma - 1);
}

// mhd/common.hpp:121-130 (mul(momentum, 1 / mass))
inline Vec3 get_velocity(const Vec3& mom, const double rho)
{
	if (rho > 0) {
		const double inv = 1 / rho;
		return {mom[0] * inv, mom[1] * inv, mom[2] * inv};
	}
	return {0, 0, 0};
}

// common_functions.hpp:136-147: sum starts from 0 and adds in index order
inline double dot(const Vec3& a, const Vec3& b)
{
	double out = 0;
	out += a[0] * b[0];
	out += a[1] * b[1];
	out += a[2] * b[2];
	return out;
}

// mhd/common.hpp:146-244
inline MHD get_flux(const MHD& s, const Vec3& bg, const double gamma, const double mu0)
{
	if (not std::isnormal(s.rho) or s.rho <= 0) {
		throw Domain_Error(PAMHD_FLAG_DENSITY, "Invalid mass density given to get_flux");
	}
	if (not std::isfinite(s.mom[0])) {
		throw Domain_Error(PAMHD_FLAG_FLUX, "Invalid momentum x density given to get_flux");
	}
	const Vec3 tot{s.mag[0] + bg[0], s.mag[1] + bg[1], s.mag[2] + bg[2]};
	const double
		inv_mu0 = 1.0 / mu0,
		p_bg = 0.5 * inv_mu0 * (bg[0] * bg[0] + bg[1] * bg[1] + bg[2] * bg[2]),
		p_b1 = 0.5 * inv_mu0 * (s.mag[0] * s.mag[0] + s.mag[1] * s.mag[1] + s.mag[2] * s.mag[2]),
		p_tot = 0.5 * inv_mu0 * (tot[0] * tot[0] + tot[1] * tot[1] + tot[2] * tot[2]),
		p_th = get_pressure(s.rho, s.mom, s.nrj, s.mag, gamma, mu0);
	const Vec3 v = get_velocity(s.mom, s.rho);

	MHD f;
	f.rho = s.mom[0];
	if (not std::isfinite(f.rho)) {
		throw Domain_Error(PAMHD_FLAG_FLUX, "Invalid mass density flux");
	}
	for (int i = 0; i < 3; i++) {
		f.mom[i] = s.mom[i] * v[0] + (-inv_mu0) * (tot[0] * tot[i] + (-bg[0]) * bg[i]);
	}
	f.mom[0] += p_th + p_tot - p_bg;
	f.nrj
		= v[0] * (s.nrj + p_th + p_b1)
		- s.mag[0] * dot(v, s.mag) * inv_mu0
		+ inv_mu0 * (
			s.mag[1] * (v[0] * bg[1] - v[1] * bg[0])
			+ s.mag[2] * (v[0] * bg[2] - v[2] * bg[0]));
	for (int i = 0; i < 3; i++) {
		f.mag[i] = v[0] * tot[i] + (-tot[0]) * v[i];
	}
	f.mag[0] = 0;
	return f;
}

// mhd/common.hpp:258-311
inline double get_total_energy_density(
	const double rho, const Vec3& vel, const double pressure, const Vec3& mag,
	const double gamma, const double mu0
) {
	if (rho <= 0) {
		throw Domain_Error(PAMHD_FLAG_DENSITY, "Non-positive mass density given to get_total_energy_density");
	}
	if (gamma <= 1 or mu0 <= 0) {
		throw std::invalid_argument("adiabatic index must be > 1 and vacuum permeability > 0");
	}
	const double
		kinetic = 0.5 * rho * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]),
		magnetic = 0.5 / mu0 * (mag[0] * mag[0] + mag[1] * mag[1] + mag[2] * mag[2]);
	return pressure / (gamma - 1) + kinetic + magnetic;
}

// mhd/common.hpp:327-368
inline double get_sound_speed(
	const double rho, const Vec3& mom, const double nrj, const Vec3& mag,
	const double gamma, const double mu0
) {
	if (not std::isnormal(rho) or rho < 0) {
		throw Domain_Error(PAMHD_FLAG_DENSITY, "Invalid mass density given to get_sound_speed");
	}
	const double p = get_pressure(rho, mom, nrj, mag, gamma, mu0);
	if (not std::isnormal(p) or p < 0) {
		throw Domain_Error(PAMHD_FLAG_PRESSURE, "Non-positive pressure given to get_sound_speed");
	}
	return std::sqrt(gamma * p / rho);
}

// mhd/common.hpp:381-405 (pow(x, 2) is x * x to the last bit)
inline double get_alfven_speed(const double rho, const Vec3& mag, const Vec3& bg, const double mu0)
{
	if (not std::isnormal(rho) or rho < 0) {
		throw Domain_Error(PAMHD_FLAG_DENSITY, "Non-positive mass density given to get_alfven_speed");
	}
	const double
		b0 = mag[0] + bg[0], b1 = mag[1] + bg[1], b2 = mag[2] + bg[2],
		b = std::sqrt(b0 * b0 + b1 * b1 + b2 * b2);
	return b / std::sqrt(mu0 * rho);
}

// mhd/common.hpp:418-491
inline double get_fast_magnetosonic_speed(
	const double rho, const Vec3& mom, const double nrj, const Vec3& mag,
	const Vec3& bg, const double gamma, const double mu0
) {
	const Vec3 tot{mag[0] + bg[0], mag[1] + bg[1], mag[2] + bg[2]};
	if (not std::isfinite(tot[0])) {
		throw Domain_Error(PAMHD_FLAG_WAVE_SPEED, "Invalid total magnetic field x");
	}
	const double
		b = std::sqrt(tot[0] * tot[0] + tot[1] * tot[1] + tot[2] * tot[2]),
		sound = get_sound_speed(rho, mom, nrj, mag, gamma, mu0);
	if (b <= 0) {
		return sound;
	}
	const double
		alfven = get_alfven_speed(rho, mag, bg, mu0),
		sound2 = sound * sound,
		alfven2 = alfven * alfven,
		sum2 = sound2 + alfven2;
	if (not std::isnormal(sum2) or sum2 < 0) {
		throw Domain_Error(PAMHD_FLAG_WAVE_SPEED, "Invalid squared speeds in get_fast_magnetosonic_speed");
	}
	const double
		cos_b = tot[0] / b,
		to_sqrt = sound2 * sound2 + alfven2 * alfven2 + 2 * sound2 * alfven2 * (1 - 2 * (cos_b * cos_b));
	if (not std::isnormal(to_sqrt) or to_sqrt < 0) {
		throw Domain_Error(PAMHD_FLAG_WAVE_SPEED, "Invalid to_sqrt in get_fast_magnetosonic_speed");
	}
	return std::sqrt(0.5 * (sum2 + std::sqrt(to_sqrt)));
}

// mhd/common.hpp:612-648; dir in {+-1, +-2, +-3}
inline Vec3 get_rotated_vector(const Vec3& v, const int dir)
{
	switch (dir) {
	case -3: case 2: return {v[1], v[2], v[0]};
	case -2: case 3: return {v[2], v[0], v[1]};
	case -1: case 1: return v;
	default: throw std::invalid_argument("invalid direction");
	}
}

// ---------------------------------------------------------------- L2

// mhd/rusanov.hpp:67-179
inline Face_Flux get_flux_rusanov(
	const MHD& neg, const MHD& pos, const Vec3& bg, const double gamma, const double mu0
) {
	if (not std::isnormal(neg.rho) or neg.rho < 0) {
		throw Domain_Error(PAMHD_FLAG_DENSITY, "Invalid mass density in state_neg");
	}
	if (not std::isnormal(pos.rho) or pos.rho < 0) {
		throw Domain_Error(PAMHD_FLAG_DENSITY, "Invalid mass density in state_pos");
	}
	const double
		fast_neg = get_fast_magnetosonic_speed(neg.rho, neg.mom, neg.nrj, neg.mag, bg, gamma, mu0),
		fast_pos = get_fast_magnetosonic_speed(pos.rho, pos.mom, pos.nrj, pos.mag, bg, gamma, mu0),
		fast = std::max(fast_neg, fast_pos),
		s = std::max(
			std::abs(neg.mom[0] / neg.rho) + fast,
			std::abs(pos.mom[0] / pos.rho) + fast);
	if (not std::isfinite(fast)) {
		throw Domain_Error(PAMHD_FLAG_WAVE_SPEED, "Invalid maximum fast magnetosonic speed");
	}
	if (not std::isfinite(s)) {
		throw Domain_Error(PAMHD_FLAG_WAVE_SPEED, "Invalid maximum signal speed");
	}
	const MHD fn = get_flux(neg, bg, gamma, mu0), fp = get_flux(pos, bg, gamma, mu0);
	if (not std::isfinite(fn.rho) or not std::isfinite(fp.rho)) {
		throw Domain_Error(PAMHD_FLAG_FLUX, "Invalid mass density flux");
	}
	Face_Flux out;
	MHD& f = out.flux;
	f.rho = (fn.rho + fp.rho) / 2 - (pos.rho - neg.rho) * (s / 2);
	f.nrj = (fn.nrj + fp.nrj) / 2 - (pos.nrj - neg.nrj) * (s / 2);
	for (int i = 0; i < 3; i++) {
		f.mom[i] = (fn.mom[i] + fp.mom[i]) * 0.5 + (pos.mom[i] + (-neg.mom[i])) * (-s / 2);
		f.mag[i] = (fn.mag[i] + fp.mag[i]) * 0.5 + (pos.mag[i] + (-neg.mag[i])) * (-s / 2);
	}
	if (not std::isfinite(f.rho)) {
		throw Domain_Error(PAMHD_FLAG_FLUX, "Invalid mass density flux");
	}
	out.speed = s;
	return out;
}

// mhd/hll_athena.hpp:65-275
inline Face_Flux get_flux_hll(
	const MHD& neg, const MHD& pos, const Vec3& bg, const double gamma, const double mu0
) {
	const Vec3
		v_neg = get_velocity(neg.mom, neg.rho),
		v_pos = get_velocity(pos.mom, pos.rho);
	const double
		p_neg = get_pressure(neg.rho, neg.mom, neg.nrj, neg.mag, gamma, mu0),
		p_pos = get_pressure(pos.rho, pos.mom, pos.nrj, pos.mag, gamma, mu0),
		pb_neg = dot(neg.mag, neg.mag) / (2 * mu0),
		pb_pos = dot(pos.mag, pos.mag) / (2 * mu0),
		fast_neg = get_fast_magnetosonic_speed(neg.rho, neg.mom, neg.nrj, neg.mag, bg, gamma, mu0),
		fast_pos = get_fast_magnetosonic_speed(pos.rho, pos.mom, pos.nrj, pos.mag, bg, gamma, mu0),
		fast = std::max(fast_neg, fast_pos),
		s_neg = (v_neg[0] <= v_pos[0]) ? v_neg[0] - fast : v_pos[0] - fast,
		s_pos = (v_neg[0] <= v_pos[0]) ? v_pos[0] + fast : v_neg[0] + fast,
		bm = std::min(s_neg, 0.0),
		bp = std::max(s_pos, 0.0);

	if (not std::isnormal(p_neg) or p_neg < 0) {
		throw Domain_Error(PAMHD_FLAG_PRESSURE, "Invalid thermal pressure in state_neg");
	}
	if (not std::isfinite(pb_neg) or pb_neg < 0) {
		throw Domain_Error(PAMHD_FLAG_PRESSURE, "Invalid magnetic pressure in state_neg");
	}
	if (not std::isfinite(s_neg)) {
		throw Domain_Error(PAMHD_FLAG_WAVE_SPEED, "Invalid max signal speed in state_neg");
	}
	if (not std::isnormal(p_pos) or p_pos < 0) {
		throw Domain_Error(PAMHD_FLAG_PRESSURE, "Invalid thermal pressure in state_pos");
	}
	if (not std::isfinite(pb_pos) or pb_pos < 0) {
		throw Domain_Error(PAMHD_FLAG_PRESSURE, "Invalid magnetic pressure in state_pos");
	}
	if (not std::isfinite(s_pos)) {
		throw Domain_Error(PAMHD_FLAG_WAVE_SPEED, "Invalid max signal speed in state_pos");
	}

	Face_Flux out;
	if (not std::isnormal(bp - bm) or bp - bm < 0) {
		// degenerate fan: zero flux and zero speed (hll_athena.hpp:194-207)
		return out;
	}

	MHD fn = get_flux(neg, bg, gamma, mu0), fp = get_flux(pos, bg, gamma, mu0);
	fn.rho -= neg.rho * bm;
	fn.nrj -= neg.nrj * bm;
	fp.rho -= pos.rho * bp;
	fp.nrj -= pos.nrj * bp;
	for (int i = 0; i < 3; i++) {
		fn.mom[i] = fn.mom[i] + neg.mom[i] * (-bm);
		fn.mag[i] = fn.mag[i] + neg.mag[i] * (-bm);
		fp.mom[i] = fp.mom[i] + pos.mom[i] * (-bp);
		fp.mag[i] = fp.mag[i] + pos.mag[i] * (-bp);
	}
	fp.mag[0] = fn.mag[0] = 0;

	MHD& f = out.flux;
	f.rho = (fn.rho + fp.rho) / 2 + (fn.rho - fp.rho) * (bp + bm) / (bp - bm) / 2.0;
	f.nrj = (fn.nrj + fp.nrj) / 2 + (fn.nrj - fp.nrj) * (bp + bm) / (bp - bm) / 2.0;
	const double w = (bp + bm) / (bp - bm) / 2.0;
	for (int i = 0; i < 3; i++) {
		f.mom[i] = 0.5 * (fn.mom[i] + fp.mom[i]) + (fn.mom[i] + (-fp.mom[i])) * w;
		f.mag[i] = 0.5 * (fn.mag[i] + fp.mag[i]) + (fn.mag[i] + (-fp.mag[i])) * w;
	}
	out.speed = std::max(std::abs(bp), std::abs(bm));
	return out;
}

// mhd/hlld_athena.hpp:62-559 (Miyoshi & Kusano 2005); background field ignored (:77)
inline Face_Flux get_flux_hlld(
	const MHD& neg, const MHD& pos, const Vec3& /*bg*/, const double gamma, const double mu0
) {
	const Vec3 zero{0, 0, 0};
	if (neg.rho <= 0) {
		throw Domain_Error(PAMHD_FLAG_DENSITY, "Non-positive mass density on negative side");
	}
	if (pos.rho <= 0) {
		throw Domain_Error(PAMHD_FLAG_DENSITY, "Non-positive mass density on positive side");
	}
	const double p_neg = get_pressure(neg.rho, neg.mom, neg.nrj, neg.mag, gamma, mu0);
	if (p_neg <= 0) {
		throw Domain_Error(PAMHD_FLAG_PRESSURE, "Non-positive pressure on negative side");
	}
	const double p_pos = get_pressure(pos.rho, pos.mom, pos.nrj, pos.mag, gamma, mu0);
	if (p_pos <= 0) {
		throw Domain_Error(PAMHD_FLAG_PRESSURE, "Non-positive pressure on positive side");
	}

	constexpr double eps = std::numeric_limits<double>::epsilon();
	const double
		inv_mu0 = 1.0 / mu0,
		inv_sqrt_mu0 = 1.0 / std::sqrt(mu0),
		bx = (neg.mag[0] + pos.mag[0]) / 2,
		bx2 = bx * bx,
		fast_neg = get_fast_magnetosonic_speed(neg.rho, neg.mom, neg.nrj, neg.mag, zero, gamma, mu0),
		fast_pos = get_fast_magnetosonic_speed(pos.rho, pos.mom, pos.nrj, pos.mag, zero, gamma, mu0),
		fast = std::max(fast_neg, fast_pos);

	const double inv_rho_neg = 1 / neg.rho, inv_rho_pos = 1 / pos.rho;
	const Vec3
		v_neg{neg.mom[0] * inv_rho_neg, neg.mom[1] * inv_rho_neg, neg.mom[2] * inv_rho_neg},
		v_pos{pos.mom[0] * inv_rho_pos, pos.mom[1] * inv_rho_pos, pos.mom[2] * inv_rho_pos};

	// eqn 67
	const double
		s_neg = (v_neg[0] <= v_pos[0]) ? v_neg[0] - fast : v_pos[0] - fast,
		s_pos = (v_neg[0] <= v_pos[0]) ? v_pos[0] + fast : v_neg[0] + fast;

	const MHD f_neg = get_flux(neg, zero, gamma, mu0), f_pos = get_flux(pos, zero, gamma, mu0);

	// supersonic: upwind flux (hlld_athena.hpp:252-257)
	if (s_neg >= 0.0) {
		return {f_neg, std::abs(s_pos)};
	} else if (s_pos <= 0.0) {
		return {f_pos, std::abs(s_neg)};
	}

	const double
		sdiff_neg = s_neg - v_neg[0],
		sdiff_pos = s_pos - v_pos[0],
		pb_neg = dot(neg.mag, neg.mag) * (inv_mu0 / 2),
		pb_pos = dot(pos.mag, pos.mag) * (inv_mu0 / 2),
		// eqn 38
		s_mid
			= (sdiff_pos * pos.mom[0] - sdiff_neg * neg.mom[0] - (p_pos + pb_pos) + (p_neg + pb_neg))
			/ (sdiff_pos * pos.rho - sdiff_neg * neg.rho),
		smid_neg = s_neg - s_mid,
		smid_pos = s_pos - s_mid,
		// eqn 43
		rho_s_neg = neg.rho * sdiff_neg / smid_neg,
		sqrt_rho_s_neg = std::sqrt(rho_s_neg),
		rho_s_pos = pos.rho * sdiff_pos / smid_pos,
		sqrt_rho_s_pos = std::sqrt(rho_s_pos),
		// eqn 51
		ss_neg = s_mid - std::abs(bx) / std::sqrt(rho_s_neg * mu0),
		ss_pos = s_mid + std::abs(bx) / std::sqrt(rho_s_pos * mu0),
		ptst = p_neg + pb_neg + neg.rho * sdiff_neg * (s_mid - v_neg[0]);

	// one side of the fan: the star state Ul* or Ur* (eqns 44-48)
	auto star = [&](const MHD& u, const Vec3& v, const double p, const double pb,
	                const double sdiff, const double smid, const double rho_s) {
		MHD st;
		const double tmp = u.rho * sdiff * smid - bx2 * inv_mu0;
		if (std::abs(tmp) < eps * ptst) {
			for (int i = 0; i < 3; i++) {
				st.mom[i] = rho_s * v[i];
			}
			st.mag = u.mag;
		} else {
			const double t1 = bx * (s_mid - v[0]) * inv_mu0 / tmp;
			for (int i = 0; i < 3; i++) {
				st.mom[i] = rho_s * (v[i] + u.mag[i] * (-t1));
			}
			const double t2 = (u.rho * (sdiff * sdiff) - bx2 * inv_mu0) / tmp;
			for (int i = 0; i < 3; i++) {
				st.mag[i] = u.mag[i] * t2;
			}
		}
		st.rho = rho_s;
		st.mom[0] = rho_s * s_mid;
		st.mag[0] = bx;
		const double vb_s = dot(st.mom, st.mag) / rho_s;
		st.nrj
			= (sdiff * u.nrj - (p + pb) * v[0] + ptst * s_mid + bx * inv_mu0 * (dot(v, u.mag) - vb_s))
			/ smid;
		return std::make_pair(st, vb_s);
	};
	const auto [st_neg, vb_s_neg] = star(neg, v_neg, p_neg, pb_neg, sdiff_neg, smid_neg, rho_s_neg);
	const auto [st_pos, vb_s_pos] = star(pos, v_pos, p_pos, pb_pos, sdiff_pos, smid_pos, rho_s_pos);

	const double inv_rs_neg = 1 / rho_s_neg, inv_rs_pos = 1 / rho_s_pos;
	const Vec3
		vs_neg{st_neg.mom[0] * inv_rs_neg, st_neg.mom[1] * inv_rs_neg, st_neg.mom[2] * inv_rs_neg},
		vs_pos{st_pos.mom[0] * inv_rs_pos, st_pos.mom[1] * inv_rs_pos, st_pos.mom[2] * inv_rs_pos};

	// the double-star states Ul**, Ur** (eqns 59-63)
	MHD ss2_neg, ss2_pos;
	if (bx2 / 2 < eps * ptst) {
		ss2_neg = st_neg;
		ss2_pos = st_pos;
	} else {
		const double
			inv_sum = 1.0 / (sqrt_rho_s_neg + sqrt_rho_s_pos),
			sgn = (bx > 0) ? 1.0 : -1.0;
		ss2_neg.rho = st_neg.rho;
		ss2_pos.rho = st_pos.rho;
		Vec3 v2;
		for (int i = 0; i < 3; i++) {
			v2[i] = inv_sum * ((sqrt_rho_s_neg * vs_neg[i] + sqrt_rho_s_pos * vs_pos[i])
				+ (sgn * inv_sqrt_mu0) * (st_pos.mag[i] + (-st_neg.mag[i])));
		}
		v2[0] = s_mid;
		for (int i = 0; i < 3; i++) {
			ss2_neg.mom[i] = st_neg.rho * v2[i];
			ss2_pos.mom[i] = st_pos.rho * v2[i];
		}
		ss2_neg.mom[0] = st_neg.mom[0];
		ss2_pos.mom[0] = st_pos.mom[0];
		const double wb = sgn * sqrt_rho_s_neg * sqrt_rho_s_pos * std::sqrt(mu0);
		for (int i = 0; i < 3; i++) {
			ss2_neg.mag[i] = inv_sum * ((sqrt_rho_s_neg * st_pos.mag[i] + sqrt_rho_s_pos * st_neg.mag[i])
				+ wb * (vs_pos[i] + (-vs_neg[i])));
		}
		ss2_neg.mag[0] = bx;
		ss2_pos.mag = ss2_neg.mag;
		const double vb2 = dot(v2, ss2_neg.mag);
		ss2_neg.nrj = st_neg.nrj - sqrt_rho_s_neg * sgn * (vb_s_neg - vb2) * inv_sqrt_mu0;
		ss2_pos.nrj = st_pos.nrj + sqrt_rho_s_pos * sgn * (vb_s_pos - vb2) * inv_sqrt_mu0;
	}

	// region select (hlld_athena.hpp:475-552)
	Face_Flux out;
	MHD& f = out.flux;
	auto outer = [&](const MHD& fu, const MHD& u, const MHD& st, const double s) {
		f.rho = fu.rho + (st.rho - u.rho) * s;
		f.nrj = fu.nrj + (st.nrj - u.nrj) * s;
		for (int i = 0; i < 3; i++) {
			f.mom[i] = fu.mom[i] + s * (st.mom[i] + (-u.mom[i]));
			f.mag[i] = fu.mag[i] + s * (st.mag[i] + (-u.mag[i]));
		}
	};
	auto inner = [&](const MHD& fu, const MHD& u, const MHD& st, const MHD& st2,
	                 const double s, const double ss) {
		f.rho = fu.rho + st2.rho * ss - st.rho * (ss - s) - u.rho * s;
		f.nrj = fu.nrj + st2.nrj * ss - st.nrj * (ss - s) - u.nrj * s;
		for (int i = 0; i < 3; i++) {
			f.mom[i] = fu.mom[i] + st2.mom[i] * ss + st.mom[i] * (-(ss - s)) + u.mom[i] * (-s);
			f.mag[i] = fu.mag[i] + st2.mag[i] * ss + st.mag[i] * (-(ss - s)) + u.mag[i] * (-s);
		}
	};
	if (ss_neg >= 0) {
		outer(f_neg, neg, st_neg, s_neg);
	} else if (s_mid >= 0) {
		inner(f_neg, neg, st_neg, ss2_neg, s_neg, ss_neg);
	} else if (ss_pos > 0) {
		inner(f_pos, pos, st_pos, ss2_pos, s_pos, ss_pos);
	} else {
		outer(f_pos, pos, st_pos, s_pos);
	}
	f.mag[0] = 0;
	out.speed = std::max(std::abs(s_neg), std::abs(s_pos));
	return out;
}

namespace roe {

constexpr int NW = 7;
using Row = std::array<double, NW>;
using Matrix = std::array<Row, NW>;

/*
Eigenvalues and right (columns) / left (rows) eigenvectors of the adiabatic
MHD Roe matrix, mhd/roe_athena.hpp:56-296 (Athena's esys_roe_adb_mhd; eqns
B17-B29 of Stone et al. 2008).  d, v1..v3, h, b1..b3: Roe averages; x, y:
the numerical factors of the averaged field.
*/
inline void eigensystem(
	const double d, const double v1, const double v2, const double v3,
	const double h, const double b1, const double b2, const double b3,
	const double x, const double y, const double gamma,
	Row& ev, Matrix& R, Matrix& L
) {
	constexpr double tiny = std::numeric_limits<double>::epsilon();
	const double g1 = gamma - 1, g2 = gamma - 2;
	const double di = 1.0 / d;
	const double vsq = v1 * v1 + v2 * v2 + v3 * v3;
	const double btsq = b2 * b2 + b3 * b3;
	const double bt_starsq = (g1 - g2 * y) * btsq;
	const double vaxsq = b1 * b1 * di;
	const double hp = h - (vaxsq + btsq * di);
	const double twid_asq = std::max((g1 * (hp - 0.5 * vsq) - g2 * x), tiny);

	// fast and slow magnetosonic speeds (B18)
	const double ct2 = bt_starsq * di;
	const double tsum = vaxsq + ct2 + twid_asq;
	const double tdif = vaxsq + ct2 - twid_asq;
	const double cf2_cs2 = std::sqrt(tdif * tdif + 4.0 * twid_asq * ct2);
	const double cfsq = 0.5 * (tsum + cf2_cs2);
	const double cf = std::sqrt(cfsq);
	const double cssq = twid_asq * vaxsq / cfsq;
	const double cs = std::sqrt(cssq);

	// betas (A17, B20, B28)
	const double bt = std::sqrt(btsq);
	const double bt_star = std::sqrt(bt_starsq);
	double bet2 = 1.0, bet3 = 0.0;
	if (bt != 0.0) {
		bet2 = b2 / bt;
		bet3 = b3 / bt;
	}
	const double bet2_star = bet2 / std::sqrt(g1 - g2 * y);
	const double bet3_star = bet3 / std::sqrt(g1 - g2 * y);
	const double bet_starsq = bet2_star * bet2_star + bet3_star * bet3_star;
	const double vbet = v2 * bet2_star + v3 * bet3_star;

	// alphas (A16)
	double alpha_f, alpha_s;
	if ((cfsq - cssq) == 0.0) {
		alpha_f = 1.0; alpha_s = 0.0;
	} else if ((twid_asq - cssq) <= 0.0) {
		alpha_f = 0.0; alpha_s = 1.0;
	} else if ((cfsq - twid_asq) <= 0.0) {
		alpha_f = 1.0; alpha_s = 0.0;
	} else {
		alpha_f = std::sqrt((twid_asq - cssq) / (cfsq - cssq));
		alpha_s = std::sqrt((cfsq - twid_asq) / (cfsq - cssq));
	}

	// Q and A (A14-15)
	const double sqrtd = std::sqrt(d);
	const double isqrtd = 1.0 / sqrtd;
	const double s = (b1 > 0) ? 1 : -1;
	const double twid_a = std::sqrt(twid_asq);
	double qf = cf * alpha_f * s;
	double qs = cs * alpha_s * s;
	const double af_prime = twid_a * alpha_f * isqrtd;
	const double as_prime = twid_a * alpha_s * isqrtd;
	const double afpbb = af_prime * bt_star * bet_starsq;
	const double aspbb = as_prime * bt_star * bet_starsq;

	// eigenvalues (B17)
	const double vax = std::sqrt(vaxsq);
	ev = {v1 - cf, v1 - vax, v1 - cs, v1, v1 + cs, v1 + vax, v1 + cf};

	// right eigenvectors as columns (B21)
	R[0] = {alpha_f, 0.0, alpha_s, 1.0, alpha_s, 0.0, alpha_f};
	R[1] = {alpha_f * ev[0], 0.0, alpha_s * ev[2], v1, alpha_s * ev[4], 0.0, alpha_f * ev[6]};
	for (int k = 0; k < 2; k++) {
		const double vt = (k == 0) ? v2 : v3;
		const double bs = (k == 0) ? bet2_star : bet3_star;
		const double qa = alpha_f * vt, qb = alpha_s * vt, qc = qs * bs, qd = qf * bs;
		const double side = (k == 0) ? -bet3 : bet2;
		R[2 + k] = {qa + qc, side, qb - qd, vt, qb + qd, -side, qa - qc};
	}
	R[4][0] = alpha_f * (hp - v1 * cf) + qs * vbet + aspbb;
	R[4][1] = -(v2 * bet3 - v3 * bet2);
	R[4][2] = alpha_s * (hp - v1 * cs) - qf * vbet - afpbb;
	R[4][3] = 0.5 * vsq + g2 * x / g1;
	R[4][4] = alpha_s * (hp + v1 * cs) + qf * vbet - afpbb;
	R[4][5] = -R[4][1];
	R[4][6] = alpha_f * (hp + v1 * cf) - qs * vbet + aspbb;
	R[5] = {as_prime * bet2_star, -bet3 * s * isqrtd, -af_prime * bet2_star, 0.0, 0.0, 0.0, 0.0};
	R[6] = {as_prime * bet3_star, bet2 * s * isqrtd, -af_prime * bet3_star, 0.0, 0.0, 0.0, 0.0};
	for (int r = 5; r < 7; r++) {
		R[r][4] = R[r][2];
		R[r][5] = R[r][1];
		R[r][6] = R[r][0];
	}

	// left eigenvectors as rows (B29), normalised by 1 / 2a^2
	double norm = 0.5 / twid_asq;
	const double cff = norm * alpha_f * cf;
	const double css = norm * alpha_s * cs;
	qf *= norm;
	qs *= norm;
	const double af = norm * af_prime * d;
	const double as = norm * as_prime * d;
	const double afpb = norm * af_prime * bt_star;
	const double aspb = norm * as_prime * bt_star;
	// then by (gamma - 1) / 2a^2
	norm *= g1;
	alpha_f *= norm;
	alpha_s *= norm;
	const double q2_star = bet2_star / bet_starsq;
	const double q3_star = bet3_star / bet_starsq;
	const double vqstr = (v2 * q2_star + v3 * q3_star);
	norm *= 2.0;

	L[0][0] = alpha_f * (vsq - hp) + cff * (cf + v1) - qs * vqstr - aspb;
	L[0][1] = -alpha_f * v1 - cff;
	L[0][2] = -alpha_f * v2 + qs * q2_star;
	L[0][3] = -alpha_f * v3 + qs * q3_star;
	L[0][4] = alpha_f;
	L[0][5] = as * q2_star - alpha_f * b2;
	L[0][6] = as * q3_star - alpha_f * b3;

	L[1] = {0.5 * (v2 * bet3 - v3 * bet2), 0.0, -0.5 * bet3, 0.5 * bet2, 0.0,
	        -0.5 * sqrtd * bet3 * s, 0.5 * sqrtd * bet2 * s};

	L[2][0] = alpha_s * (vsq - hp) + css * (cs + v1) + qf * vqstr + afpb;
	L[2][1] = -alpha_s * v1 - css;
	L[2][2] = -alpha_s * v2 - qf * q2_star;
	L[2][3] = -alpha_s * v3 - qf * q3_star;
	L[2][4] = alpha_s;
	L[2][5] = -af * q2_star - alpha_s * b2;
	L[2][6] = -af * q3_star - alpha_s * b3;

	L[3] = {1.0 - norm * (0.5 * vsq - g2 * x / g1), norm * v1, norm * v2, norm * v3,
	        -norm, norm * b2, norm * b3};

	L[4][0] = alpha_s * (vsq - hp) + css * (cs - v1) - qf * vqstr + afpb;
	L[4][1] = -alpha_s * v1 + css;
	L[4][2] = -alpha_s * v2 + qf * q2_star;
	L[4][3] = -alpha_s * v3 + qf * q3_star;
	L[4][4] = alpha_s;
	L[4][5] = L[2][5];
	L[4][6] = L[2][6];

	L[5] = {-L[1][0], 0.0, -L[1][2], -L[1][3], 0.0, L[1][5], L[1][6]};

	L[6][0] = alpha_f * (vsq - hp) + cff * (cf - v1) + qs * vqstr - aspb;
	L[6][1] = -alpha_f * v1 + cff;
	L[6][2] = -alpha_f * v2 - qs * q2_star;
	L[6][3] = -alpha_f * v3 - qs * q3_star;
	L[6][4] = alpha_f;
	L[6][5] = L[0][5];
	L[6][6] = L[0][6];
}

// 1-D conserved (d, Mx, My, Mz, E, By, Bz) and primitive (d, Vx, Vy, Vz, P, By, Bz) vectors
using Cons = Row;
using Prim = Row;

// mhd/roe_athena.hpp:341-559; field in units where mu0 = 1
inline Cons fluxes(const Cons& Ul, const Cons& Ur, const Prim& Wl, const Prim& Wr,
                   const double bxi, const double gamma)
{
	const double sqrtdl = std::sqrt(Wl[0]);
	const double sqrtdr = std::sqrt(Wr[0]);
	const double isdlpdr = 1.0 / (sqrtdl + sqrtdr);

	// Roe averages (step 2)
	const double droe = sqrtdl * sqrtdr;
	const double v1roe = (sqrtdl * Wl[1] + sqrtdr * Wr[1]) * isdlpdr;
	const double v2roe = (sqrtdl * Wl[2] + sqrtdr * Wr[2]) * isdlpdr;
	const double v3roe = (sqrtdl * Wl[3] + sqrtdr * Wr[3]) * isdlpdr;
	const double b2roe = (sqrtdr * Wl[5] + sqrtdl * Wr[5]) * isdlpdr;
	const double b3roe = (sqrtdr * Wl[6] + sqrtdl * Wr[6]) * isdlpdr;
	const double dby = Wl[5] - Wr[5], dbz = Wl[6] - Wr[6], sd = sqrtdl + sqrtdr;
	const double x = 0.5 * (dby * dby + dbz * dbz) / (sd * sd);
	const double y = 0.5 * (Wl[0] + Wr[0]) / droe;
	const double pbl = 0.5 * (bxi * bxi + Wl[5] * Wl[5] + Wl[6] * Wl[6]);
	const double pbr = 0.5 * (bxi * bxi + Wr[5] * Wr[5] + Wr[6] * Wr[6]);
	// enthalpy average (Roe 1981)
	const double hroe = ((Ul[4] + Wl[4] + pbl) / sqrtdl + (Ur[4] + Wr[4] + pbr) / sqrtdr) * isdlpdr;

	Row ev;
	Matrix R{}, L{};
	eigensystem(droe, v1roe, v2roe, v3roe, hroe, bxi, b2roe, b3roe, x, y, gamma, ev, R, L);

	// physical fluxes of both states (step 4)
	auto phys = [bxi](const Cons& U, const Prim& W, const double pb) {
		Cons F;
		F[0] = U[1];
		F[1] = U[1] * W[1];
		F[2] = U[1] * W[2];
		F[3] = U[1] * W[3];
		F[1] += W[4];
		F[4] = (U[4] + W[4]) * W[1];
		F[1] -= 0.5 * (bxi * bxi - W[5] * W[5] - W[6] * W[6]);
		F[2] -= bxi * W[5];
		F[3] -= bxi * W[6];
		F[4] += pb * W[1] - bxi * (bxi * W[1] + W[5] * W[2] + W[6] * W[3]);
		F[5] = W[5] * W[1] - bxi * W[2];
		F[6] = W[6] * W[1] - bxi * W[3];
		return F;
	};
	const Cons Fl = phys(Ul, Wl, pbl), Fr = phys(Ur, Wr, pbr);

	// supersonic (step 5)
	if (ev[0] >= 0.0) return Fl;
	if (ev[NW - 1] <= 0.0) return Fr;

	// wave strengths (step 6)
	Row dU, a;
	for (int m = 0; m < NW; m++) dU[m] = Ur[m] - Ul[m];
	for (int n = 0; n < NW; n++) {
		a[n] = 0.0;
		for (int m = 0; m < NW; m++) a[n] += L[n][m] * dU[m];
	}

	// positivity of the intermediate states (step 7)
	Row u = Ul;
	for (int n = 0; n < NW - 1; n++) {
		for (int m = 0; m < NW; m++) u[m] += a[n] * R[m][n];
		if (ev[n + 1] > ev[n]) {
			if (u[0] <= 0.0) {
				throw Domain_Error(PAMHD_FLAG_ROE_DENSITY, "Non-physical density in intermediate state");
			}
			double p = u[4] - 0.5 * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / u[0];
			p -= 0.5 * (u[5] * u[5] + u[6] * u[6] + bxi * bxi);
			if (p < 0.0) {
				throw Domain_Error(PAMHD_FLAG_ROE_PRESSURE, "Non-physical pressure in intermediate state");
			}
		}
	}

	// Roe flux (step 8)
	Row coeff;
	for (int m = 0; m < NW; m++) coeff[m] = 0.5 * a[m] * std::max(std::fabs(ev[m]), 0.0);
	Cons F;
	for (int r = 0; r < NW; r++) F[r] = 0.5 * (Fl[r] + Fr[r]);
	for (int m = 0; m < NW; m++) {
		for (int r = 0; r < NW; r++) F[r] -= coeff[m] * R[r][m];
	}
	return F;
}

} // namespace roe

// mhd/roe_athena.hpp:575-818; background field ignored (:584)
inline Face_Flux get_flux_roe(
	const MHD& neg, const MHD& pos, const Vec3& /*bg*/, const double gamma, const double mu0
) {
	const Vec3 zero{0, 0, 0};
	if (neg.rho <= 0) {
		throw Domain_Error(PAMHD_FLAG_DENSITY, "Non-positive mass density on negative side");
	}
	if (pos.rho <= 0) {
		throw Domain_Error(PAMHD_FLAG_DENSITY, "Non-positive mass density on positive side");
	}
	const double p_neg = get_pressure(neg.rho, neg.mom, neg.nrj, neg.mag, gamma, mu0);
	if (p_neg <= 0) {
		throw Domain_Error(PAMHD_FLAG_PRESSURE, "Non-positive pressure on negative side");
	}
	const double p_pos = get_pressure(pos.rho, pos.mom, pos.nrj, pos.mag, gamma, mu0);
	if (p_pos <= 0) {
		throw Domain_Error(PAMHD_FLAG_PRESSURE, "Non-positive pressure on positive side");
	}

	const double bxi = (neg.mag[0] + pos.mag[0]) / (2.0 * std::sqrt(mu0));
	const roe::Cons
		Ul{neg.rho, neg.mom[0], neg.mom[1], neg.mom[2], neg.nrj,
		   neg.mag[1] / std::sqrt(mu0), neg.mag[2] / std::sqrt(mu0)},
		Ur{pos.rho, pos.mom[0], pos.mom[1], pos.mom[2], pos.nrj,
		   pos.mag[1] / std::sqrt(mu0), pos.mag[2] / std::sqrt(mu0)};
	// primitives with the pressure of get_primitive (common.hpp:566), which
	// the reference calls with vacuum permeability 1 (roe_athena.hpp:706-721)
	const Vec3 vl = get_velocity(neg.mom, neg.rho), vr = get_velocity(pos.mom, pos.rho);
	const double
		pl = get_pressure(neg.rho, neg.mom, neg.nrj, neg.mag, gamma, 1.0),
		pr = get_pressure(pos.rho, pos.mom, pos.nrj, pos.mag, gamma, 1.0);
	const roe::Prim
		Wl{neg.rho, vl[0], vl[1], vl[2], pl, neg.mag[1] / std::sqrt(mu0), neg.mag[2] / std::sqrt(mu0)},
		Wr{pos.rho, vr[0], vr[1], vr[2], pr, pos.mag[1] / std::sqrt(mu0), pos.mag[2] / std::sqrt(mu0)};

	const roe::Cons F = roe::fluxes(Ul, Ur, Wl, Wr, bxi, gamma);

	Face_Flux out;
	out.flux.rho = F[0];
	out.flux.mom = {F[1], F[2], F[3]};
	out.flux.nrj = F[4];
	out.flux.mag = {0, F[5] * std::sqrt(mu0), F[6] * std::sqrt(mu0)};

	// signal speed (roe_athena.hpp:763-815)
	const double
		fast_neg = get_fast_magnetosonic_speed(neg.rho, neg.mom, neg.nrj, neg.mag, zero, gamma, mu0),
		fast_pos = get_fast_magnetosonic_speed(pos.rho, pos.mom, pos.nrj, pos.mag, zero, gamma, mu0),
		fast = std::max(fast_neg, fast_pos);
	const double inv_rho_neg = 1 / neg.rho, inv_rho_pos = 1 / pos.rho;
	const double vx_neg = neg.mom[0] * inv_rho_neg, vx_pos = pos.mom[0] * inv_rho_pos;
	const double
		s_neg = (vx_neg <= vx_pos) ? vx_neg - fast : vx_pos - fast,
		s_pos = (vx_neg <= vx_pos) ? vx_pos + fast : vx_neg + fast;
	if (s_neg >= 0.0) {
		out.speed = std::fabs(s_pos);
	} else if (s_pos <= 0.0) {
		out.speed = std::fabs(s_neg);
	} else {
		out.speed = std::max(std::fabs(s_neg), std::fabs(s_pos));
	}
	return out;
}

// dispatch of mhd/solve.hpp:135-154
struct Restated_Solvers {
	Face_Flux operator()(
		const int solver, const MHD& neg, const MHD& pos, const Vec3& bg,
		const double gamma, const double mu0
	) const {
		switch (solver) {
		case PAMHD_RUSANOV: return get_flux_rusanov(neg, pos, bg, gamma, mu0);
		case PAMHD_HLL_ATHENA: return get_flux_hll(neg, pos, bg, gamma, mu0);
		case PAMHD_HLLD_ATHENA: return get_flux_hlld(neg, pos, bg, gamma, mu0);
		case PAMHD_ROE_ATHENA: return get_flux_roe(neg, pos, bg, gamma, mu0);
		default: throw std::invalid_argument("invalid solver");
		}
	}
};

} // namespace oracle

#endif
