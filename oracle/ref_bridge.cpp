/*
libpamhd_ref.so: the reference's OWN solver headers (mhd/rusanov.hpp,
mhd/hll_athena.hpp, mhd/hlld_athena.hpp, mhd/roe_athena.hpp), compiled
unchanged from the reference tree by oracle/Makefile, behind the same C
entry points as liboracle.so (prefix ref_) and the same Mode C grid
restatement.  It pins the oracle's restated solvers and is the timed
"reference" CPU baseline: the reference solver code on the host's cores.

TEST INFRASTRUCTURE - see mhd_oracle.hpp for who may use this.

Built with the stand-ins in ref_shim/ (gensimcell container, variable tags).
*/
#include "mhd/rusanov.hpp"
#include "mhd/hll_athena.hpp"
#include "mhd/hlld_athena.hpp"
#include "mhd/roe_athena.hpp"
#include "mhd/N_rusanov.hpp"
#include "mhd/N_hll_athena.hpp"

#include "n_solve.hpp"

namespace {

// calls the reference's solver templates the way mhd/solve.hpp:122-155 does
struct Reference_Solvers {
	oracle::Face_Flux operator()(
		const int solver, const oracle::MHD& neg, const oracle::MHD& pos,
		const oracle::Vec3& bg, const double gamma, const double mu0
	) const {
		using pamhd::mhd::detail::MHD;
		const pamhd::mhd::Mass_Density Mas{};
		const pamhd::mhd::Momentum_Density Mom{};
		const pamhd::mhd::Total_Energy_Density Nrj{};
		const pamhd::Magnetic_Field Mag{};
		MHD a, b;
		a[Mas] = neg.rho; a[Mom] = neg.mom; a[Nrj] = neg.nrj; a[Mag] = neg.mag;
		b[Mas] = pos.rho; b[Mom] = pos.mom; b[Nrj] = pos.nrj; b[Mag] = pos.mag;
		const std::array<double, 3> bg_face{bg[0], bg[1], bg[2]};
		MHD f;
		double s = -1;
		try {
			#define REF_SOLVER(name) name< \
				pamhd::mhd::Mass_Density, pamhd::mhd::Momentum_Density, \
				pamhd::mhd::Total_Energy_Density, pamhd::Magnetic_Field>( \
				a, b, bg_face, gamma, mu0)
			switch (solver) {
			case PAMHD_RUSANOV: std::tie(f, s) = REF_SOLVER(pamhd::mhd::get_flux_rusanov); break;
			case PAMHD_HLL_ATHENA: std::tie(f, s) = REF_SOLVER(pamhd::mhd::athena::get_flux_hll); break;
			case PAMHD_HLLD_ATHENA: std::tie(f, s) = REF_SOLVER(pamhd::mhd::athena::get_flux_hlld); break;
			case PAMHD_ROE_ATHENA: std::tie(f, s) = REF_SOLVER(pamhd::mhd::athena::get_flux_roe); break;
			default: throw std::invalid_argument("invalid solver");
			}
			#undef REF_SOLVER
		} catch (const std::domain_error& e) {
			// the reference throws plain std::domain_error; classify by its message
			const std::string w = e.what();
			uint32_t flag = PAMHD_FLAG_WAVE_SPEED;
			auto has = [&w](const char* text) { return w.find(text) != std::string::npos; };
			if (has("intermediate")) {
				flag = has("density") ? PAMHD_FLAG_ROE_DENSITY : PAMHD_FLAG_ROE_PRESSURE;
			} else if (has("mass density flux") or has("momentum x density")) {
				flag = PAMHD_FLAG_FLUX;
			} else if (has("mass density")) {
				flag = PAMHD_FLAG_DENSITY;
			} else if (has("pressure")) {
				flag = PAMHD_FLAG_PRESSURE;
			}
			throw oracle::Domain_Error(flag, w);
		}
		oracle::Face_Flux out;
		out.flux.rho = f[Mas];
		out.flux.mom = f[Mom];
		out.flux.nrj = f[Nrj];
		out.flux.mag = f[Mag];
		out.speed = s;
		return out;
	}
};

// calls the reference's two-population split solvers the way mhd/N_solve.hpp:290-320 does
struct Reference_Split_Solvers {
	oracle::Split_Flux operator()(
		const int solver, const oracle::MHD& neg, const oracle::MHD& pos, const oracle::Vec3& bg,
		const double area, const double dt, const double gamma, const double mu0
	) const {
		using pamhd::mhd::detail::MHD;
		const pamhd::mhd::Mass_Density Mas{};
		const pamhd::mhd::Momentum_Density Mom{};
		const pamhd::mhd::Total_Energy_Density Nrj{};
		const pamhd::Magnetic_Field Mag{};
		MHD a, b;
		a[Mas] = neg.rho; a[Mom] = neg.mom; a[Nrj] = neg.nrj; a[Mag] = neg.mag;
		b[Mas] = pos.rho; b[Mom] = pos.mom; b[Nrj] = pos.nrj; b[Mag] = pos.mag;
		const std::array<double, 3> bg_face{bg[0], bg[1], bg[2]};
		MHD fn, fp;
		double s = -1;
		try {
			#define REF_SPLIT(name) name< \
				pamhd::mhd::Mass_Density, pamhd::mhd::Momentum_Density, \
				pamhd::mhd::Total_Energy_Density, pamhd::Magnetic_Field>( \
				a, b, bg_face, area, dt, gamma, mu0)
			switch (solver) {
			case PAMHD_RUSANOV: std::tie(fn, fp, s) = REF_SPLIT(pamhd::mhd::get_flux_N_rusanov); break;
			case PAMHD_HLL_ATHENA: std::tie(fn, fp, s) = REF_SPLIT(pamhd::mhd::athena::get_flux_N_hll); break;
			default: throw std::invalid_argument("the two-population step has Rusanov and HLL only");
			}
			#undef REF_SPLIT
		} catch (const std::domain_error& e) {
			const std::string w = e.what();
			uint32_t flag = PAMHD_FLAG_WAVE_SPEED;
			auto has = [&w](const char* text) { return w.find(text) != std::string::npos; };
			if (has("mass density flux") or has("momentum x density")) {
				flag = PAMHD_FLAG_FLUX;
			} else if (has("mass density")) {
				flag = PAMHD_FLAG_DENSITY;
			} else if (has("pressure")) {
				flag = PAMHD_FLAG_PRESSURE;
			}
			throw oracle::Domain_Error(flag, w);
		}
		oracle::Split_Flux out;
		out.neg.rho = fn[Mas]; out.neg.mom = fn[Mom]; out.neg.nrj = fn[Nrj]; out.neg.mag = fn[Mag];
		out.pos.rho = fp[Mas]; out.pos.mom = fp[Mom]; out.pos.nrj = fp[Nrj]; out.pos.mag = fp[Mag];
		out.speed = s;
		return out;
	}
};

} // namespace

#define ORACLE_API(name) ref_##name
#define ORACLE_FLUX Reference_Solvers
#define ORACLE_SPLIT Reference_Split_Solvers
#include "capi_body.hpp"
