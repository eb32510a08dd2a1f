/*
A C++ host program that drives the library through its C ABI only, the way
a PAMHD program replaces its MHD step (tests/mhd/test.cpp:462-530): set the
initial state, take the dt = 0 priming step, step to the end time with the
time left as the cap, report the result and write it as a .dc file.

    abi_driver <solver id> <cells> <output.dc>

The workload is the Brio-Wu shock tube: cells on [0, 1], gamma 2, mu0 1,
CFL 0.5, copy boundaries, t = 0 .. 0.1; left rho 1, p 1, B (0.75, 1, 0),
right rho 0.125, p 0.1, B (0.75, -1, 0).  Every step's dt is checked against
the one computed here from the previous step's max_signal output.  Prints
"steps time rho_sum" and exits 0, or prints the error and exits 1.
*/
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "pamhd_gpu.h"

namespace {

int fail(const char* what, const int rc)
{
	std::fprintf(stderr, "%s: %s\n", what, pamhd_gpu_errstr(rc));
	return 1;
}

// total energy density at rest (mu0 = 1)
double total_energy(const double p, const double bx, const double by, const double gamma)
{
	return p / (gamma - 1) + 0.5 * (bx * bx + by * by);
}

} // namespace

int main(int argc, char** argv)
{
	if (argc != 4) {
		std::fprintf(stderr, "usage: %s <solver id> <cells> <output.dc>\n", argv[0]);
		return 2;
	}
	const int solver = std::atoi(argv[1]), n = std::atoi(argv[2]);
	const double gamma = 2.0, t_end = 0.1;

	pamhd_cfg cfg{};
	cfg.n[0] = n;
	cfg.n[1] = cfg.n[2] = 1;
	cfg.solver = solver;
	cfg.cell_length[0] = 1.0 / n;
	cfg.cell_length[1] = cfg.cell_length[2] = 1.0;
	cfg.adiabatic_index = gamma;
	cfg.vacuum_permeability = 1.0;
	cfg.time_step_factor = 0.5;
	cfg.bc_lo[0] = cfg.bc_hi[0] = PAMHD_BC_COPY;
	cfg.device = 0;
	pamhd_ctx* ctx = nullptr;
	int rc = pamhd_gpu_create(&cfg, &ctx);
	if (rc != PAMHD_OK) return fail("pamhd_gpu_create", rc);

	std::vector<std::vector<double>> U(8, std::vector<double>(n, 0.0));
	for (int i = 0; i < n; i++) {
		const bool left = (i + 0.5) / n < 0.5;
		const double rho = left ? 1.0 : 0.125, p = left ? 1.0 : 0.1, by = left ? 1.0 : -1.0;
		U[0][i] = rho;
		U[4][i] = total_energy(p, 0.75, by, gamma);
		U[5][i] = 0.75;
		U[6][i] = by;
	}
	const double* in[8];
	double* out[8];
	for (int v = 0; v < 8; v++) {
		in[v] = U[v].data();
		out[v] = U[v].data();
	}
	rc = pamhd_gpu_set_state(ctx, in);
	if (rc != PAMHD_OK) return fail("pamhd_gpu_set_state", rc);

	// the priming step, then steps capped by the time left, as the reference's time loop
	double t = 0.0, dt = 0.0, signal[3] = {0.0, 0.0, 0.0};
	rc = pamhd_gpu_step(ctx, 0.0, &dt, signal);
	if (rc != PAMHD_OK) return fail("pamhd_gpu_step", rc);
	uint64_t steps = 0;
	while (t < t_end) {
		// the step's dt from the previous step's largest face speed, as a caller with its own
		// timestep logic computes it (mhd/solve.hpp:1983-2003, capped as substepping.hpp:331-338)
		double expect = signal[0] > 0.0 ? (cfg.time_step_factor * cfg.cell_length[0]) / signal[0] : 0.0;
		if (t_end - t <= expect) expect = t_end - t;
		rc = pamhd_gpu_step(ctx, t_end - t, &dt, signal);
		if (rc == PAMHD_OK and dt != expect) {
			std::fprintf(stderr, "step %llu: dt %.17g, from max_signal %.17g\n",
			             static_cast<unsigned long long>(steps), dt, expect);
			return 1;
		}
		if (rc == PAMHD_ERR_PHYSICS) {
			uint32_t flags = 0;
			int32_t cell[3], dir = 0;
			pamhd_gpu_status(ctx, &flags, cell, &dir);
			std::fprintf(stderr, "solver failed at cell %d, face %d, flags %u\n", cell[0], dir, flags);
			return 1;
		}
		if (rc != PAMHD_OK) return fail("pamhd_gpu_step", rc);
		t += dt;
		steps++;
	}
	rc = pamhd_gpu_get_state(ctx, out);
	if (rc != PAMHD_OK) return fail("pamhd_gpu_get_state", rc);

	pamhd_dc_info info{};
	info.step = steps;
	info.time = t;
	info.adiabatic_index = gamma;
	info.proton_mass = 1.0;
	info.vacuum_permeability = 1.0;
	info.n[0] = n;
	info.n[1] = info.n[2] = 1;
	info.periodic[1] = info.periodic[2] = 1;
	info.cell_length[0] = 1.0 / n;
	info.cell_length[1] = info.cell_length[2] = 1.0;
	const double* cout_[8];
	for (int v = 0; v < 8; v++) cout_[v] = U[v].data();
	rc = pamhd_dc_write(argv[3], &info, cout_);
	if (rc != PAMHD_OK) return fail("pamhd_dc_write", rc);

	double mass = 0.0;
	for (int i = 0; i < n; i++) mass += U[0][i];
	std::printf("%llu %.17g %.17g\n", static_cast<unsigned long long>(steps), t, mass / n);
	pamhd_gpu_destroy(ctx);
	return 0;
}
