/*
Host build of the face adjoint (pamhd_b200/csrc/adjoint_face.cuh) for the
CPU tests: the same source the GPU kernels inline, compiled by g++, so that
the hand-written reverse mode can be checked against finite differences of
the oracle without a GPU.  Test infrastructure; not part of the library.
*/
#include <cstdint>

#include "../../pamhd_b200/csrc/adjoint_face.cuh"

extern "C" void adj_face_vjp(int32_t solver, int64_t n, const double* UL, const double* UR, double gamma,
                             double mu0, const double* phi, double* gL, double* gR, double* F)
{
	pamhd_b200::adjoint::Gas_Adj g;
	g.gamma = gamma;
	g.inv_mu0 = 1.0 / mu0;
	g.sqrt_mu0 = std::sqrt(mu0);
	g.inv_sqrt_mu0 = 1.0 / g.sqrt_mu0;
	for (int64_t i = 0; i < n; i++) {
		const double* a = UL + 8 * i;
		const double* b = UR + 8 * i;
		const double* p = phi + 8 * i;
		double* x = gL + 8 * i;
		double* y = gR + 8 * i;
		double* f = F + 8 * i;
		switch (solver) {
		case 0: pamhd_b200::adjoint::face_vjp<0>(a, b, g, p, x, y, f); break;
		case 2: pamhd_b200::adjoint::face_vjp<2>(a, b, g, p, x, y, f); break;
		case 3: pamhd_b200::adjoint::face_vjp<3>(a, b, g, p, x, y, f); break;
		default: pamhd_b200::adjoint::face_vjp<4>(a, b, g, p, x, y, f); break;
		}
	}
}
