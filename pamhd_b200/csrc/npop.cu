/*
The two-population MHD step (the reference's N_solve + apply_fluxes_N,
mhd/N_solve.hpp:79-587) on uniform grids periodic in every dimension,
behind pamhd_gpu_npop_* of include/pamhd_gpu.h.

Two fluid populations share one magnetic field.  Every face is solved for
the total state of its two cells with a split solver that returns the flux
leaving the negative side and the flux entering from the positive side
(times area and dt): get_flux_N_rusanov (mhd/N_rusanov.hpp:61-170) or
get_flux_N_hll (mhd/N_hll_athena.hpp:47-231, with the reference's second
scaling of the positive side's momentum flux and its unscaled field flux,
:224-227).  Each side's mass, momentum and energy flux goes to the
populations by that side's mass fractions, the field flux is the sum of
the two sides' (mhd/N_solve.hpp:354-437).  Dimensions of one cell have no
faces.

Data in HBM: 13 arrays (rho1, mom1 xyz, E1, rho2, mom2 xyz, E2, B xyz) of
n0 n1 n2 doubles, x fastest, no ghosts (neighbours wrap), ping-pong.

One step, one fused launch (npop_fused_kernel, described below) and a
one-flag check (restore_kernel):
  dt (given, or min(CFL max_dt, t_end - t) from the previous step's face
  speeds, the loop of tests/mhd/two_reference.cpp:936-960); every face
  solved once from per-cell records staged in shared memory by z-marching
  tiles (the fast speed of a cell along each axis computed once, not once
  per face side), its contributions summed by the cells on both sides in
  the order -x, +x, -y, +y, -z, +z, applied times 1/volume (apply_fluxes_N,
  mhd/N_solve.hpp:505-546) with the total pressure raised to min_pressure
  where it is below (:553-583); the signal speeds max-reduced per axis into
  a three-slot ring; the clock advanced.
The next step's limit is min over axes of d_len / max signal speed
(mhd/N_solve.hpp:345).  Every operation is written in the order of the CPU
oracle's restatement (oracle/n_solve.hpp) and the file is compiled without
FMA contraction: +, -, *, / and sqrt round the same on both, so the GPU
computes the oracle's bits.
*/
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <new>

#include "pamhd_gpu.h"
#include "step.cuh"

using namespace pamhd_b200;

namespace {

constexpr int THREADS = 256;
constexpr int NV = 13;

struct Npop_Control {
	double dt;       // >= 0: the step's dt; < 0: min(cfl max_dt, t_end - t)
	double cfl;
	double t_end;
};

struct Npop_Params {
	const double* __restrict__ U;   // 13 x N
	double* __restrict__ Uo;
	int n[3];
	int active[3];
	long long N;
	double len[3];
	double area[3];
	double gamma, mu0, min_pressure;
	double inv_mu0, half_inv_mu0;   // 1 / mu0 and 0.5 / mu0
	Speed_Max* red;                 // [3] ring by step phase: max signal speed per axis
	Clock* clock;                   // [3]
	Status* status;
	Npop_Control control;
	int phase;
	int kchunk;                     // z planes per face-solve block
};

/*
A total state: mass, momentum, energy, field, with inv = 1 / rho and
half = 0.5 / rho divided once per cell (the same IEEE divisions as the
expressions they stand for, so the same bits).
*/
struct St {
	double rho, m[3], e, b[3];
	double inv, half;
};

// the run's constants, 1 / mu0 and 0.5 / mu0 divided once (on the host: IEEE division, the same bits)
struct Gas_N {
	double gamma, mu0, inv_mu0, half_inv_mu0;
};

__device__ __forceinline__ void set_reciprocals(St& s)
{
	s.inv = 1 / s.rho;
	s.half = 0.5 / s.rho;
}

__device__ __forceinline__ double max_of(const double a, const double b)
{
	return (a < b) ? b : a;   // std::max
}

__device__ __forceinline__ double min_of(const double a, const double b)
{
	return (b < a) ? b : a;   // std::min
}

// get_pressure (mhd/common.hpp:79-118); rho <= 0 is the reference's throw
__device__ __forceinline__ double pressure(const St& s, const Gas_N& g, uint32_t& flag)
{
	if (s.rho <= 0 and flag == 0) flag = PAMHD_FLAG_DENSITY;
	const double
		kinetic = s.half * (s.m[0] * s.m[0] + s.m[1] * s.m[1] + s.m[2] * s.m[2]),
		magnetic = g.half_inv_mu0 * (s.b[0] * s.b[0] + s.b[1] * s.b[1] + s.b[2] * s.b[2]);
	return (s.e - kinetic - magnetic) * (g.gamma - 1);
}

// get_velocity (mhd/common.hpp:121-130)
__device__ __forceinline__ void velocity(const St& s, double v[3])
{
	if (s.rho > 0) {
		v[0] = s.m[0] * s.inv;
		v[1] = s.m[1] * s.inv;
		v[2] = s.m[2] * s.inv;
	} else {
		v[0] = v[1] = v[2] = 0;
	}
}

// get_fast_magnetosonic_speed without background field (mhd/common.hpp:418-491)
__device__ double fast_speed(const St& s, const Gas_N& g, uint32_t& flag)
{
	const double t0 = s.b[0] + 0.0, t1 = s.b[1] + 0.0, t2 = s.b[2] + 0.0;
	if (not is_finite(t0)) {
		if (flag == 0) flag = PAMHD_FLAG_WAVE_SPEED;
		return 0;
	}
	const double b = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
	// get_sound_speed
	if (not (is_normal(s.rho) and not (s.rho < 0))) {
		if (flag == 0) flag = PAMHD_FLAG_DENSITY;
		return 0;
	}
	const double p = pressure(s, g, flag);
	if (not (is_normal(p) and not (p < 0))) {
		if (flag == 0) flag = PAMHD_FLAG_PRESSURE;
		return 0;
	}
	const double sound = sqrt(g.gamma * p / s.rho);
	if (b <= 0) return sound;
	// get_alfven_speed
	const double bb = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
	const double alfven = bb / sqrt(g.mu0 * s.rho);
	const double sound2 = sound * sound, alfven2 = alfven * alfven, sum2 = sound2 + alfven2;
	if (not (is_normal(sum2) and not (sum2 < 0))) {
		if (flag == 0) flag = PAMHD_FLAG_WAVE_SPEED;
		return 0;
	}
	const double cos_b = t0 / b;
	const double to_sqrt = sound2 * sound2 + alfven2 * alfven2 + 2 * sound2 * alfven2 * (1 - 2 * (cos_b * cos_b));
	if (not (is_normal(to_sqrt) and not (to_sqrt < 0))) {
		if (flag == 0) flag = PAMHD_FLAG_WAVE_SPEED;
		return 0;
	}
	return sqrt(0.5 * (sum2 + sqrt(to_sqrt)));
}

// get_flux without background field (mhd/common.hpp:146-244), the physical flux along x
__device__ void physical(const St& s, const Gas_N& g, double F[8], uint32_t& flag)
{
	if (not (is_normal(s.rho) and s.rho > 0)) {
		if (flag == 0) flag = PAMHD_FLAG_DENSITY;
		return;
	}
	if (not is_finite(s.m[0])) {
		if (flag == 0) flag = PAMHD_FLAG_FLUX;
		return;
	}
	const double bg = 0.0;
	const double tot[3] = {s.b[0] + bg, s.b[1] + bg, s.b[2] + bg};
	const double
		inv_mu0 = g.inv_mu0,
		p_bg = 0.5 * inv_mu0 * (bg * bg + bg * bg + bg * bg),
		p_b1 = 0.5 * inv_mu0 * (s.b[0] * s.b[0] + s.b[1] * s.b[1] + s.b[2] * s.b[2]),
		p_tot = 0.5 * inv_mu0 * (tot[0] * tot[0] + tot[1] * tot[1] + tot[2] * tot[2]),
		p_th = pressure(s, g, flag);
	double v[3];
	velocity(s, v);
	F[0] = s.m[0];
	if (not is_finite(F[0])) {
		if (flag == 0) flag = PAMHD_FLAG_FLUX;
		return;
	}
	#pragma unroll
	for (int i = 0; i < 3; i++) F[1 + i] = s.m[i] * v[0] + (-inv_mu0) * (tot[0] * tot[i] + (-bg) * bg);
	F[1] += p_th + p_tot - p_bg;
	double vb = 0;
	vb += v[0] * s.b[0];
	vb += v[1] * s.b[1];
	vb += v[2] * s.b[2];
	F[4] = v[0] * (s.e + p_th + p_b1)
		- s.b[0] * vb * inv_mu0
		+ inv_mu0 * (
			s.b[1] * (v[0] * bg - v[1] * bg)
			+ s.b[2] * (v[0] * bg - v[2] * bg));
	#pragma unroll
	for (int i = 0; i < 3; i++) F[5 + i] = v[0] * tot[i] + (-tot[0]) * v[i];
	F[5] = 0;
}

__device__ __forceinline__ void state_row(const St& s, double u[8])
{
	u[0] = s.rho; u[1] = s.m[0]; u[2] = s.m[1]; u[3] = s.m[2];
	u[4] = s.e; u[5] = s.b[0]; u[6] = s.b[1]; u[7] = s.b[2];
}

/*
The fast speed of a side along the face normal is computed once per cell and
axis (fast_speed of the rotated total state, with the flag it raises from a
clear start); the split solvers take it with that flag.
*/
struct Fast {
	double speed;
	uint32_t flag;
};

// get_flux_N_rusanov (mhd/N_rusanov.hpp:61-170)
__device__ double split_rusanov(const St& L, const St& R, const Fast& fl, const Fast& fr, const double area,
                                const double dt, const Gas_N& g, double fn[8], double fp[8], uint32_t& flag)
{
	if (not (is_normal(L.rho) and not (L.rho < 0)) or not (is_normal(R.rho) and not (R.rho < 0))) {
		flag = PAMHD_FLAG_DENSITY;
		return 0;
	}
	flag = fl.flag;
	if (flag) return 0;
	const double fast_neg = fl.speed;
	flag = fr.flag;
	if (flag) return 0;
	const double fast_pos = fr.speed;
	const double max_fast = max_of(fast_neg, fast_pos);
	double vl[3], vr[3];
	velocity(L, vl);
	velocity(R, vr);
	const double s = max_of(fabs(vl[0]) + max_fast, fabs(vr[0]) + max_fast);
	double FL[8], FR[8];
	physical(L, g, FL, flag);
	if (flag) return 0;
	physical(R, g, FR, flag);
	if (flag) return 0;
	double uL[8], uR[8];
	state_row(L, uL);
	state_row(R, uR);
	const double c = 0.5 * area * dt;
	fn[0] = c * (FL[0] + uL[0] * s);
	#pragma unroll
	for (int i = 1; i <= 3; i++) fn[i] = c * (FL[i] + uL[i] * s);
	fn[4] = c * (FL[4] + uL[4] * s);
	#pragma unroll
	for (int i = 5; i <= 7; i++) fn[i] = c * (FL[i] + uL[i] * s);
	fp[0] = c * (FR[0] - uR[0] * s);
	#pragma unroll
	for (int i = 1; i <= 3; i++) fp[i] = c * (FR[i] + uR[i] * -s);
	fp[4] = c * (FR[4] - uR[4] * s);
	#pragma unroll
	for (int i = 5; i <= 7; i++) fp[i] = c * (FR[i] + uR[i] * -s);
	return s;
}

// get_flux_N_hll (mhd/N_hll_athena.hpp:47-231)
__device__ double split_hll(const St& L, const St& R, const Fast& fl, const Fast& fr, const double area,
                            const double dt, const Gas_N& g, double fn[8], double fp[8], uint32_t& flag)
{
	double vn[3], vp[3];
	velocity(L, vn);
	velocity(R, vp);
	const double p_neg = pressure(L, g, flag);
	const double p_pos = pressure(R, g, flag);
	if (flag) return 0;
	const double
		pb_neg = (L.b[0] * L.b[0] + L.b[1] * L.b[1] + L.b[2] * L.b[2]) / (2 * g.mu0),
		pb_pos = (R.b[0] * R.b[0] + R.b[1] * R.b[1] + R.b[2] * R.b[2]) / (2 * g.mu0);
	flag = fl.flag;
	if (flag) return 0;
	const double fast_neg = fl.speed;
	flag = fr.flag;
	if (flag) return 0;
	const double fast_pos = fr.speed;
	const double
		max_signal = max_of(fast_neg, fast_pos),
		s_neg = (vn[0] <= vp[0]) ? vn[0] - max_signal : vp[0] - max_signal,
		s_pos = (vn[0] <= vp[0]) ? vp[0] + max_signal : vn[0] + max_signal,
		bm = min_of(s_neg, 0.0),
		bp = max_of(s_pos, 0.0);
	if (not (is_normal(p_neg) and not (p_neg < 0)) or not (is_finite(pb_neg) and not (pb_neg < 0))) {
		flag = PAMHD_FLAG_PRESSURE;
		return 0;
	}
	if (not is_finite(s_neg)) {
		flag = PAMHD_FLAG_WAVE_SPEED;
		return 0;
	}
	if (not (is_normal(p_pos) and not (p_pos < 0)) or not (is_finite(pb_pos) and not (pb_pos < 0))) {
		flag = PAMHD_FLAG_PRESSURE;
		return 0;
	}
	if (not is_finite(s_pos)) {
		flag = PAMHD_FLAG_WAVE_SPEED;
		return 0;
	}
	if (not (is_normal(bp - bm) and not (bp - bm < 0))) {
		#pragma unroll
		for (int i = 0; i < 8; i++) fn[i] = fp[i] = 0;
		return 0;
	}
	double FL[8], FR[8];
	physical(L, g, FL, flag);
	if (flag) return 0;
	physical(R, g, FR, flag);
	if (flag) return 0;
	double uL[8], uR[8];
	state_row(L, uL);
	state_row(R, uR);
	const double
		neg_factor = bp / (bp - bm) * area * dt,
		pos_factor = bm / (bm - bp) * area * dt;
	fn[0] = neg_factor * (FL[0] - uL[0] * bm);
	#pragma unroll
	for (int i = 1; i <= 3; i++) fn[i] = neg_factor * (FL[i] + uL[i] * -bm);
	fn[4] = neg_factor * (FL[4] - uL[4] * bm);
	#pragma unroll
	for (int i = 5; i <= 7; i++) fn[i] = neg_factor * (FL[i] + uL[i] * -bm);
	fp[0] = pos_factor * (FR[0] - uR[0] * bp);
	#pragma unroll
	for (int i = 1; i <= 3; i++) fp[i] = pos_factor * (FR[i] + uR[i] * -bp);
	fp[4] = pos_factor * (FR[4] - uR[4] * bp);
	// as the reference: the positive side's momentum flux scaled a second time, its field flux unscaled
	#pragma unroll
	for (int i = 1; i <= 3; i++) fp[i] = pos_factor * (fp[i] + uR[i] * -bp);
	#pragma unroll
	for (int i = 5; i <= 7; i++) fp[i] = FR[i];
	return max_of(fabs(bp), fabs(bm));
}

__device__ __forceinline__ long long wrap(const Npop_Params& P, int i, int j, int k)
{
	i = i < 0 ? i + P.n[0] : (i >= P.n[0] ? i - P.n[0] : i);
	j = j < 0 ? j + P.n[1] : (j >= P.n[1] ? j - P.n[1] : j);
	k = k < 0 ? k + P.n[2] : (k >= P.n[2] ? k - P.n[2] : k);
	return (long long)i + (long long)P.n[0] * ((long long)j + (long long)P.n[1] * k);
}

__device__ __forceinline__ void load13(const Npop_Params& P, const long long c, double u[NV])
{
	#pragma unroll
	for (int v = 0; v < NV; v++) u[v] = P.U[v * P.N + c];
}

// the total state of a cell, rotated into the frame of axis A (get_rotated_vector, mhd/common.hpp:612-648),
// with the reciprocals of its density given
template <int A>
__device__ __forceinline__ St total_rotated(const double u[NV], const double inv, const double half)
{
	St s;
	s.inv = inv;
	s.half = half;
	s.rho = u[0] + u[5];
	const double m[3] = {u[1] + u[6], u[2] + u[7], u[3] + u[8]};
	s.e = u[4] + u[9];
	rotate<A>(m[0], m[1], m[2], s.m[0], s.m[1], s.m[2]);
	rotate<A>(u[10], u[11], u[12], s.b[0], s.b[1], s.b[2]);
	return s;
}

// the step's dt: given, or min(CFL max_dt, t_end - t) with max_dt from the previous step's speeds
__device__ __forceinline__ double step_dt(const Npop_Params& P)
{
	if (P.control.dt >= 0.0) return P.control.dt;
	const Speed_Max& r = P.red[P.phase];
	double max_dt = DBL_MAX;
	if (r.zero == 0u) {
		#pragma unroll
		for (int d = 0; d < 3; d++) {
			const double s = __longlong_as_double((long long)r.smax[d]);
			if (P.active[d] and s > 0.0) max_dt = min_of(max_dt, P.len[d] / s);
		}
	} else {
		max_dt = 0.0;   // no speeds yet: the first step of the loop has dt 0
	}
	const double until_end = P.control.t_end - P.clock[P.phase].t;
	return min_of(P.control.cfl * max_dt, until_end);
}

__device__ __forceinline__ double warp_max(double v)
{
	#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
	return v;
}

/*
One fused launch per step: a block of NTX x NTY threads owns a column of
cells and marches it in z through a chunk of planes.  Per plane k:
  (a) the plane's cells, with the columns left and right of the tile and the
      rows below and above it, are read once into a shared-memory record (the
      13 state values, the two density reciprocals and, per active axis, the
      fast speed of the rotated total state with its check flag);
  (b) every cell solves its -x and -y faces from the records (the tile's
      +x faces by four lanes of warp 2, its +y faces by the last row) and
      its -z face against its own record of plane k - 1, kept in registers;
  (c) the x and y contributions go through shared memory to the cells on
      their other side, and every cell sums its faces' contributions in the
      order -x, +x, -y, +y, -z (the +z one arrives with plane k + 1);
  (d) the cell of plane k - 1 takes its +z contribution and is updated as
      apply_fluxes_N does (mhd/N_solve.hpp:505-583) and written out.
The contributions never reach HBM.  A face that fails sets the status; the
step's state is then restored by restore_kernel after the launch, as the
reference stops before applying any flux of that step.  Partial tiles read
wrapped cells in their unused positions (computed, not written), so that
every owned cell's neighbours are the right ones.
*/
constexpr int NTX = 32, NTY = 4;
constexpr int NW = NTX + 2;                 // a record row: halo columns at 0 and NTX + 1
constexpr int NH = NTY + 2;                 // record rows: halo rows at 0 and NTY + 1
constexpr int NCELLS = NW * NH;
constexpr int NREC = NV + 5;                // state, fast speed along x, y, z, 1 / rho, 0.5 / rho
enum { N_CF = NV, N_INV = NV + 3, N_HALF = NV + 4 };
constexpr int NXF = (NTX + 1) * NTY;        // x faces of the tile: the -x face of every column and the last +x
constexpr int NYF = NTX * (NTY + 1);        // y faces: the -y face of every row and the last +y
constexpr size_t SMEM_RECORDS = size_t(NREC) * NCELLS * sizeof(double) + NCELLS * sizeof(uint32_t);
constexpr size_t SMEM_EXCHANGE = size_t(NV) * (NXF + NYF) * sizeof(double);
constexpr size_t SMEM_PENDING = size_t(NV) * NTX * NTY * sizeof(double);   // the sums waiting for +z
constexpr size_t SMEM_FUSED = SMEM_RECORDS + SMEM_EXCHANGE + SMEM_PENDING;

__device__ __forceinline__ Gas_N gas_of(const Npop_Params& P)
{
	return Gas_N{P.gamma, P.mu0, P.inv_mu0, P.half_inv_mu0};
}

__device__ __forceinline__ int wrap_any(const int i, const int n)
{
	const int r = i % n;
	return r < 0 ? r + n : r;
}

// the fast speed of a cell's rotated total state along axis A, with its flag in byte A of flags
template <int A>
__device__ __forceinline__ double fast_of(const Npop_Params& P, const double u[NV], const double inv,
                                          const double half, uint32_t& flags)
{
	uint32_t f = 0;
	const double cf = fast_speed(total_rotated<A>(u, inv, half), gas_of(P), f);
	flags |= f << (8 * A);
	return cf;
}

// read cell c into record position r, with its fast speeds along the axes its faces in the tile need
template <bool CX, bool CY, bool CZ>
__device__ __forceinline__ void stage_cell(const Npop_Params& P, double* rec, uint32_t* flg, const int r,
                                           const long long c)
{
	double u[NV];
	load13(P, c, u);
	#pragma unroll
	for (int v = 0; v < NV; v++) rec[v * NCELLS + r] = u[v];
	const double rho = u[0] + u[5];
	const double inv = 1 / rho, half = 0.5 / rho;
	rec[N_INV * NCELLS + r] = inv;
	rec[N_HALF * NCELLS + r] = half;
	uint32_t flags = 0;
	if (CX and P.active[0]) rec[N_CF * NCELLS + r] = fast_of<0>(P, u, inv, half, flags);
	if (CY and P.active[1]) rec[(N_CF + 1) * NCELLS + r] = fast_of<1>(P, u, inv, half, flags);
	if (CZ and P.active[2]) rec[(N_CF + 2) * NCELLS + r] = fast_of<2>(P, u, inv, half, flags);
	flg[r] = flags;
}

// a cell as the -z side of a face, kept in registers from one plane to the next
struct Zrec {
	double u[NV];
	double inv, half, cf;
	uint32_t flag;
};

/*
The contribution x of the -A face between the cells with states um (left,
reciprocals iml / hml, fast speed fl) and uc (right): the split solver's two
fluxes, shared among the populations by each side's mass fractions, the
field flux the sum of the two sides' (mhd/N_solve.hpp:354-437), written to
x[v * stride].  Returns the failure flag (0: none); m names the face's
negative cell.
*/
template <int SOLVER, int A>
__device__ __forceinline__ uint32_t face_contribution(const Npop_Params& P, const double um[NV], const double iml,
                                                      const double hml, const Fast& fl, const double uc[NV],
                                                      const double imr, const double hmr, const Fast& fr,
                                                      const double dt, const long long m, double& smax,
                                                      double* x, const int stride)
{
	const St L = total_rotated<A>(um, iml, hml);
	const St R = total_rotated<A>(uc, imr, hmr);
	double fn[8], fp[8];
	uint32_t flag = 0;
	const double s = SOLVER == PAMHD_RUSANOV
		? split_rusanov(L, R, fl, fr, P.area[A], dt, gas_of(P), fn, fp, flag)
		: split_hll(L, R, fl, fr, P.area[A], dt, gas_of(P), fn, fp, flag);
	if (flag != 0) {
		atomicOr(&P.status->flags, flag);
		atomicMin(&P.status->first, ((unsigned long long)(m * 3 + A) << 8) | flag);
		#pragma unroll
		for (int v = 0; v < NV; v++) x[v * stride] = 0.0;
		return flag;
	}
	smax = fmax(smax, s);
	double gn[8], gp[8];
	gn[0] = fn[0]; gn[4] = fn[4]; gp[0] = fp[0]; gp[4] = fp[4];
	unrotate<A>(fn[1], fn[2], fn[3], gn[1], gn[2], gn[3]);
	unrotate<A>(fp[1], fp[2], fp[3], gp[1], gp[2], gp[3]);
	unrotate<A>(fn[5], fn[6], fn[7], gn[5], gn[6], gn[7]);
	unrotate<A>(fp[5], fp[6], fp[7], gp[5], gp[6], gp[7]);
	const double
		f1n = um[0] / (um[0] + um[5]), f2n = um[5] / (um[0] + um[5]),
		f1p = uc[0] / (uc[0] + uc[5]), f2p = uc[5] / (uc[0] + uc[5]);
	x[0] = f1n * gn[0] + f1p * gp[0];
	x[5 * stride] = f2n * gn[0] + f2p * gp[0];
	x[4 * stride] = f1n * gn[4] + f1p * gp[4];
	x[9 * stride] = f2n * gn[4] + f2p * gp[4];
	#pragma unroll
	for (int v = 0; v < 3; v++) {
		x[(1 + v) * stride] = f1n * gn[1 + v] + f1p * gp[1 + v];
		x[(6 + v) * stride] = f2n * gn[1 + v] + f2p * gp[1 + v];
		x[(10 + v) * stride] = gn[5 + v] + gp[5 + v];
	}
	return 0;
}

// the -A face between record positions rl and rr, its contribution to x[v * stride]
template <int SOLVER, int A>
__device__ __forceinline__ void record_face(const Npop_Params& P, const double* rec, const uint32_t* flg,
                                            const int rl, const int rr, const double dt, const long long m,
                                            double& smax, double* x, const int stride)
{
	double um[NV], uc[NV];
	#pragma unroll
	for (int v = 0; v < NV; v++) {
		um[v] = rec[v * NCELLS + rl];
		uc[v] = rec[v * NCELLS + rr];
	}
	const Fast fl{rec[(N_CF + A) * NCELLS + rl], (flg[rl] >> (8 * A)) & 0xffu};
	const Fast fr{rec[(N_CF + A) * NCELLS + rr], (flg[rr] >> (8 * A)) & 0xffu};
	face_contribution<SOLVER, A>(P, um, rec[N_INV * NCELLS + rl], rec[N_HALF * NCELLS + rl], fl, uc,
	                             rec[N_INV * NCELLS + rr], rec[N_HALF * NCELLS + rr], fr, dt, m, smax, x, stride);
}

// apply_fluxes_N for one cell (mhd/N_solve.hpp:505-583): the summed contributions f times 1 / volume,
// then the minimum total pressure
__device__ __forceinline__ void apply_cell(const Npop_Params& P, double u[NV], const double f[NV],
                                           const double inverse_volume)
{
	u[0] += f[0] * inverse_volume;
	u[5] += f[5] * inverse_volume;
	#pragma unroll
	for (int v = 1; v <= 3; v++) u[v] += f[v] * inverse_volume;
	#pragma unroll
	for (int v = 6; v <= 8; v++) u[v] += f[v] * inverse_volume;
	u[4] += f[4] * inverse_volume;
	u[9] += f[9] * inverse_volume;
	#pragma unroll
	for (int v = 10; v <= 12; v++) u[v] += f[v] * inverse_volume;
	St t;
	t.rho = u[0] + u[5];
	t.e = u[4] + u[9];
	t.m[0] = u[1] + u[6];
	t.m[1] = u[2] + u[7];
	t.m[2] = u[3] + u[8];
	t.b[0] = u[10];
	t.b[1] = u[11];
	t.b[2] = u[12];
	set_reciprocals(t);
	uint32_t flag = 0;
	const double p = pressure(t, gas_of(P), flag);
	if (not (p >= P.min_pressure)) {
		double v[3];
		velocity(t, v);
		const double
			kinetic = 0.5 * t.rho * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]),
			magnetic = 0.5 / P.mu0 * (t.b[0] * t.b[0] + t.b[1] * t.b[1] + t.b[2] * t.b[2]);
		const double e = P.min_pressure / (P.gamma - 1) + kinetic + magnetic;
		u[4] = u[0] / t.rho * e;
		u[9] = u[5] / t.rho * e;
	}
}

template <int SOLVER>
__global__ void __launch_bounds__(NTX * NTY, 3) npop_fused_kernel(const Npop_Params P)
{
	extern __shared__ __align__(16) double smem[];
	double* const rec = smem;
	uint32_t* const flg = reinterpret_cast<uint32_t*>(smem + NREC * NCELLS);
	double* const xch = reinterpret_cast<double*>(reinterpret_cast<char*>(smem) + SMEM_RECORDS);
	double* const ych = xch + NV * NXF;
	double* const pend = ych + NV * NYF;
	__shared__ double s_dt;
	__shared__ int s_skip;
	const int tx = threadIdx.x, ty = threadIdx.y;
	const int tid = ty * NTX + tx;
	if (tx == 0 and ty == 0) {
		const Clock c = P.clock[P.phase];
		// a failure in an earlier step leaves every later one as it is, as a run past t_end
		const bool skip = P.status->flags != 0u or (P.control.dt < 0.0 and c.t >= P.control.t_end);
		const double dt = skip ? 0.0 : step_dt(P);
		s_skip = skip ? 1 : 0;
		s_dt = dt;
		if (blockIdx.x == 0 and blockIdx.y == 0 and blockIdx.z == 0) {
			Clock& next = P.clock[(P.phase + 1) % 3];
			next.t = skip ? c.t : c.t + dt;
			next.dt = skip ? c.dt : dt;
			next.steps = skip ? c.steps : c.steps + 1;
			Speed_Max& z = P.red[(P.phase + 2) % 3];
			z.smax[0] = z.smax[1] = z.smax[2] = 0ull;
			z.zero = 0u;
		}
	}
	__syncthreads();
	const double dt = s_dt;
	const int nx = P.n[0], ny = P.n[1], nz = P.n[2];
	const int gx0 = blockIdx.x * NTX, gy0 = blockIdx.y * NTY;
	const int gx = gx0 + tx, gy = gy0 + ty;
	const bool own = gx < nx and gy < ny;
	const int kb = blockIdx.z * P.kchunk;
	const int ke = min(nz, kb + P.kchunk);
	const long long plane = (long long)nx * ny;
	const long long N = P.N;
	if (s_skip != 0) {
		if (own) {
			for (int k = kb; k < ke; k++) {
				const long long c = gx + (long long)nx * gy + plane * k;
				#pragma unroll
				for (int v = 0; v < NV; v++) P.Uo[v * N + c] = P.U[v * N + c];
			}
		}
		return;
	}
	const bool ax = P.active[0] != 0, ay = P.active[1] != 0, az = P.active[2] != 0;
	const int ri = (ty + 1) * NW + tx + 1;
	const int xi = ty * (NTX + 1) + tx;   // this cell's -x face in the exchange; +1 its +x face
	const int yi = ty * NTX + tx;         // this cell's -y face; + NTX its +y face
	// this position's cell (wrapped in a partial tile) and its halo cell, if any: warp 0 the row below
	// the tile, warp 1 the row above (their y speeds), warp 2 the columns left and right (x speeds)
	const int wx = wrap_any(gx, nx), wy = wrap_any(gy, ny);
	const long long col = wx + (long long)nx * wy;
	int hr = -1, haxis = 0;
	long long hcol = 0;
	if (ty == 0) {
		hr = tx + 1;
		hcol = wx + (long long)nx * wrap_any(gy0 - 1, ny);
		haxis = 1;
	} else if (ty == 1) {
		hr = (NTY + 1) * NW + tx + 1;
		hcol = wx + (long long)nx * wrap_any(gy0 + NTY, ny);
		haxis = 1;
	} else if (ty == 2 and tx < 2 * NTY) {
		const int row = tx % NTY;
		const bool left = tx < NTY;
		hr = (row + 1) * NW + (left ? 0 : NTX + 1);
		hcol = wrap_any(left ? gx0 - 1 : gx0 + NTX, nx) + (long long)nx * wrap_any(gy0 + row, ny);
		haxis = 0;
	}
	// the faces' negative cells (failure reports name them)
	const long long col_mx = wrap_any(gx - 1, nx) + (long long)nx * wy;
	const long long col_my = wx + (long long)nx * wrap_any(gy - 1, ny);
	const double inverse_volume = 1.0 / (P.len[0] * P.len[1] * P.len[2]);
	double s0 = 0.0, s1 = 0.0, s2 = 0.0;
	// the own cell of the plane before the chunk: the -z side of the first plane's -z faces
	Zrec zr;
	if (az) {
		load13(P, col + plane * wrap_any(kb - 1, nz), zr.u);
		const double rho = zr.u[0] + zr.u[5];
		zr.inv = 1 / rho;
		zr.half = 0.5 / rho;
		uint32_t f = 0;
		zr.cf = fast_of<2>(P, zr.u, zr.inv, zr.half, f);
		zr.flag = (f >> 16) & 0xffu;
	}
	for (int k = kb; k <= ke; k++) {
		const long long kofs = plane * wrap_any(k, nz);
		if (k < ke) {
			// (a) records
			stage_cell<true, true, true>(P, rec, flg, ri, col + kofs);
			if (hr >= 0) {
				if (haxis == 1) stage_cell<false, true, false>(P, rec, flg, hr, hcol + kofs);
				else stage_cell<true, false, false>(P, rec, flg, hr, hcol + kofs);
			}
			__syncthreads();
			// (b) the faces, straight into the exchange: own -x (and the last column's +x), own -y
			// (and the last row's +y)
			if (ax) {
				record_face<SOLVER, 0>(P, rec, flg, ri - 1, ri, dt, col_mx + kofs, s0, xch + xi, NXF);
				// the last column's +x faces: one lane per row of warp 2 (one extra pass for one warp,
				// instead of one for every warp with its last lane alone active)
				if (ty == 2 and tx < NTY) {
					const int rl = (tx + 1) * NW + NTX;
					const long long m = wrap_any(gx0 + NTX - 1, nx) + (long long)nx * wrap_any(gy0 + tx, ny);
					record_face<SOLVER, 0>(P, rec, flg, rl, rl + 1, dt, m + kofs, s0, xch + tx * (NTX + 1) + NTX, NXF);
				}
			}
			if (ay) {
				record_face<SOLVER, 1>(P, rec, flg, ri - NW, ri, dt, col_my + kofs, s1, ych + yi, NYF);
				if (ty == NTY - 1) record_face<SOLVER, 1>(P, rec, flg, ri, ri + NW, dt, col + kofs, s1, ych + yi + NTX, NYF);
			}
			// the -z face of this cell: its contribution closes the cell below and opens this one
			double xz[NV];
			if (az) {
				double uc[NV];
				#pragma unroll
				for (int v = 0; v < NV; v++) uc[v] = rec[v * NCELLS + ri];
				const Fast fl{zr.cf, zr.flag};
				const Fast fr{rec[(N_CF + 2) * NCELLS + ri], (flg[ri] >> 16) & 0xffu};
				face_contribution<SOLVER, 2>(P, zr.u, zr.inv, zr.half, fl, uc, rec[N_INV * NCELLS + ri],
				                             rec[N_HALF * NCELLS + ri], fr, dt, col + plane * wrap_any(k - 1, nz),
				                             s2, xz, 1);
				#pragma unroll
				for (int v = 0; v < NV; v++) zr.u[v] = uc[v];
				zr.inv = rec[N_INV * NCELLS + ri];
				zr.half = rec[N_HALF * NCELLS + ri];
				zr.cf = fr.speed;
				zr.flag = fr.flag;
			}
			__syncthreads();
			// (c) this cell's sum in the reference's order: -x, +x, -y, +y, -z
			double f[NV];
			#pragma unroll
			for (int v = 0; v < NV; v++) f[v] = 0;
			if (ax) {
				#pragma unroll
				for (int v = 0; v < NV; v++) {
					f[v] += xch[v * NXF + xi];
					f[v] -= xch[v * NXF + xi + 1];
				}
			}
			if (ay) {
				#pragma unroll
				for (int v = 0; v < NV; v++) {
					f[v] += ych[v * NYF + yi];
					f[v] -= ych[v * NYF + yi + NTX];
				}
			}
			if (az) {
				#pragma unroll
				for (int v = 0; v < NV; v++) f[v] += xz[v];
				// (d) the cell below takes its +z contribution and is updated
				if (k > kb and own) {
					const long long c = col + plane * (k - 1);
					double u[NV], g[NV];
					load13(P, c, u);
					#pragma unroll
					for (int v = 0; v < NV; v++) g[v] = pend[v * (NTX * NTY) + tid] - xz[v];
					apply_cell(P, u, g, inverse_volume);
					#pragma unroll
					for (int v = 0; v < NV; v++) P.Uo[v * N + c] = u[v];
				}
				#pragma unroll
				for (int v = 0; v < NV; v++) pend[v * (NTX * NTY) + tid] = f[v];
			} else if (own) {
				// no z faces: this plane's cells are complete
				const long long c = col + kofs;
				double u[NV];
				load13(P, c, u);
				apply_cell(P, u, f, inverse_volume);
				#pragma unroll
				for (int v = 0; v < NV; v++) P.Uo[v * N + c] = u[v];
			}
			// the records and the exchange are written again only after this barrier
			__syncthreads();
		} else if (az) {
			// the plane above the chunk: the last plane's +z faces
			double uc[NV], xz[NV];
			load13(P, col + kofs, uc);
			const double rho = uc[0] + uc[5];
			const double inv = 1 / rho, half = 0.5 / rho;
			uint32_t fflag = 0;
			const double cf = fast_of<2>(P, uc, inv, half, fflag);
			const Fast fl{zr.cf, zr.flag};
			const Fast fr{cf, (fflag >> 16) & 0xffu};
			face_contribution<SOLVER, 2>(P, zr.u, zr.inv, zr.half, fl, uc, inv, half, fr, dt,
			                             col + plane * (ke - 1), s2, xz, 1);
			if (own and ke > kb) {
				const long long c = col + plane * (ke - 1);
				double u[NV], g[NV];
				load13(P, c, u);
				#pragma unroll
				for (int v = 0; v < NV; v++) g[v] = pend[v * (NTX * NTY) + tid] - xz[v];
				apply_cell(P, u, g, inverse_volume);
				#pragma unroll
				for (int v = 0; v < NV; v++) P.Uo[v * N + c] = u[v];
			}
		}
	}
	s0 = warp_max(s0);
	s1 = warp_max(s1);
	s2 = warp_max(s2);
	if (tx == 0) {
		Speed_Max& r = P.red[(P.phase + 1) % 3];
		atomicMax(&r.smax[0], (unsigned long long)__double_as_longlong(s0));
		atomicMax(&r.smax[1], (unsigned long long)__double_as_longlong(s1));
		atomicMax(&r.smax[2], (unsigned long long)__double_as_longlong(s2));
	}
}

/*
After the fused launch: if a face has failed (in this step, or in an earlier
one, which the fused launch skipped), the step leaves the state and the
clock as they were: the reference stops before applying any flux of the
step.  One flag read per block otherwise.
*/
__global__ void __launch_bounds__(THREADS) restore_kernel(const Npop_Params P)
{
	if (P.status->flags == 0u) return;
	if (blockIdx.x == 0 and threadIdx.x == 0) P.clock[(P.phase + 1) % 3] = P.clock[P.phase];
	const long long total = (long long)NV * P.N;
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += stride) P.Uo[t] = P.U[t];
}

template <int SOLVER>
int launch_pair(const Npop_Params& P, const int grid, cudaStream_t stream)
{
	const dim3 tiles((P.n[0] + NTX - 1) / NTX, (P.n[1] + NTY - 1) / NTY, (P.n[2] + P.kchunk - 1) / P.kchunk);
	npop_fused_kernel<SOLVER><<<tiles, dim3(NTX, NTY), SMEM_FUSED, stream>>>(P);
	if (cudaGetLastError() != cudaSuccess) return PAMHD_ERR_CUDA;
	restore_kernel<<<grid, THREADS, 0, stream>>>(P);
	return cudaGetLastError() == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

int check(const cudaError_t e)
{
	return e == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

#define PAMHD_TRY(expr) do { const int rc_ = (expr); if (rc_ != PAMHD_OK) return rc_; } while (0)

} // namespace

struct pamhd_npop {
	int device = 0;
	int solver = 0;
	cudaStream_t stream = nullptr;
	long long N = 0;
	double* U[2] = {nullptr, nullptr};
	Speed_Max* red = nullptr;
	Clock* clock = nullptr;
	Status* status = nullptr;
	int cur = 0;
	long long steps = 0;
	int grid = 0;
	bool loaded = false;
	Npop_Params base;
};

namespace {

int issue(pamhd_npop& x, const Npop_Control& control)
{
	Npop_Params P = x.base;
	P.U = x.U[x.cur];
	P.Uo = x.U[x.cur ^ 1];
	P.phase = int(x.steps % 3);
	P.control = control;
	const int rc = x.solver == PAMHD_RUSANOV ? launch_pair<PAMHD_RUSANOV>(P, x.grid, x.stream)
	                                         : launch_pair<PAMHD_HLL_ATHENA>(P, x.grid, x.stream);
	if (rc != PAMHD_OK) return rc;
	x.cur ^= 1;
	x.steps++;
	return PAMHD_OK;
}

int reset(pamhd_npop& x)
{
	Speed_Max r[3] = {};
	r[0].zero = 1u;
	const Clock c[3] = {};
	const Status s{0u, 0u, ~0ull};
	PAMHD_TRY(check(cudaMemcpyAsync(x.red, r, sizeof r, cudaMemcpyHostToDevice, x.stream)));
	PAMHD_TRY(check(cudaMemcpyAsync(x.clock, c, sizeof c, cudaMemcpyHostToDevice, x.stream)));
	PAMHD_TRY(check(cudaMemcpyAsync(x.status, &s, sizeof s, cudaMemcpyHostToDevice, x.stream)));
	x.steps = 0;
	return check(cudaStreamSynchronize(x.stream));
}

} // namespace

extern "C" {

int pamhd_gpu_npop_create(const int32_t n[3], const double cell_length[3], const int32_t solver, const double gamma,
                          const double mu0, const double min_pressure, const int32_t device, pamhd_npop** out)
{
	if (n == nullptr or cell_length == nullptr or out == nullptr) return PAMHD_ERR_ARGUMENT;
	*out = nullptr;
	if (solver != PAMHD_RUSANOV and solver != PAMHD_HLL_ATHENA) return PAMHD_ERR_ARGUMENT;
	for (int d = 0; d < 3; d++) {
		if (n[d] < 1 or not (cell_length[d] > 0.0)) return PAMHD_ERR_ARGUMENT;
	}
	if (not (gamma > 1.0) or not (mu0 > 0.0) or not (min_pressure >= 0.0)) return PAMHD_ERR_ARGUMENT;
	const long long N = (long long)n[0] * n[1] * n[2];
	if (N > (1ll << 31)) return PAMHD_ERR_ARGUMENT;
	if ((n[1] + NTY - 1) / NTY > 65535) return PAMHD_ERR_ARGUMENT;   // rows of face tiles: the grid's y extent
	pamhd_npop* x = new (std::nothrow) pamhd_npop;
	if (x == nullptr) return PAMHD_ERR_ARGUMENT;
	x->device = device;
	x->solver = solver;
	x->N = N;
	auto fail = [&](const int rc) {
		pamhd_gpu_npop_destroy(x);
		return rc;
	};
	if (cudaSetDevice(device) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	if (cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	const size_t bytes = size_t(NV) * size_t(N) * sizeof(double);
	if (cudaMalloc(&x->U[0], bytes) != cudaSuccess or cudaMalloc(&x->U[1], bytes) != cudaSuccess
		or cudaMalloc(&x->red, 3 * sizeof(Speed_Max)) != cudaSuccess
		or cudaMalloc(&x->clock, 3 * sizeof(Clock)) != cudaSuccess
		or cudaMalloc(&x->status, sizeof(Status)) != cudaSuccess) {
		return fail(PAMHD_ERR_CUDA);
	}
	int sms = 0;
	if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	const long long blocks = (N + THREADS - 1) / THREADS;
	x->grid = int(blocks < 8ll * sms ? blocks : 8ll * sms);
	const cudaError_t attr = solver == PAMHD_RUSANOV
		? cudaFuncSetAttribute(npop_fused_kernel<PAMHD_RUSANOV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
		                       int(SMEM_FUSED))
		: cudaFuncSetAttribute(npop_fused_kernel<PAMHD_HLL_ATHENA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
		                       int(SMEM_FUSED));
	if (attr != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	Npop_Params& P = x->base;
	std::memset(&P, 0, sizeof P);
	// z chunks so that the face tiles fill the SMs about six times over
	const long long tiles = (long long)((n[0] + NTX - 1) / NTX) * ((n[1] + NTY - 1) / NTY);
	const long long chunks = std::max(1ll, std::min((long long)n[2], 18ll * sms / tiles));
	P.kchunk = int((n[2] + chunks - 1) / chunks);
	for (int d = 0; d < 3; d++) {
		P.n[d] = n[d];
		P.active[d] = n[d] > 1;
		P.len[d] = cell_length[d];
	}
	P.area[0] = cell_length[1] * cell_length[2];
	P.area[1] = cell_length[0] * cell_length[2];
	P.area[2] = cell_length[0] * cell_length[1];
	P.N = N;
	P.gamma = gamma;
	P.mu0 = mu0;
	P.inv_mu0 = 1.0 / mu0;
	P.half_inv_mu0 = 0.5 / mu0;
	P.min_pressure = min_pressure;
	P.red = x->red;
	P.clock = x->clock;
	P.status = x->status;
	if (cudaMemsetAsync(x->U[0], 0, bytes, x->stream) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	if (reset(*x) != PAMHD_OK) return fail(PAMHD_ERR_CUDA);
	*out = x;
	return PAMHD_OK;
}

int pamhd_gpu_npop_destroy(pamhd_npop* x)
{
	if (x == nullptr) return PAMHD_OK;
	cudaSetDevice(x->device);
	if (x->stream != nullptr) cudaStreamSynchronize(x->stream);
	cudaFree(x->U[0]);
	cudaFree(x->U[1]);
	cudaFree(x->red);
	cudaFree(x->clock);
	cudaFree(x->status);
	if (x->stream != nullptr) cudaStreamDestroy(x->stream);
	delete x;
	return PAMHD_OK;
}

int pamhd_gpu_npop_set_state(pamhd_npop* x, const double* const state[13])
{
	if (x == nullptr or state == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int v = 0; v < NV; v++) if (state[v] == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	const size_t n = size_t(x->N);
	x->cur = 0;
	// one copy per array straight from the caller's memory (at full speed when it is pinned)
	for (int v = 0; v < NV; v++) {
		PAMHD_TRY(check(cudaMemcpyAsync(x->U[0] + v * n, state[v], n * sizeof(double), cudaMemcpyHostToDevice,
		                                x->stream)));
	}
	PAMHD_TRY(reset(*x));
	x->loaded = true;
	return PAMHD_OK;
}

int pamhd_gpu_npop_get_state(pamhd_npop* x, double* const state[13])
{
	if (x == nullptr or state == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int v = 0; v < NV; v++) if (state[v] == nullptr) return PAMHD_ERR_ARGUMENT;
	if (not x->loaded) return PAMHD_ERR_STATE;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	const size_t n = size_t(x->N);
	for (int v = 0; v < NV; v++) {
		PAMHD_TRY(check(cudaMemcpyAsync(state[v], x->U[x->cur] + v * n, n * sizeof(double), cudaMemcpyDeviceToHost,
		                                x->stream)));
	}
	return check(cudaStreamSynchronize(x->stream));
}

int pamhd_gpu_npop_sync(pamhd_npop* x)
{
	if (x == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	Status s;
	PAMHD_TRY(check(cudaMemcpy(&s, x->status, sizeof s, cudaMemcpyDeviceToHost)));
	return s.flags != 0u ? PAMHD_ERR_PHYSICS : PAMHD_OK;
}

int pamhd_gpu_npop_step(pamhd_npop* x, const double dt, double* max_dt)
{
	if (x == nullptr or not (dt >= 0.0)) return PAMHD_ERR_ARGUMENT;
	if (not x->loaded) return PAMHD_ERR_STATE;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(issue(*x, Npop_Control{dt, 0.0, 0.0}));
	const int rc = pamhd_gpu_npop_sync(x);
	if (max_dt != nullptr) {
		Speed_Max r;
		PAMHD_TRY(check(cudaMemcpy(&r, x->red + (x->steps % 3), sizeof r, cudaMemcpyDeviceToHost)));
		double m = DBL_MAX;
		for (int d = 0; d < 3; d++) {
			double s;
			std::memcpy(&s, &r.smax[d], sizeof s);
			if (x->base.active[d] and s > 0.0) {
				const double q = x->base.len[d] / s;
				m = (q < m) ? q : m;
			}
		}
		*max_dt = m;
	}
	return rc;
}

int pamhd_gpu_npop_run(pamhd_npop* x, const int32_t nsteps, const double cfl, const double t_end)
{
	if (x == nullptr or nsteps < 0 or not (cfl > 0.0) or not (t_end == t_end)) return PAMHD_ERR_ARGUMENT;
	if (not x->loaded) return PAMHD_ERR_STATE;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	for (int32_t s = 0; s < nsteps; s++) PAMHD_TRY(issue(*x, Npop_Control{-1.0, cfl, t_end}));
	return PAMHD_OK;
}

int pamhd_gpu_npop_time(pamhd_npop* x, double* time, int64_t* steps, double* last_dt)
{
	if (x == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	Clock c;
	PAMHD_TRY(check(cudaMemcpy(&c, x->clock + (x->steps % 3), sizeof c, cudaMemcpyDeviceToHost)));
	if (time != nullptr) *time = c.t;
	if (steps != nullptr) *steps = c.steps;
	if (last_dt != nullptr) *last_dt = c.dt;
	return PAMHD_OK;
}

int pamhd_gpu_npop_status(pamhd_npop* x, uint32_t* flags, int32_t cell[3], int32_t* dir)
{
	if (x == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	Status s;
	PAMHD_TRY(check(cudaMemcpy(&s, x->status, sizeof s, cudaMemcpyDeviceToHost)));
	if (flags != nullptr) *flags = s.flags;
	const int* n = x->base.n;
	if (s.flags != 0u and s.first != ~0ull) {
		const long long key = (long long)(s.first >> 8);
		const long long c = key / 3;
		if (cell != nullptr) {
			cell[0] = int32_t(c % n[0]);
			cell[1] = int32_t((c / n[0]) % n[1]);
			cell[2] = int32_t(c / ((long long)n[0] * n[1]));
		}
		if (dir != nullptr) *dir = int32_t(key % 3) + 1;
	} else {
		if (cell != nullptr) cell[0] = cell[1] = cell[2] = -1;
		if (dir != nullptr) *dir = 0;
	}
	return PAMHD_OK;
}

int pamhd_gpu_npop_get_stream(pamhd_npop* x, void** stream)
{
	if (x == nullptr or stream == nullptr) return PAMHD_ERR_ARGUMENT;
	*stream = static_cast<void*>(x->stream);
	return PAMHD_OK;
}

} // extern "C"
