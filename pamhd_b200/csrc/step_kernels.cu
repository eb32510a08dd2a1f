/*
Kernels of the fused finite-volume MHD step (sm_100a, FP64 CUDA cores).

step_kernel<SOLVER, TY, MINB> - one launch = one whole step (the reference's
  get_all_fluxes + update_mhd_state + minimize_timestep, mhd/solve.hpp:
  1702-1811, :1518-1614, :1933-2014, in their cell-centred form):
  * a block owns a 32 x TY column tile and marches along z through a chunk
    of planes ("2.5-D blocking");
  * each plane of the tile plus a one-cell halo in x and y is read once
    from HBM (coalesced along x), its derived quantities (1/rho, pressure,
    fast speeds along x, y, z) computed once per cell into shared memory;
  * every x and y face of the tile is solved once from shared memory and
    its dt-scaled flux kept in shared memory; the z face between the
    previous and the current plane is solved by the thread owning the
    column and kept in registers, so every z face is solved once;
  * the new state of a cell is written as soon as its last (+z) face is
    known, plus its periodic image or COPY ghost (so no separate ghost
    fill pass is needed);
  * the face signal speeds are max-reduced per axis (warp shuffles, then
    one atomicMax per block on the bits of the non-negative double) into a
    three-slot ring; the next step's dt is computed from that ring by
    every block at kernel start, so consecutive steps never wait on the
    host and can be replayed from a CUDA graph.
Only the redundant halo faces of each tile (1/32 + 1/TY of the x/y faces)
and one z plane per chunk are solved twice.
*/
#include <cuda_runtime.h>

#include "step.cuh"

namespace pamhd_b200 {

constexpr int TX = 32;
#ifndef PAMHD_TY
#define PAMHD_TY 4
#endif
#ifndef PAMHD_MINB
#define PAMHD_MINB 3
#endif
#ifndef PAMHD_STEP_TY
#define PAMHD_STEP_TY 8
#endif
#ifndef PAMHD_STEP_MINB
#define PAMHD_STEP_MINB 2
#endif
constexpr int TY_3D = PAMHD_TY;     // tile rows of the batched step on 2-D and 3-D grids
constexpr int MINB = PAMHD_MINB;    // resident blocks per SM asked of the register allocator
constexpr int TY_STEP = PAMHD_STEP_TY;  // tile rows of the single-grid step (Roe aside)
// record of a cell in shared memory: rho, mom xyz, E, B xyz, 1/rho, p, cf x, cf y (the fast
// speed along z is needed by the column's owner only, which keeps it in a register)
constexpr int NV = 12;
enum { R_RINV = 8, R_P = 9, R_CF = 10 };

/*
Rows of a face flux kept in shared memory, in the face frame: rho, the
normal and the two tangential momenta, E, the two tangential field
components, and the normal field component only for Rusanov, the one
solver whose flux of it is not zero (mhd/rusanov.hpp diffuses it).
*/
template <int SOLVER> struct Flux_Rows { static constexpr int N = SOLVER == PAMHD_RUSANOV ? 8 : 7; };

template <int TY, int NF = 8> struct Tile {
	static constexpr int JO = (TY > 1) ? 1 : 0;            // halo rows exist when y is active
	static constexpr int W = TX + 2;                       // record row width (halo columns)
	static constexpr int H = TY + 2 * JO;                  // record rows
	static constexpr int CELLS = W * H;
	static constexpr int REC = NV * CELLS;                 // doubles per plane slot
	static constexpr int FXN = TY * (TX + 1);              // x faces of a plane
	static constexpr int FYN = (TY > 1) ? (TY + 1) * TX : 0;
	// two record slots, the x and y face fluxes, one validity byte per cell and slot
	static constexpr size_t BYTES = size_t(2 * REC + NF * FXN + NF * FYN) * 8 + size_t(2 * CELLS);
};

template <int SOLVER, int TY> constexpr size_t tile_bytes() { return Tile<TY, Flux_Rows<SOLVER>::N>::BYTES; }

/*
Tile rows of the single-grid step on 2-D and 3-D grids and the resident
blocks per SM it is built for: 32 x 8 tiles, two blocks of 256 threads per
SM at 128 registers (16 warps per SM; a taller tile solves fewer halo
faces and records per cell); Roe's solver needs more registers than that,
so it keeps 32 x 4 tiles at three blocks per SM.
*/
template <int SOLVER> struct Step_Shape {
	static constexpr int rows = SOLVER == PAMHD_ROE_ATHENA ? TY_3D : TY_STEP;
	static constexpr int blocks = SOLVER == PAMHD_ROE_ATHENA ? MINB : PAMHD_STEP_MINB;
};

template <int SOLVER, int TY> struct Step_Minb {
	static constexpr int value = (TY > 1 and TY == Step_Shape<SOLVER>::rows) ? Step_Shape<SOLVER>::blocks : MINB;
};

int step_tile_rows(const int solver)
{
	return solver == PAMHD_ROE_ATHENA ? Step_Shape<PAMHD_ROE_ATHENA>::rows : TY_STEP;
}

int batch_tile_rows()
{
	return TY_3D;
}

// ------------------------------------------------------------------ helpers

__device__ __forceinline__ double warp_max(double v)
{
	#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
	return v;
}

/*
dt of the step from the previous step's face speeds: the minimum over
faces of CFL * d_len / s (solve.hpp:1983-2003), which equals
CFL * d_len / max(s) per axis because rounding is monotonic; 0 when any
face speed was <= 0; replaced by the cap when cap <= that minimum
(substepping.hpp:331-338).
*/
__device__ __forceinline__ double step_dt(const Step_Params& P)
{
	if (P.forced_dt >= 0.0) return P.forced_dt;
	// read at L2 (ld.global.cg): a persistent launch reads what other blocks wrote a step before
	const Speed_Max& r = P.red[P.phase];
	bool zero = __ldcg(&r.zero) != 0;
	double smallest = 1.7976931348623157e308;
	#pragma unroll
	for (int d = 0; d < 3; d++) {
		if (not P.active[d]) continue;
		const double s = __longlong_as_double((long long)__ldcg(&r.smax[d]));
		if (not (s > 0.0)) {
			zero = true;
		} else {
			smallest = fmin(smallest, (P.cfl * P.len[d]) / s);
		}
	}
	if (zero) smallest = 0.0;
	const double t = __ldcg(&P.clock[P.phase].t);
	const double cap = P.control->max_dt >= 0.0 ? P.control->max_dt : P.control->t_end - t;
	return (cap <= smallest) ? cap : smallest;
}

/*
Whether the grid stopped in an earlier step: a face failed there (the
reference aborts at that step, mhd/solve.hpp:156-181).  Such a step leaves
the state as it is and the clock where it is.  The failing step itself is
completed (every block of it sees the same answer: the failure is dated by
the clock's step count).
*/
__device__ __forceinline__ bool stopped_before(const Step_Params& P)
{
	const unsigned int at = __ldcg(&P.status->fail_step);
	return at != 0u and (long long)(at - 1u) < __ldcg(&P.clock[P.phase].steps);
}

// block-wide start of a step: every block computes dt; block 0 advances the clock ring.  *s_stop:
// the grid stopped in an earlier step (dt 0, the clock held)
__device__ __forceinline__ double begin_step(const Step_Params& P, double* s_dt, const bool first_block,
                                             int* s_stop)
{
	if (threadIdx.x == 0 and threadIdx.y == 0) {
		const bool stop = stopped_before(P);
		const double dt = stop ? 0.0 : step_dt(P);
		*s_dt = dt;
		*s_stop = stop ? 1 : 0;
		if (first_block) {
			Clock c;
			c.t = __ldcg(&P.clock[P.phase].t);
			c.steps = __ldcg(&P.clock[P.phase].steps);
			Clock& next = P.clock[(P.phase + 1) % 3];
			next.t = c.t + dt;
			next.dt = dt;
			next.steps = stop ? c.steps : c.steps + 1;
			if (P.dt_hist != nullptr and not stop) P.dt_hist[c.steps % P.hist_len] = dt;
			Speed_Max& z = P.red[(P.phase + 2) % 3];
			z.smax[0] = z.smax[1] = z.smax[2] = 0ull;
			z.zero = 0u;
			if (stop) {
				// no face is solved: the failing step's maxima stay the latest
				const Speed_Max& r = P.red[P.phase];
				Speed_Max& o = P.red[(P.phase + 1) % 3];
				o.smax[0] = __ldcg(&r.smax[0]);
				o.smax[1] = __ldcg(&r.smax[1]);
				o.smax[2] = __ldcg(&r.smax[2]);
				o.zero = __ldcg(&r.zero);
			}
		}
	}
	__syncthreads();
	return *s_dt;
}

// the first failing face, numbered as the oracle's extended grid (x fastest)
__device__ void record_failure(const Step_Params& P, const uint32_t flag, const int i, const int j,
                               const int k, const int dir)
{
	int c[3] = {i, j, k};
	#pragma unroll
	for (int d = 0; d < 3; d++) {
		if (P.periodic[d] and c[d] < 0) c[d] += P.L.n[d];
	}
	const unsigned long long nx = P.L.n[0] + 2 * P.ext[0], ny = P.L.n[1] + 2 * P.ext[1];
	const unsigned long long lin = (unsigned long long)(c[0] + P.ext[0])
		+ nx * ((unsigned long long)(c[1] + P.ext[1]) + ny * (unsigned long long)(c[2] + P.ext[2]));
	atomicOr(&P.status->flags, flag);
	atomicMin(&P.status->first, ((lin * 4ull + (unsigned long long)dir) << 8) | flag);
	// every failure of a step writes the same date
	P.status->fail_step = (unsigned int)(__ldcg(&P.clock[P.phase].steps) + 1);
}

__device__ __forceinline__ void flush_speeds(const Step_Params& P, double smax[3], bool zero)
{
	__shared__ double part[3][32];
	__shared__ int part_zero[32];
	const int tid = threadIdx.y * blockDim.x + threadIdx.x;
	const int warp = tid >> 5, lane = tid & 31, warps = (blockDim.x * blockDim.y + 31) >> 5;
	#pragma unroll
	for (int d = 0; d < 3; d++) smax[d] = warp_max(smax[d]);
	const int z = __any_sync(0xffffffffu, zero);
	if (lane == 0) {
		part[0][warp] = smax[0];
		part[1][warp] = smax[1];
		part[2][warp] = smax[2];
		part_zero[warp] = z;
	}
	__syncthreads();
	if (tid == 0) {
		Speed_Max& r = P.red[(P.phase + 1) % 3];
		int any_zero = 0;
		#pragma unroll
		for (int d = 0; d < 3; d++) {
			double m = 0.0;
			for (int w = 0; w < warps; w++) m = fmax(m, part[d][w]);
			if (P.active[d] and m > 0.0) {
				atomicMax(&r.smax[d], (unsigned long long)__double_as_longlong(m));
			}
		}
		for (int w = 0; w < warps; w++) any_zero |= part_zero[w];
		if (any_zero) atomicOr(&r.zero, 1u);
	}
}

// ghost copy of COPY sides: density, velocity, pressure and field of the neighbour
// (mhd/boundaries.hpp:818-1030 with the constant-pressure field copy)
__device__ __forceinline__ void copy_state(const double U[8], const Gas& g, double C[8])
{
	const double ir = 1.0 / U[0];
	const double vx = U[1] * ir, vy = U[2] * ir, vz = U[3] * ir;
	const double b2 = U[5] * U[5] + U[6] * U[6] + U[7] * U[7];
	const double p = (U[4] - 0.5 * ir * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) - 0.5 * g.inv_mu0 * b2)
		* (g.gamma - 1.0);
	C[0] = U[0];
	C[1] = U[0] * vx;
	C[2] = U[0] * vy;
	C[3] = U[0] * vz;
	const double ic = 1.0 / C[0];
	const double wx = C[1] * ic, wy = C[2] * ic, wz = C[3] * ic;
	C[4] = p / (g.gamma - 1.0) + 0.5 * C[0] * (wx * wx + wy * wy + wz * wz) + 0.5 * g.inv_mu0 * b2;
	C[5] = U[5];
	C[6] = U[6];
	C[7] = U[7];
}

__device__ __forceinline__ void store_cell(double* out, const Layout& L, const int i, const int j,
                                           const int k, const double U[8])
{
	const long long off = L.offset(i, j, k);
	#pragma unroll
	for (int v = 0; v < 8; v++) out[v * L.var + off] = U[v];
}

// the state of a time-stamped inflow at time t
__device__ __forceinline__ const double* inflow_at(const Inflow_Table& T, const double t)
{
	int i = 0;
	while (i < T.count and t >= T.times[i]) i++;
	return T.states + 8 * i;
}

/*
New state of an interior cell plus its periodic image / COPY ghost, and the
ghost of a time-stamped VALUE side at the time the new state holds: the
step's start time plus dt, as begin_step advances the clock.
*/
__device__ void write_cell(const Step_Params& P, const int i, const int j, const int k, const double U[8],
                           const double dt)
{
	store_cell(P.out, P.L, i, j, k, U);
	const int c[3] = {i, j, k};
	#pragma unroll
	for (int d = 0; d < 3; d++) {
		if (not P.active[d]) continue;
		const int n = P.L.n[d];
		int t[3] = {i, j, k};
		if (c[d] == 0) {
			if (P.periodic[d]) {
				t[d] = n;
				store_cell(P.out, P.L, t[0], t[1], t[2], U);
			} else if (P.bc_lo[d] == PAMHD_BC_COPY) {
				double C[8];
				copy_state(U, P.gas, C);
				t[d] = -1;
				store_cell(P.out, P.L, t[0], t[1], t[2], C);
			} else if (P.bc_lo[d] == PAMHD_BC_VALUE and P.inflow != nullptr and P.inflow[2 * d].states != nullptr) {
				t[d] = -1;
				store_cell(P.out, P.L, t[0], t[1], t[2], inflow_at(P.inflow[2 * d], __ldcg(&P.clock[P.phase].t) + dt));
			}
		}
		if (c[d] == n - 1) {
			t[0] = i; t[1] = j; t[2] = k;
			if (P.periodic[d]) {
				t[d] = -1;
				store_cell(P.out, P.L, t[0], t[1], t[2], U);
			} else if (P.bc_hi[d] == PAMHD_BC_COPY) {
				double C[8];
				copy_state(U, P.gas, C);
				t[d] = n;
				store_cell(P.out, P.L, t[0], t[1], t[2], C);
			} else if (P.bc_hi[d] == PAMHD_BC_VALUE and P.inflow != nullptr and P.inflow[2 * d + 1].states != nullptr) {
				t[d] = n;
				store_cell(P.out, P.L, t[0], t[1], t[2], inflow_at(P.inflow[2 * d + 1], __ldcg(&P.clock[P.phase].t) + dt));
			}
		}
	}
}

/*
Read a cell from HBM, derive its per-cell quantities into a record slot.
CO: loads at L2 (ld.global.cg) instead of through the read-only cache, for a
persistent launch whose later steps read what other blocks wrote (the
non-coherent L1 could hold a line of the same buffer from two steps before).
*/
template <bool CX, bool CY, bool CZ, bool CO>
__device__ __forceinline__ double load_record(const Step_Params& P, double* rec, uint8_t* bad, const int cells,
                                              const int ri, const int i, const int j, const int k)
{
	const long long off = P.L.offset(i, j, k);
	double U[8];
	#pragma unroll
	for (int v = 0; v < 8; v++) U[v] = CO ? __ldcg(P.in + v * P.L.var + off) : __ldg(P.in + v * P.L.var + off);
	const Derived d = derive<CX, CY, CZ, true>(U[0], U[1], U[2], U[3], U[4], U[5], U[6], U[7], P.gas);
	#pragma unroll
	for (int v = 0; v < 8; v++) rec[v * cells + ri] = U[v];
	rec[R_RINV * cells + ri] = d.rinv;
	rec[R_P * cells + ri] = d.p;
	if (CX) rec[(R_CF + 0) * cells + ri] = d.cf[0];
	if (CY) rec[(R_CF + 1) * cells + ri] = d.cf[1];
	bad[ri] = uint8_t(d.bad);
	// the fast speed along z, for the caller's z faces
	return CZ ? d.cf[2] : 0.0;
}

// one cell of a record slot seen from a face normal to axis A (rotation by index permutation),
// with its fast speed along A
template <int A>
__device__ __forceinline__ Side side_at(const double* rec, const uint8_t* bad, const int cells, const int ri,
                                        const double cf)
{
	Side s;
	s.rho = rec[ri];
	rotate<A>(rec[1 * cells + ri], rec[2 * cells + ri], rec[3 * cells + ri], s.m0, s.m1, s.m2);
	s.E = rec[4 * cells + ri];
	rotate<A>(rec[5 * cells + ri], rec[6 * cells + ri], rec[7 * cells + ri], s.b0, s.b1, s.b2);
	s.rinv = rec[R_RINV * cells + ri];
	s.p = rec[R_P * cells + ri];
	s.cf = cf;
	s.v0 = s.m0 * s.rinv;
	s.v1 = s.m1 * s.rinv;
	s.v2 = s.m2 * s.rinv;
	s.bad = bad[ri];
	return s;
}

/*
Solves one z face, folds its speed into the running max and returns the
unscaled flux in the xyz frame (the update multiplies by dt / dz once per
cell).  Each kernel inlines this once, so a z face is computed by the same
instructions wherever it lies in the tiling.
*/
template <int SOLVER, int CELLS>
__device__ __forceinline__ void solve_z(const Step_Params& P, const double* rec_l, const uint8_t* bad_l,
                                        const double* rec_r, const uint8_t* bad_r, const int ri, const double cf_l,
                                        const double cf_r, double d[8], double& smax, bool& zero, const int i,
                                        const int j, const int k)
{
	const Side L = side_at<2>(rec_l, bad_l, CELLS, ri, cf_l);
	const Side R = side_at<2>(rec_r, bad_r, CELLS, ri, cf_r);
	double F[8];
	uint32_t flag = 0;
	// the side an HLLD flux is taken from, read again from the records (see flux_hlld)
	const auto pick = [&](const bool left) {
		return side_at<2>(left ? rec_l : rec_r, left ? bad_l : bad_r, CELLS, ri, left ? cf_l : cf_r);
	};
	const double s = solve_face<SOLVER, true>(L, R, P.gas, F, flag, pick);
	if (flag != 0) record_failure(P, flag, i, j, k, 3);
	smax = fmax(smax, s);
	zero = zero or not (s > 0.0);
	d[0] = F[0];
	unrotate<2>(F[1], F[2], F[3], d[1], d[2], d[3]);
	d[4] = F[4];
	unrotate<2>(F[5], F[6], F[7], d[5], d[6], d[7]);
}

/*
One x or y face (axis a, 0 or 1, known only at run time) between record
positions rl and rr of one slot.  The x and y faces of a plane share this
one inlined solver instance (half the code of one instance per axis, which
the instruction cache rewards); the rotation into the face frame is a
choice of record rows to read.  The unscaled flux goes to out[r][idx] in
the face frame, Flux_Rows<SOLVER>::N rows (the caller rotates it back).
*/
template <int SOLVER, int CELLS>
__device__ __forceinline__ void solve_xy(const Step_Params& P, const double* rec, const uint8_t* bad,
                                         const int rl, const int rr, const int a, double* out, const int nout,
                                         const int idx, double& s0, double& s1, bool& zero,
                                         const int i, const int j, const int k)
{
	const int a1 = a + 1, a2 = a == 0 ? 2 : 0;  // the face frame's tangential axes
	auto side = [&](const int r) {
		Side s;
		s.rho = rec[r];
		s.m0 = rec[(1 + a) * CELLS + r];
		s.m1 = rec[(1 + a1) * CELLS + r];
		s.m2 = rec[(1 + a2) * CELLS + r];
		s.E = rec[4 * CELLS + r];
		s.b0 = rec[(5 + a) * CELLS + r];
		s.b1 = rec[(5 + a1) * CELLS + r];
		s.b2 = rec[(5 + a2) * CELLS + r];
		s.rinv = rec[R_RINV * CELLS + r];
		s.p = rec[R_P * CELLS + r];
		s.cf = rec[(R_CF + a) * CELLS + r];
		s.v0 = s.m0 * s.rinv;
		s.v1 = s.m1 * s.rinv;
		s.v2 = s.m2 * s.rinv;
		s.bad = bad[r];
		return s;
	};
	const Side L = side(rl);
	const Side R = side(rr);
	double F[8];
	uint32_t flag = 0;
	const auto pick = [&](const bool left) { return side(left ? rl : rr); };
	const double sp = solve_face<SOLVER, true>(L, R, P.gas, F, flag, pick);
	if (flag != 0) record_failure(P, flag, i, j, k, a + 1);
	if (a == 0) s0 = fmax(s0, sp); else s1 = fmax(s1, sp);
	zero = zero or not (sp > 0.0);
	out[idx] = F[0];
	out[1 * nout + idx] = F[1];
	out[2 * nout + idx] = F[2];
	out[3 * nout + idx] = F[3];
	out[4 * nout + idx] = F[4];
	out[5 * nout + idx] = F[6];
	out[6 * nout + idx] = F[7];
	if (Flux_Rows<SOLVER>::N == 8) out[7 * nout + idx] = F[5];
}

// ------------------------------------------------------------------ the step

// the planes [kb, ke) of block row bz: a z chunk, or with kpart 1 the first (bz 0) or the last
// (bz 1) plane alone, or with kpart 2 a chunk of the planes between them
__device__ __forceinline__ void tile_planes(const Step_Params& P, const int bz, int& kb, int& ke)
{
	const int nz = P.L.n[2];
	const int kbase = P.kpart == 2 ? 1 : 0, ktop = P.kpart == 2 ? nz - 1 : nz;
	kb = P.kpart == 1 ? (bz == 0 ? 0 : nz - 1) : kbase + bz * P.kchunk;
	ke = P.kpart == 1 ? kb + 1 : min(ktop, kb + P.kchunk);
}

/*
A step of a grid that stopped: the tile's cells are copied into the new
state unchanged, with the ghosts a step writes, so that both states hold
the failing step's result.  CO: loads at L2 (see load_record).
*/
template <int TY, bool CO>
__device__ void tile_hold(const Step_Params& P, const int bx, const int by, const int bz)
{
	int kb, ke;
	tile_planes(P, bz, kb, ke);
	const int gx = bx * TX + threadIdx.x, gy = by * TY + threadIdx.y;
	if (gx >= P.L.n[0] or gy >= P.L.n[1]) return;
	for (int k = kb; k < ke; k++) {
		const long long off = P.L.offset(gx, gy, k);
		double U[8];
		#pragma unroll
		for (int v = 0; v < 8; v++) U[v] = CO ? __ldcg(P.in + v * P.L.var + off) : P.in[v * P.L.var + off];
		write_cell(P, gx, gy, k, U, 0.0);
	}
}

/*
One work item of a step: the tile (bx, by) of 32 x TY columns over the z
chunk bz, marched plane by plane; the face speeds are folded into
s0, s1, s2 and zero (flushed by the caller).  Shared by the single-grid
and the batched kernels, so that both compute the same bits.

Per plane k: (a) stage the plane's records (two slots alternate, so the
z face between planes k - 1 and k can read both); (b) every x and y face
of the plane into shared memory, and the z face below each own cell in
registers, which completes the cell below: its new state is written; (c)
each own cell's state plus its x and y flux differences, and the flux of
its -z face, held in registers until the +z face of the next plane.
*/
template <int SOLVER, int TY, bool CO = false>
__device__ __forceinline__ void tile_step(const Step_Params& P, double* const smem, const double dt,
                                          const int bx, const int by, const int bz,
                                          double& s0, double& s1, double& s2, bool& zero)
{
	constexpr int NF = Flux_Rows<SOLVER>::N;
	using T = Tile<TY, NF>;
	double* const rec_base = smem;
	double* const fx = smem + 2 * T::REC;        // [NF][TY][TX + 1]
	double* const fy = fx + NF * T::FXN;         // [NF][TY + 1][TX]
	uint8_t* const bad_base = reinterpret_cast<uint8_t*>(fy + NF * T::FYN);

	constexpr bool YACT = TY > 1;
	const bool zact = P.active[2] != 0;
	const int nx = P.L.n[0], ny = P.L.n[1];
	const int tx = threadIdx.x, ty = threadIdx.y;
	const int warp = ty, lane = tx;  // TX = 32: one warp per tile row
	// warps given the halo columns and the tile's extra +x / +y faces (kept apart from the
	// warps loading the halo rows, so that no warp does more than one extra pass per phase)
	static_assert(TY == 1 or TY >= 4, "tile rows: 1 or at least 4");
	constexpr int XHALO_WARP = TY >= 4 ? 2 : 0;
	constexpr int XFACE_WARP = TY >= 4 ? TY - 2 : 0;
	constexpr int YFACE_WARP = TY >= 4 ? TY - 1 : 0;
	const int gx0 = bx * TX, gy0 = by * TY;
	const int gx = gx0 + tx, gy = gy0 + ty;
	const bool own = gx < nx and gy < ny;
	// the +x / +y ghost of a partial tile lies inside the tile's own columns / rows
	const bool stage = gx <= nx and (TY == 1 ? gy == 0 : gy <= ny);
	// the planes of this block
	int kb, ke;
	tile_planes(P, bz, kb, ke);
	const int kfirst = zact ? kb - 1 : kb;
	const int klast = zact ? ke : ke - 1;
	const int ri = (ty + T::JO) * T::W + tx + 1;
	// the flux terms are dt F / dx: dt / dx once per axis and cell
	const double cx = dt * P.inv_len[0], cy = dt * P.inv_len[1], cz = dt * P.inv_len[2];

	// the cell below the current plane: its state plus its x and y flux differences plus the
	// flux of its -z face, all scaled; its +z face completes it
	double Acc[8];
	#pragma unroll
	for (int v = 0; v < 8; v++) Acc[v] = 0.0;
	// the own column's fast speed along z in the previous and the current plane
	double cfz_prev = 0.0, cfz = 0.0;

	for (int k = kfirst; k <= klast; k++) {
		const int slot = (k - kfirst) & 1;
		double* const rec = rec_base + slot * T::REC;
		uint8_t* const bad = bad_base + slot * T::CELLS;
		const double* const prev = rec_base + (slot ^ 1) * T::REC;
		const uint8_t* const prev_bad = bad_base + (slot ^ 1) * T::CELLS;
		const bool inner = k >= kb and k < ke;

		// (a) stage the plane: own cells, and the halo for planes with x / y faces
		cfz_prev = cfz;
		if (stage) cfz = load_record<true, YACT, true, CO>(P, rec, bad, T::CELLS, ri, gx, gy, k);
		// halo, spread over warps: the rows below / above the tile on warps 0 and 1, the columns
		// left / right of it on warp 2 (warp 0 when y is inactive)
		if (inner) {
			if (YACT and warp < 2) {
				const bool top = warp == 1;
				const int hy = top ? gy0 + TY : gy0 - 1;
				if (gx0 + lane < nx and hy <= ny) {
					const int hri = (top ? TY + 1 : 0) * T::W + lane + 1;
					load_record<false, true, false, CO>(P, rec, bad, T::CELLS, hri, gx0 + lane, hy, k);
				}
			} else if (warp == XHALO_WARP and lane < 2 * TY) {
				const int row = lane % TY;
				const bool right = lane >= TY;
				const int hx = right ? gx0 + TX : gx0 - 1;
				if (gy0 + row < ny and hx <= nx) {
					const int hri = (row + T::JO) * T::W + (right ? TX + 1 : 0);
					load_record<true, false, false, CO>(P, rec, bad, T::CELLS, hri, hx, gy0 + row, k);
				}
			}
		}
		__syncthreads();

		// (b) x and y faces: every thread its -x and -y face; the tile's last column and row also
		// need their +x / +y faces, taken by one warp each in a further pass of the same loop
		if (inner) {
			#pragma unroll 1
			for (int task = 0; task < 4; task++) {
				// 0: own -x face, 1: own -y face, 2: the tile's +x faces, 3: its +y faces
				if (task == 1 and not YACT) continue;
				if (task == 2 and warp != XFACE_WARP) continue;
				if (task == 3 and (not YACT or warp != YFACE_WARP)) continue;
				const int a = (task == 0 or task == 2) ? 0 : 1;
				const int row = task == 2 ? lane : (task == 3 ? TY : ty);
				const int col = task == 2 ? TX : tx;
				// one call site: the x and y faces share one inlined solver instance
				bool ok;
				int rl, rr, idx, i, j;
				if (a == 0) {
					ok = (task == 2 ? lane < TY : true) and gx0 + col <= nx and gy0 + row < ny;
					rl = (row + T::JO) * T::W + col;
					rr = rl + 1;
					idx = row * (TX + 1) + col;
					i = gx0 + col - 1;
					j = gy0 + row;
				} else {
					ok = gy0 + row <= ny and gx0 + col < nx;
					rl = row * T::W + col + 1;
					rr = rl + T::W;
					idx = row * TX + col;
					i = gx0 + col;
					j = gy0 + row - 1;
				}
				if (ok) {
					solve_xy<SOLVER, T::CELLS>(P, rec, bad, rl, rr, a, a == 0 ? fx : fy, a == 0 ? T::FXN : T::FYN,
					                           idx, s0, s1, zero, i, j, k);
				}
			}
		}
		// the z face between the previous plane and this one, by the column's owner; it completes
		// the cell below (U += (F- - F+) dt/dx, then y, then z: solve.hpp:1551-1587)
		if (zact and k > kfirst and own) {
			double Fz[8];
			solve_z<SOLVER, T::CELLS>(P, prev, prev_bad, rec, bad, ri, cfz_prev, cfz, Fz, s2, zero, gx, gy, k - 1);
			if (k > kb) {
				#pragma unroll
				for (int v = 0; v < 8; v++) Acc[v] = Acc[v] - Fz[v] * cz;
				write_cell(P, gx, gy, k - 1, Acc, dt);
			}
			#pragma unroll
			for (int v = 0; v < 8; v++) Acc[v] = Fz[v] * cz;
		}
		__syncthreads();

		// (c) the own cell: state plus x and y flux differences (plus its -z flux, held in Acc)
		if (own and inner) {
			// the flux row of each xyz variable in the x and the y face frames; -1: the normal
			// field component, whose flux is zero unless the solver keeps an eighth row (adding
			// 0.0 keeps the bits of adding a zero flux difference)
			constexpr int XROW[8] = {0, 1, 2, 3, 4, NF == 8 ? 7 : -1, 5, 6};
			constexpr int YROW[8] = {0, 3, 1, 2, 4, 6, NF == 8 ? 7 : -1, 5};
			double Un[8];
			#pragma unroll
			for (int v = 0; v < 8; v++) {
				const double u = rec[v * T::CELLS + ri];
				if (XROW[v] >= 0) {
					const double* f = fx + XROW[v] * T::FXN + ty * (TX + 1) + tx;
					Un[v] = u + (f[0] - f[1]) * cx;
				} else {
					Un[v] = u + 0.0;
				}
			}
			if (YACT) {
				#pragma unroll
				for (int v = 0; v < 8; v++) {
					if (YROW[v] >= 0) {
						const double* f = fy + YROW[v] * T::FYN + ty * TX + tx;
						Un[v] += (f[0] - f[TX]) * cy;
					} else {
						Un[v] += 0.0;
					}
				}
			}
			if (zact) {
				#pragma unroll
				for (int v = 0; v < 8; v++) Acc[v] = Un[v] + Acc[v];
			} else {
				write_cell(P, gx, gy, k, Un, dt);
			}
		}
	}
}

template <int SOLVER, int TY, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB) step_kernel(const Step_Params P)
{
	extern __shared__ __align__(16) double smem[];
	__shared__ double s_dt;
	__shared__ int s_stop;
	const bool first_block = blockIdx.x == 0 and blockIdx.y == 0 and blockIdx.z == 0;
	const double dt = begin_step(P, &s_dt, first_block, &s_stop);
	if (s_stop) {
		tile_hold<TY, false>(P, blockIdx.x, blockIdx.y, blockIdx.z);
		return;
	}
	double s0 = 0.0, s1 = 0.0, s2 = 0.0;
	bool zero = false;
	tile_step<SOLVER, TY>(P, smem, dt, blockIdx.x, blockIdx.y, blockIdx.z, s0, s1, s2, zero);
	double smax[3] = {s0, s1, s2};
	flush_speeds(P, smax, zero);
}

/*
The batched step: every box of an ensemble advances one step in one launch.
Blocks walk the work-item table (box, tile x, tile y, z chunk) with a grid
stride; each box has its own parameters (state buffers, layout, boundary
kinds, reduction ring, clock, status), so each advances with its own dt.
The block holding a box's first item advances that box's clock.
*/
template <int SOLVER, int TY, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB) batch_step_kernel(const Step_Params* __restrict__ boxes,
                                                                  const int4* __restrict__ items,
                                                                  const int nitems, const int phase)
{
	extern __shared__ __align__(16) double smem[];
	__shared__ Step_Params sp;
	__shared__ double s_dt;
	__shared__ int s_stop;
	const int tid = threadIdx.y * blockDim.x + threadIdx.x;
	for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
		const int4 w = items[item];
		__syncthreads();  // the previous item is done with sp
		if (tid == 0) {
			sp = boxes[w.x];
			sp.phase = phase;
		}
		__syncthreads();
		const bool first = w.y == 0 and w.z == 0 and w.w == 0;
		const double dt = begin_step(sp, &s_dt, first, &s_stop);
		const int tiles_x = (sp.L.n[0] + TX - 1) / TX;
		if (s_stop) {
			tile_hold<TY, false>(sp, w.y % tiles_x, w.y / tiles_x, w.z);
			continue;
		}
		double s0 = 0.0, s1 = 0.0, s2 = 0.0;
		bool zero = false;
		tile_step<SOLVER, TY>(sp, smem, dt, w.y % tiles_x, w.y / tiles_x, w.z, s0, s1, s2, zero);
		double smax[3] = {s0, s1, s2};
		flush_speeds(sp, smax, zero);
	}
}

// the (ghost dimension d, side, tangential axis e) combinations with ghost-ghost faces
__device__ __forceinline__ int boundary_combos(const Step_Params& P, int combos[12][3])
{
	int nc = 0;
	for (int d = 0; d < 3; d++) {
		if (not P.active[d] or P.periodic[d]) continue;
		for (int side = 0; side < 2; side++) {
			// the ghost layer of a slab cut is the neighbouring slab's interior: its faces are counted there
			if ((side ? P.bc_hi[d] : P.bc_lo[d]) == PAMHD_BC_EXTERNAL) continue;
			for (int e = 0; e < 3; e++) {
				if (e == d or not P.active[e]) continue;
				combos[nc][0] = d; combos[nc][1] = side; combos[nc][2] = e;
				nc++;
			}
		}
	}
	return nc;
}

// faces of one combination: along a slab cut at the high side, the face into the ghost plane is
// this slab's (the one into the low ghost plane is the lower neighbour's)
__device__ __forceinline__ long long boundary_count(const Step_Params& P, const int d, const int e)
{
	const int f = 3 - d - e;
	const int ne = (P.periodic[e] or P.bc_hi[e] == PAMHD_BC_EXTERNAL) ? P.L.n[e] : P.L.n[e] - 1;
	return (long long)ne * P.L.n[f];
}

// face t of combination (d, side, e): solved for its speed only (CO: loads at L2, see load_record)
template <int SOLVER, bool CO>
__device__ __forceinline__ void boundary_face(const Step_Params& P, const int d, const int side, const int e,
                                              const long long t, double smax[3], bool& zero)
{
	const int f = 3 - d - e;
	const int ne = (P.periodic[e] or P.bc_hi[e] == PAMHD_BC_EXTERNAL) ? P.L.n[e] : P.L.n[e] - 1;
	int a[3], b[3];
	a[d] = b[d] = side ? P.L.n[d] : -1;
	a[e] = int(t % ne);
	b[e] = (a[e] + 1 == P.L.n[e] and P.periodic[e]) ? 0 : a[e] + 1;
	a[f] = b[f] = int(t / ne);
	double UA[8], UB[8];
	const long long oa = P.L.offset(a[0], a[1], a[2]), ob = P.L.offset(b[0], b[1], b[2]);
	#pragma unroll
	for (int v = 0; v < 8; v++) {
		UA[v] = CO ? __ldcg(P.in + v * P.L.var + oa) : P.in[v * P.L.var + oa];
		UB[v] = CO ? __ldcg(P.in + v * P.L.var + ob) : P.in[v * P.L.var + ob];
	}
	const Derived da = derive<true, true, true>(UA[0], UA[1], UA[2], UA[3], UA[4], UA[5], UA[6], UA[7], P.gas);
	const Derived db = derive<true, true, true>(UB[0], UB[1], UB[2], UB[3], UB[4], UB[5], UB[6], UB[7], P.gas);
	Side L, R;
	auto fill = [e](Side& s, const double U[8], const Derived& dd) {
		s.rho = U[0];
		s.E = U[4];
		double m[3] = {U[1], U[2], U[3]}, B[3] = {U[5], U[6], U[7]};
		const int i0 = e, i1 = (e + 1) % 3, i2 = (e + 2) % 3;
		s.m0 = m[i0]; s.m1 = m[i1]; s.m2 = m[i2];
		s.b0 = B[i0]; s.b1 = B[i1]; s.b2 = B[i2];
		s.rinv = dd.rinv;
		s.v0 = s.m0 * s.rinv; s.v1 = s.m1 * s.rinv; s.v2 = s.m2 * s.rinv;
		s.p = dd.p;
		s.cf = dd.cf[e];
		s.bad = dd.bad;
	};
	fill(L, UA, da);
	fill(R, UB, db);
	double F[8];
	uint32_t flag = 0;
	const double sp = solve_face<SOLVER, true>(L, R, P.gas, F, flag);
	if (flag != 0) record_failure(P, flag, a[0], a[1], a[2], e + 1);
	smax[e] = fmax(smax[e], sp);
	zero = zero or not (sp > 0.0);
}

/*
Speeds of the faces between two boundary ghosts of a non-periodic side
(cells of class 0 on both sides).  The reference solves those faces too
(mhd/solve.hpp:254-311 visits every cell of class >= 0) and their speeds
enter the timestep (:1965-2005); their fluxes change nothing.
blockIdx.y enumerates (ghost dimension d, side, tangential axis e).
*/
template <int SOLVER>
__device__ __forceinline__ void boundary_speeds(const Step_Params& P)
{
	// a grid that stopped solves no face (the value is the same for every thread)
	if (stopped_before(P)) return;
	int combos[12][3];
	const int nc = boundary_combos(P, combos);
	double smax[3] = {0.0, 0.0, 0.0};
	bool zero = false;
	if ((int)blockIdx.y < nc) {
		const int d = combos[blockIdx.y][0], side = combos[blockIdx.y][1], e = combos[blockIdx.y][2];
		const long long count = boundary_count(P, d, e);
		for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < count;
		     t += (long long)gridDim.x * blockDim.x) {
			boundary_face<SOLVER, false>(P, d, side, e, t, smax, zero);
		}
	}
	flush_speeds(P, smax, zero);
}

template <int SOLVER>
__global__ void boundary_speed_kernel(const Step_Params P)
{
	boundary_speeds<SOLVER>(P);
}

// the same for every box of a batch: blockIdx.z is the box
template <int SOLVER>
__global__ void batch_boundary_speed_kernel(const Step_Params* __restrict__ boxes, const int phase)
{
	__shared__ Step_Params sp;
	if (threadIdx.x == 0) {
		sp = boxes[blockIdx.z];
		sp.phase = phase;
	}
	__syncthreads();
	boundary_speeds<SOLVER>(sp);
}

// ------------------------------------------------------------------ layout and ghosts

__global__ void scatter_kernel(const double* __restrict__ packed, double* __restrict__ var, const Layout L)
{
	const long long n = (long long)L.n[0] * L.n[1] * L.n[2];
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		const int i = int(t % L.n[0]);
		const int j = int((t / L.n[0]) % L.n[1]);
		const int k = int(t / ((long long)L.n[0] * L.n[1]));
		var[L.offset(i, j, k)] = packed[t];
	}
}

__global__ void gather_kernel(const double* __restrict__ var, double* __restrict__ packed, const Layout L)
{
	const long long n = (long long)L.n[0] * L.n[1] * L.n[2];
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		const int i = int(t % L.n[0]);
		const int j = int((t / L.n[0]) % L.n[1]);
		const int k = int(t / ((long long)L.n[0] * L.n[1]));
		packed[t] = var[L.offset(i, j, k)];
	}
}

/*
Fills every face ghost of `state` from its interior (periodic image, COPY)
or the configured VALUE state (apply_boundaries, mhd/boundaries.hpp:1261).
value_lo/hi are passed through the params of the host context.
*/
struct Ghost_Values {
	double lo[3][8];
	double hi[3][8];
};

__global__ void fill_ghosts_kernel(const Step_Params P, double* state, const Ghost_Values V)
{
	for (int d = 0; d < 3; d++) {
		if (not P.active[d]) continue;
		const int e = (d + 1) % 3, f = (d + 2) % 3;
		const long long count = (long long)P.L.n[e] * P.L.n[f];
		for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 2 * count;
		     t += (long long)gridDim.x * blockDim.x) {
			const int side = int(t / count);
			const long long r = t % count;
			int c[3];
			c[e] = int(r % P.L.n[e]);
			c[f] = int(r / P.L.n[e]);
			c[d] = side ? P.L.n[d] : -1;
			int s[3] = {c[0], c[1], c[2]};
			double U[8];
			const int kind = side ? P.bc_hi[d] : P.bc_lo[d];
			if (kind == PAMHD_BC_EXTERNAL) continue;  // written by the halo exchange
			if (P.periodic[d]) {
				s[d] = side ? 0 : P.L.n[d] - 1;
				const long long o = P.L.offset(s[0], s[1], s[2]);
				for (int v = 0; v < 8; v++) U[v] = state[v * P.L.var + o];
			} else if (kind == PAMHD_BC_COPY) {
				s[d] = side ? P.L.n[d] - 1 : 0;
				const long long o = P.L.offset(s[0], s[1], s[2]);
				double W[8];
				for (int v = 0; v < 8; v++) W[v] = state[v * P.L.var + o];
				copy_state(W, P.gas, U);
			} else {
				for (int v = 0; v < 8; v++) U[v] = side ? V.hi[d][v] : V.lo[d][v];
			}
			store_cell(state, P.L, c[0], c[1], c[2], U);
		}
	}
}

// ------------------------------------------------------------------ the persistent batched run

// marks every box's status with PAMHD_FLAG_TIMEOUT, once per launch
__device__ void run_timeout(Run_Sync* sync, const Step_Params* boxes, const int nboxes)
{
	if (atomicExch(&sync->error, 1u) == 0u) {
		for (int b = 0; b < nboxes; b++) atomicOr(&boxes[b].status->flags, (unsigned int)PAMHD_FLAG_TIMEOUT);
	}
}

/*
The batched ensemble advanced nsteps steps in one launch.  The grid is the
resident capacity of the SMs (a cooperative launch, so that every block
runs at once).  The work is the sequence of (step, work item) pairs, the
items of a step being the boxes' tiles as in batch_step_kernel, largest
boxes first, then, for boxes with non-periodic sides, chunks of their
ghost-ghost faces, whose speeds enter the timestep.  Blocks take the pairs
one at a time from a shared counter.  An item of step s of box b first
waits until all items of step s - 1 of box b are done (done[b] counts the
box's finished items): the only dependency of a box's step, since each box
has its own state, reduction ring and clock.  Boxes therefore advance at
their own pace, without a grid-wide barrier, and a block that finishes
early takes the next item, of this step or the next.  The pairs are handed
out in order and all blocks are resident, so the earliest unfinished item
has its dependency met: the run always progresses.  A wait gives up after
wait_limit polls: it sets the error word and PAMHD_FLAG_TIMEOUT on every
box, and every block stops at its next item.  boxes_even / boxes_odd are
the boxes' parameters of the two state parities, the first used by step
step0.  Loads that read what another block wrote before go through L2 (CO).
*/
template <int SOLVER, int TY, int MINB>
__global__ void __launch_bounds__(TX * TY, MINB) batch_run_kernel(
	const Step_Params* __restrict__ boxes_even, const Step_Params* __restrict__ boxes_odd,
	const int4* __restrict__ items, const int nitems, const int* __restrict__ box_items, unsigned int* done,
	const int nboxes, const long long step0, const int nsteps, Run_Sync* sync, const long long wait_limit)
{
	extern __shared__ __align__(16) double smem[];
	__shared__ Step_Params sp;
	__shared__ double s_dt;
	__shared__ unsigned int s_q;
	__shared__ int s_go;
	__shared__ int s_stop;
	const int tid = threadIdx.y * blockDim.x + threadIdx.x;
	const int nthreads = blockDim.x * blockDim.y;
	const unsigned int total = (unsigned int)nsteps * (unsigned int)nitems;
	for (;;) {
		__syncthreads();  // the previous item is done with sp and the shared words
		if (tid == 0) {
			volatile unsigned int* verr = &sync->error;
			s_q = *verr != 0u ? total : atomicAdd(&sync->next, 1u);
		}
		__syncthreads();
		const unsigned int q = s_q;
		if (q >= total) return;
		const int s = int(q / (unsigned int)nitems);
		const int4 w = items[q % (unsigned int)nitems];
		const Step_Params* boxes = (s & 1) ? boxes_odd : boxes_even;
		if (tid == 0) {
			// the box's previous step: all its items done
			const unsigned int need = (unsigned int)s * (unsigned int)box_items[w.x];
			volatile unsigned int* vdone = done + w.x;
			volatile unsigned int* verr = &sync->error;
			long long polls = 0;
			int go = 1;
			while (*vdone < need) {
				if (*verr != 0u) {
					go = 0;
					break;
				}
				if (polls >= wait_limit) {
					run_timeout(sync, boxes, nboxes);
					go = 0;
					break;
				}
				polls++;
				__nanosleep(100);
			}
			__threadfence();
			s_go = go;
			sp = boxes[w.x];
			sp.phase = int((step0 + s) % 3);
		}
		__syncthreads();
		if (not s_go) return;
		double smax[3] = {0.0, 0.0, 0.0};
		bool zero = false;
		if (w.w == 0) {
			const bool first = w.y == 0 and w.z == 0;
			const double dt = begin_step(sp, &s_dt, first, &s_stop);
			const int tiles_x = (sp.L.n[0] + TX - 1) / TX;
			if (s_stop) {
				tile_hold<TY, true>(sp, w.y % tiles_x, w.y / tiles_x, w.z);
			} else {
				tile_step<SOLVER, TY, true>(sp, smem, dt, w.y % tiles_x, w.y / tiles_x, w.z, smax[0], smax[1],
				                            smax[2], zero);
			}
		} else if (not stopped_before(sp)) {
			// ghost-ghost faces: combination w.y, faces [w.z BOUNDARY_CHUNK, (w.z + 1) BOUNDARY_CHUNK)
			int combos[12][3];
			const int nc = boundary_combos(sp, combos);
			if (w.y < nc) {
				const int d = combos[w.y][0], side = combos[w.y][1], e = combos[w.y][2];
				const long long count = boundary_count(sp, d, e);
				const long long t1 = min(count, (long long)(w.z + 1) * BOUNDARY_CHUNK);
				for (long long t = (long long)w.z * BOUNDARY_CHUNK + tid; t < t1; t += nthreads) {
					boundary_face<SOLVER, true>(sp, d, side, e, t, smax, zero);
				}
			}
		}
		flush_speeds(sp, smax, zero);
		// publish the item's writes (every thread's), then count it done
		__threadfence();
		__syncthreads();
		if (tid == 0) atomicAdd(done + w.x, 1u);
	}
}

// ------------------------------------------------------------------ solver-level entry

__device__ __forceinline__ Side face_side(const double* s, const double* bg, const bool use_bg, const Gas& g)
{
	Side out;
	out.rho = s[0]; out.m0 = s[1]; out.m1 = s[2]; out.m2 = s[3]; out.E = s[4];
	out.b0 = s[5]; out.b1 = s[6]; out.b2 = s[7];
	const Derived d = derive<true, false, false>(s[0], s[1], s[2], s[3], s[4], s[5], s[6], s[7], g);
	out.rinv = d.rinv;
	out.v0 = d.vx; out.v1 = d.vy; out.v2 = d.vz;
	out.p = d.p;
	out.cf = d.cf[0];
	out.bad = d.bad;
	if (use_bg) {
		// fast speed with the total field (get_fast_magnetosonic_speed, mhd/common.hpp:433-490)
		const double t0 = s[5] + bg[0], t1 = s[6] + bg[1], t2 = s[7] + bg[2];
		const double t2s = t0 * t0 + t1 * t1 + t2 * t2;
		const double cs2 = g.gamma * d.p * d.rinv;
		if (t2s > 0.0) {
			const double va2 = t2s * g.inv_mu0 * d.rinv;
			const double sum2 = cs2 + va2;
			const double to_sqrt = cs2 * cs2 + va2 * va2 + 2.0 * cs2 * va2 * (1.0 - 2.0 * (t0 * t0 / t2s));
			if (out.bad == 0 and not (is_normal(sum2) and to_sqrt > 0.0 and is_normal(to_sqrt))) {
				out.bad = PAMHD_FLAG_WAVE_SPEED;
			}
			out.cf = sqrt(0.5 * (sum2 + sqrt(fmax(to_sqrt, 0.0))));
		} else {
			out.cf = sqrt(fmax(cs2, 0.0));
		}
	}
	return out;
}

template <int SOLVER>
__global__ void face_flux_kernel(long long n, const double* __restrict__ neg, const double* __restrict__ pos,
                                 const double* __restrict__ bg, const Gas g, double* __restrict__ flux,
                                 double* __restrict__ speed, uint32_t* __restrict__ flags)
{
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		const bool use_bg = bg != nullptr and (SOLVER == PAMHD_RUSANOV or SOLVER == PAMHD_HLL_ATHENA);
		const double zero3[3] = {0.0, 0.0, 0.0};
		const double* b = use_bg ? bg + 3 * t : zero3;
		const Side L = face_side(neg + 8 * t, b, use_bg, g);
		const Side R = face_side(pos + 8 * t, b, use_bg, g);
		double F[8];
		uint32_t flag = L.bad | R.bad;
		if (flag & PAMHD_FLAG_DENSITY) flag = PAMHD_FLAG_DENSITY;
		else if (flag & PAMHD_FLAG_PRESSURE) flag = PAMHD_FLAG_PRESSURE;
		double s;
		if (SOLVER == PAMHD_RUSANOV) s = use_bg ? flux_rusanov<true>(L, R, g, F, flag, b) : flux_rusanov<false, true>(L, R, g, F, flag);
		else if (SOLVER == PAMHD_HLL_ATHENA) s = use_bg ? flux_hll<true>(L, R, g, F, flag, b) : flux_hll<false, true>(L, R, g, F, flag);
		else if (SOLVER == PAMHD_HLLD_ATHENA) s = flux_hlld<true>(L, R, g, F, flag);
		else s = flux_roe(L, R, g, F, flag);
		for (int v = 0; v < 8; v++) flux[8 * t + v] = flag ? 0.0 : F[v];
		speed[t] = flag ? 0.0 : s;
		flags[t] = flag;
	}
}

// ------------------------------------------------------------------ conserved totals

/*
Per-block partial sums of the eight conserved variables over interior
cells (compensated summation inside a thread, a fixed-order tree across
the block), so that totals are deterministic run to run.
*/
__global__ void totals_kernel(const double* __restrict__ state, const Layout L, double* __restrict__ partial)
{
	__shared__ double red[8][256];
	const long long n = (long long)L.n[0] * L.n[1] * L.n[2];
	const long long per = (n + gridDim.x - 1) / gridDim.x;
	const long long a = blockIdx.x * per, b = min(n, a + per);
	double sum[8], comp[8];
	for (int v = 0; v < 8; v++) sum[v] = comp[v] = 0.0;
	for (long long t = a + threadIdx.x; t < b; t += blockDim.x) {
		const int i = int(t % L.n[0]);
		const int j = int((t / L.n[0]) % L.n[1]);
		const int k = int(t / ((long long)L.n[0] * L.n[1]));
		const long long o = L.offset(i, j, k);
		for (int v = 0; v < 8; v++) {
			const double y = state[v * L.var + o] - comp[v];
			const double s = sum[v] + y;
			comp[v] = (s - sum[v]) - y;
			sum[v] = s;
		}
	}
	for (int v = 0; v < 8; v++) red[v][threadIdx.x] = sum[v];
	__syncthreads();
	for (int w = blockDim.x / 2; w > 0; w >>= 1) {
		if ((int)threadIdx.x < w) {
			for (int v = 0; v < 8; v++) red[v][threadIdx.x] += red[v][threadIdx.x + w];
		}
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		for (int v = 0; v < 8; v++) partial[8 * blockIdx.x + v] = red[v][0];
	}
}

// ------------------------------------------------------------------ launchers

template <int SOLVER, int TY>
static int prepare_t()
{
	const auto kernel = step_kernel<SOLVER, TY, Step_Minb<SOLVER, TY>::value>;
	cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                     int(tile_bytes<SOLVER, TY>()));
	// all of the SM's memory as shared memory, so that the blocks the registers allow fit
	if (e == cudaSuccess) e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
	return e == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

int prepare_step_kernels(const int solver, const bool y)
{
	switch (solver) {
	case PAMHD_RUSANOV: return y ? prepare_t<PAMHD_RUSANOV, Step_Shape<PAMHD_RUSANOV>::rows>() : prepare_t<PAMHD_RUSANOV, 1>();
	case PAMHD_HLL_ATHENA: return y ? prepare_t<PAMHD_HLL_ATHENA, Step_Shape<PAMHD_HLL_ATHENA>::rows>() : prepare_t<PAMHD_HLL_ATHENA, 1>();
	case PAMHD_HLLD_ATHENA: return y ? prepare_t<PAMHD_HLLD_ATHENA, Step_Shape<PAMHD_HLLD_ATHENA>::rows>() : prepare_t<PAMHD_HLLD_ATHENA, 1>();
	case PAMHD_ROE_ATHENA: return y ? prepare_t<PAMHD_ROE_ATHENA, Step_Shape<PAMHD_ROE_ATHENA>::rows>() : prepare_t<PAMHD_ROE_ATHENA, 1>();
	default: return PAMHD_ERR_ARGUMENT;
	}
}

template <int SOLVER, int TY>
static int launch_step_t(const Step_Params& P, cudaStream_t stream)
{
	const size_t smem = tile_bytes<SOLVER, TY>();
	const dim3 block(TX, TY);
	const int nz = P.L.n[2];
	const int chunks = P.kpart == 1 ? (nz > 1 ? 2 : 1)
	                 : P.kpart == 2 ? (nz - 2 + P.kchunk - 1) / P.kchunk
	                 : (nz + P.kchunk - 1) / P.kchunk;
	if (chunks < 1) return PAMHD_OK;  // no planes between the first and the last
	const dim3 grid((P.L.n[0] + TX - 1) / TX, (P.L.n[1] + TY - 1) / TY, chunks);
	step_kernel<SOLVER, TY, Step_Minb<SOLVER, TY>::value><<<grid, block, smem, stream>>>(P);
	return cudaGetLastError() == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

int launch_step(const Step_Params& P, const int solver, cudaStream_t stream)
{
	const bool y = P.active[1] != 0;
	switch (solver) {
	case PAMHD_RUSANOV: return y ? launch_step_t<PAMHD_RUSANOV, Step_Shape<PAMHD_RUSANOV>::rows>(P, stream) : launch_step_t<PAMHD_RUSANOV, 1>(P, stream);
	case PAMHD_HLL_ATHENA: return y ? launch_step_t<PAMHD_HLL_ATHENA, Step_Shape<PAMHD_HLL_ATHENA>::rows>(P, stream) : launch_step_t<PAMHD_HLL_ATHENA, 1>(P, stream);
	case PAMHD_HLLD_ATHENA: return y ? launch_step_t<PAMHD_HLLD_ATHENA, Step_Shape<PAMHD_HLLD_ATHENA>::rows>(P, stream) : launch_step_t<PAMHD_HLLD_ATHENA, 1>(P, stream);
	case PAMHD_ROE_ATHENA: return y ? launch_step_t<PAMHD_ROE_ATHENA, Step_Shape<PAMHD_ROE_ATHENA>::rows>(P, stream) : launch_step_t<PAMHD_ROE_ATHENA, 1>(P, stream);
	default: return PAMHD_ERR_ARGUMENT;
	}
}

// tile rows the batched step is built for (the autotuner picks one): 1 when y is inactive
constexpr int TY_WIDE = 8;
constexpr int MINB_WIDE = 2;   // resident blocks per SM of the 32 x 8 tile

template <int TY> struct Batch_Build { static constexpr int MINB_OF = MINB; };
template <> struct Batch_Build<TY_WIDE> { static constexpr int MINB_OF = MINB_WIDE; };

template <int SOLVER, int TY>
static int prepare_batch_t()
{
	const cudaError_t e = cudaFuncSetAttribute(batch_step_kernel<SOLVER, TY, Batch_Build<TY>::MINB_OF>,
	                                           cudaFuncAttributeMaxDynamicSharedMemorySize, int(tile_bytes<SOLVER, TY>()));
	return e == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

template <int SOLVER>
static int prepare_batch_s(const int ty)
{
	switch (ty) {
	case 1: return prepare_batch_t<SOLVER, 1>();
	case TY_3D: return prepare_batch_t<SOLVER, TY_3D>();
	case TY_WIDE: return prepare_batch_t<SOLVER, TY_WIDE>();
	default: return PAMHD_ERR_ARGUMENT;
	}
}

int prepare_batch_kernels(const int solver, const int ty)
{
	switch (solver) {
	case PAMHD_RUSANOV: return prepare_batch_s<PAMHD_RUSANOV>(ty);
	case PAMHD_HLL_ATHENA: return prepare_batch_s<PAMHD_HLL_ATHENA>(ty);
	case PAMHD_HLLD_ATHENA: return prepare_batch_s<PAMHD_HLLD_ATHENA>(ty);
	case PAMHD_ROE_ATHENA: return prepare_batch_s<PAMHD_ROE_ATHENA>(ty);
	default: return PAMHD_ERR_ARGUMENT;
	}
}

template <int SOLVER, int TY>
static cudaError_t occupancy_t(int* blocks)
{
	return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, batch_step_kernel<SOLVER, TY, Batch_Build<TY>::MINB_OF>,
	                                                     TX * TY, tile_bytes<SOLVER, TY>());
}

template <int SOLVER>
static cudaError_t occupancy_s(const int ty, int* blocks)
{
	switch (ty) {
	case 1: return occupancy_t<SOLVER, 1>(blocks);
	case TY_3D: return occupancy_t<SOLVER, TY_3D>(blocks);
	case TY_WIDE: return occupancy_t<SOLVER, TY_WIDE>(blocks);
	default: return cudaErrorInvalidValue;
	}
}

int batch_blocks_per_sm(const int solver, const int ty, int* blocks)
{
	cudaError_t e = cudaErrorInvalidValue;
	switch (solver) {
	case PAMHD_RUSANOV: e = occupancy_s<PAMHD_RUSANOV>(ty, blocks); break;
	case PAMHD_HLL_ATHENA: e = occupancy_s<PAMHD_HLL_ATHENA>(ty, blocks); break;
	case PAMHD_HLLD_ATHENA: e = occupancy_s<PAMHD_HLLD_ATHENA>(ty, blocks); break;
	case PAMHD_ROE_ATHENA: e = occupancy_s<PAMHD_ROE_ATHENA>(ty, blocks); break;
	default: return PAMHD_ERR_ARGUMENT;
	}
	return e == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

template <int SOLVER, int TY>
static int prepare_run_t()
{
	const cudaError_t e = cudaFuncSetAttribute(batch_run_kernel<SOLVER, TY, Batch_Build<TY>::MINB_OF>,
	                                           cudaFuncAttributeMaxDynamicSharedMemorySize, int(tile_bytes<SOLVER, TY>()));
	return e == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

template <int SOLVER, int TY>
static cudaError_t run_occupancy_t(int* blocks)
{
	return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks, batch_run_kernel<SOLVER, TY, Batch_Build<TY>::MINB_OF>,
	                                                     TX * TY, tile_bytes<SOLVER, TY>());
}

template <int SOLVER, int TY>
static int launch_run_t(const Step_Params* even, const Step_Params* odd, const int4* items, const int nitems,
                        const int* box_items, unsigned int* done, const int nboxes, const long long step0,
                        const int nsteps, Run_Sync* sync, const long long wait_limit, const int grid,
                        cudaStream_t stream)
{
	cudaLaunchConfig_t c = {};
	c.gridDim = dim3(grid);
	c.blockDim = dim3(TX, TY);
	c.dynamicSmemBytes = tile_bytes<SOLVER, TY>();
	c.stream = stream;
	cudaLaunchAttribute a[1];
	a[0].id = cudaLaunchAttributeCooperative;
	a[0].val.cooperative = 1;
	c.attrs = a;
	c.numAttrs = 1;
	const cudaError_t e = cudaLaunchKernelEx(&c, batch_run_kernel<SOLVER, TY, Batch_Build<TY>::MINB_OF>, even, odd,
	                                         items, nitems, box_items, done, nboxes, step0, nsteps, sync, wait_limit);
	return e == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

template <int SOLVER>
static int prepare_run_s(const int ty)
{
	switch (ty) {
	case 1: return prepare_run_t<SOLVER, 1>();
	case TY_3D: return prepare_run_t<SOLVER, TY_3D>();
	case TY_WIDE: return prepare_run_t<SOLVER, TY_WIDE>();
	default: return PAMHD_ERR_ARGUMENT;
	}
}

template <int SOLVER>
static cudaError_t run_occupancy_s(const int ty, int* blocks)
{
	switch (ty) {
	case 1: return run_occupancy_t<SOLVER, 1>(blocks);
	case TY_3D: return run_occupancy_t<SOLVER, TY_3D>(blocks);
	case TY_WIDE: return run_occupancy_t<SOLVER, TY_WIDE>(blocks);
	default: return cudaErrorInvalidValue;
	}
}

template <int SOLVER>
static int launch_run_s(const Step_Params* even, const Step_Params* odd, const int4* items, const int nitems,
                        const int* box_items, unsigned int* done, const int nboxes, const long long step0,
                        const int nsteps, Run_Sync* sync, const long long wait_limit, const int grid, const int ty,
                        cudaStream_t stream)
{
	switch (ty) {
	case 1: return launch_run_t<SOLVER, 1>(even, odd, items, nitems, box_items, done, nboxes, step0, nsteps, sync, wait_limit, grid, stream);
	case TY_3D: return launch_run_t<SOLVER, TY_3D>(even, odd, items, nitems, box_items, done, nboxes, step0, nsteps, sync, wait_limit, grid, stream);
	case TY_WIDE: return launch_run_t<SOLVER, TY_WIDE>(even, odd, items, nitems, box_items, done, nboxes, step0, nsteps, sync, wait_limit, grid, stream);
	default: return PAMHD_ERR_ARGUMENT;
	}
}

int prepare_batch_run_kernels(const int solver, const int ty)
{
	switch (solver) {
	case PAMHD_RUSANOV: return prepare_run_s<PAMHD_RUSANOV>(ty);
	case PAMHD_HLL_ATHENA: return prepare_run_s<PAMHD_HLL_ATHENA>(ty);
	case PAMHD_HLLD_ATHENA: return prepare_run_s<PAMHD_HLLD_ATHENA>(ty);
	case PAMHD_ROE_ATHENA: return prepare_run_s<PAMHD_ROE_ATHENA>(ty);
	default: return PAMHD_ERR_ARGUMENT;
	}
}

int batch_run_blocks_per_sm(const int solver, const int ty, int* blocks)
{
	cudaError_t e = cudaErrorInvalidValue;
	switch (solver) {
	case PAMHD_RUSANOV: e = run_occupancy_s<PAMHD_RUSANOV>(ty, blocks); break;
	case PAMHD_HLL_ATHENA: e = run_occupancy_s<PAMHD_HLL_ATHENA>(ty, blocks); break;
	case PAMHD_HLLD_ATHENA: e = run_occupancy_s<PAMHD_HLLD_ATHENA>(ty, blocks); break;
	case PAMHD_ROE_ATHENA: e = run_occupancy_s<PAMHD_ROE_ATHENA>(ty, blocks); break;
	default: return PAMHD_ERR_ARGUMENT;
	}
	return e == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

int launch_batch_run(const Step_Params* even, const Step_Params* odd, const int4* items, const int nitems,
                     const int* box_items, unsigned int* done, const int nboxes, const long long step0,
                     const int nsteps, Run_Sync* sync, const long long wait_limit, const int grid, const int solver,
                     const int ty, cudaStream_t stream)
{
	switch (solver) {
	case PAMHD_RUSANOV: return launch_run_s<PAMHD_RUSANOV>(even, odd, items, nitems, box_items, done, nboxes, step0, nsteps, sync, wait_limit, grid, ty, stream);
	case PAMHD_HLL_ATHENA: return launch_run_s<PAMHD_HLL_ATHENA>(even, odd, items, nitems, box_items, done, nboxes, step0, nsteps, sync, wait_limit, grid, ty, stream);
	case PAMHD_HLLD_ATHENA: return launch_run_s<PAMHD_HLLD_ATHENA>(even, odd, items, nitems, box_items, done, nboxes, step0, nsteps, sync, wait_limit, grid, ty, stream);
	case PAMHD_ROE_ATHENA: return launch_run_s<PAMHD_ROE_ATHENA>(even, odd, items, nitems, box_items, done, nboxes, step0, nsteps, sync, wait_limit, grid, ty, stream);
	default: return PAMHD_ERR_ARGUMENT;
	}
}

template <int SOLVER, int TY>
static void launch_batch_t(const Step_Params* boxes, const int4* items, const int nitems, const int phase,
                           const int grid, cudaStream_t stream)
{
	batch_step_kernel<SOLVER, TY, Batch_Build<TY>::MINB_OF><<<grid, dim3(TX, TY), tile_bytes<SOLVER, TY>(), stream>>>(
		boxes, items, nitems, phase);
}

template <int SOLVER>
static int launch_batch_s(const Step_Params* boxes, const int4* items, const int nitems, const int phase,
                          const int grid, const int ty, cudaStream_t stream)
{
	switch (ty) {
	case 1: launch_batch_t<SOLVER, 1>(boxes, items, nitems, phase, grid, stream); break;
	case TY_3D: launch_batch_t<SOLVER, TY_3D>(boxes, items, nitems, phase, grid, stream); break;
	case TY_WIDE: launch_batch_t<SOLVER, TY_WIDE>(boxes, items, nitems, phase, grid, stream); break;
	default: return PAMHD_ERR_ARGUMENT;
	}
	return PAMHD_OK;
}

int launch_batch_step(const Step_Params* boxes, const int4* items, const int nitems, const int phase,
                      const int grid, const int solver, const int ty, cudaStream_t stream)
{
	int rc = PAMHD_ERR_ARGUMENT;
	switch (solver) {
	case PAMHD_RUSANOV: rc = launch_batch_s<PAMHD_RUSANOV>(boxes, items, nitems, phase, grid, ty, stream); break;
	case PAMHD_HLL_ATHENA: rc = launch_batch_s<PAMHD_HLL_ATHENA>(boxes, items, nitems, phase, grid, ty, stream); break;
	case PAMHD_HLLD_ATHENA: rc = launch_batch_s<PAMHD_HLLD_ATHENA>(boxes, items, nitems, phase, grid, ty, stream); break;
	case PAMHD_ROE_ATHENA: rc = launch_batch_s<PAMHD_ROE_ATHENA>(boxes, items, nitems, phase, grid, ty, stream); break;
	default: return PAMHD_ERR_ARGUMENT;
	}
	if (rc != PAMHD_OK) return rc;
	return cudaGetLastError() == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

int launch_batch_boundary_speeds(const Step_Params* boxes, const int nboxes, const int largest, const int phase,
                                 const int solver, cudaStream_t stream)
{
	const dim3 grid(min(1024, (largest + 255) / 256), 12, nboxes);
	switch (solver) {
	case PAMHD_RUSANOV: batch_boundary_speed_kernel<PAMHD_RUSANOV><<<grid, 256, 0, stream>>>(boxes, phase); break;
	case PAMHD_HLL_ATHENA: batch_boundary_speed_kernel<PAMHD_HLL_ATHENA><<<grid, 256, 0, stream>>>(boxes, phase); break;
	case PAMHD_HLLD_ATHENA: batch_boundary_speed_kernel<PAMHD_HLLD_ATHENA><<<grid, 256, 0, stream>>>(boxes, phase); break;
	case PAMHD_ROE_ATHENA: batch_boundary_speed_kernel<PAMHD_ROE_ATHENA><<<grid, 256, 0, stream>>>(boxes, phase); break;
	default: return PAMHD_ERR_ARGUMENT;
	}
	return cudaGetLastError() == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

int launch_boundary_speeds(const Step_Params& P, const int solver, cudaStream_t stream)
{
	int combos = 0, largest = 0;
	for (int d = 0; d < 3; d++) {
		if (not P.active[d] or P.periodic[d]) continue;
		for (int e = 0; e < 3; e++) {
			if (e == d or not P.active[e]) continue;
			combos += 2;
			const int f = 3 - d - e;
			largest = max(largest, P.L.n[e] * P.L.n[f]);
		}
	}
	if (combos == 0) return PAMHD_OK;
	const dim3 grid(min(1024, (largest + 255) / 256), combos);
	switch (solver) {
	case PAMHD_RUSANOV: boundary_speed_kernel<PAMHD_RUSANOV><<<grid, 256, 0, stream>>>(P); break;
	case PAMHD_HLL_ATHENA: boundary_speed_kernel<PAMHD_HLL_ATHENA><<<grid, 256, 0, stream>>>(P); break;
	case PAMHD_HLLD_ATHENA: boundary_speed_kernel<PAMHD_HLLD_ATHENA><<<grid, 256, 0, stream>>>(P); break;
	case PAMHD_ROE_ATHENA: boundary_speed_kernel<PAMHD_ROE_ATHENA><<<grid, 256, 0, stream>>>(P); break;
	default: return PAMHD_ERR_ARGUMENT;
	}
	return cudaGetLastError() == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

int launch_scatter(const double* packed, double* var_base, const Layout& L, cudaStream_t stream)
{
	scatter_kernel<<<1184, 256, 0, stream>>>(packed, var_base, L);
	return cudaGetLastError() == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

int launch_gather(const double* var_base, double* packed, const Layout& L, cudaStream_t stream)
{
	gather_kernel<<<1184, 256, 0, stream>>>(var_base, packed, L);
	return cudaGetLastError() == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

int launch_fill_ghosts_values(const Step_Params& P, double* state, const double lo[3][8], const double hi[3][8],
                              cudaStream_t stream)
{
	Ghost_Values V;
	for (int d = 0; d < 3; d++) {
		for (int v = 0; v < 8; v++) {
			V.lo[d][v] = lo[d][v];
			V.hi[d][v] = hi[d][v];
		}
	}
	fill_ghosts_kernel<<<296, 256, 0, stream>>>(P, state, V);
	return cudaGetLastError() == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

int launch_face_flux(const int solver, const long long n, const double* neg, const double* pos, const double* bg,
                     const Gas& gas, double* flux, double* speed, uint32_t* flags, cudaStream_t stream)
{
	const int blocks = int(min(4096LL, (n + 127) / 128));
	if (blocks == 0) return PAMHD_OK;
	switch (solver) {
	case PAMHD_RUSANOV: face_flux_kernel<PAMHD_RUSANOV><<<blocks, 128, 0, stream>>>(n, neg, pos, bg, gas, flux, speed, flags); break;
	case PAMHD_HLL_ATHENA: face_flux_kernel<PAMHD_HLL_ATHENA><<<blocks, 128, 0, stream>>>(n, neg, pos, bg, gas, flux, speed, flags); break;
	case PAMHD_HLLD_ATHENA: face_flux_kernel<PAMHD_HLLD_ATHENA><<<blocks, 128, 0, stream>>>(n, neg, pos, bg, gas, flux, speed, flags); break;
	case PAMHD_ROE_ATHENA: face_flux_kernel<PAMHD_ROE_ATHENA><<<blocks, 128, 0, stream>>>(n, neg, pos, bg, gas, flux, speed, flags); break;
	default: return PAMHD_ERR_ARGUMENT;
	}
	return cudaGetLastError() == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

int launch_totals(const double* state, const Layout& L, const double /*volume*/, double* partial, const int nblocks,
                  cudaStream_t stream)
{
	totals_kernel<<<nblocks, 256, 0, stream>>>(state, L, partial);
	return cudaGetLastError() == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

} // namespace pamhd_b200
