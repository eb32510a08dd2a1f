/*
The staggered-field MHD step (the reference's timestep() with face magnetic
field, mhd/solve.hpp:1837-1924) on uniform grids, behind
pamhd_gpu_staggered_* of include/pamhd_gpu.h.  Periodic grids take the
tiled kernels described here; bounded grids (a layer of boundary cells
outside the walls) the same face and face-field kernels over the grid with
its layer, and the cell and layer kernels described further down.

Data in HBM, every array x fastest over the n0 x n1 x n2 cells, no ghosts
(neighbours wrap around):
  U[2]  cell state, 8 arrays (rho, mom xyz, E, volume B xyz), ping-pong;
  B[2]  normal field of every cell's -x, -y and -z face, 3 arrays, ping-pong
        (the +d face of a cell is the -d face of its +d neighbour);
  F     raw flux through every cell's -d face, 3 x 8 arrays.
A dimension of one cell is its own neighbour, as in the reference's emulated
1-D and 2-D runs: its faces are solved with the cell on both sides.

One step is three launches on the context's stream:
  faces_kernel   every cell solves its three -d faces (the +d faces of its
                 -d neighbours, get_fluxes, mhd/solve.hpp:217-392) from
                 per-cell records staged in shared memory by z-marching
                 tiles, stores the unrotated flux, and max-reduces the face
                 speeds per axis into a three-slot ring, as the fused
                 cell-centred step;
  field_kernel   dt from the previous step's speeds and the cap (lagged CFL
                 rule, mhd/solve.hpp:1933-2007, substepping.hpp:285-338);
                 the new normal field of every cell's three -d faces from
                 the twelve edge terms of assign_face_dBs_f{x,y,z}
                 (mhd/solve.hpp:587-1494, equal-size neighbours), read from
                 planes of tangential fluxes staged in shared memory, and
                 Face_B += Face_dB / area (mhd/solve.hpp:1589-1593);
  cell_kernel    the same dt (all its inputs loaded first); the cell update of update_mhd_state
                 (mhd/solve.hpp:1543-1587), then update_vol_B with constant
                 thermal pressure twice (mhd/solve.hpp:1631-1683,
                 :1895-1918), the volume field the mean of each pair of new
                 faces; advances the clock ring.
This file is compiled without FMA contraction and writes the cell and face
updates in the same operation order as the CPU oracle, so that given the same
face fluxes both compute the same bits.
*/
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "pamhd_gpu.h"
#include "step.cuh"

using namespace pamhd_b200;

namespace {

constexpr int THREADS = 256;

struct Stag_Params {
	const double* __restrict__ U;    // 8 x N
	double* __restrict__ Uo;
	const double* __restrict__ B;    // 3 x N
	double* __restrict__ Bo;
	double* __restrict__ F;          // (3 x 8) x N
	const double* __restrict__ bg;   // (3 x 3) x N background field at every cell's -d face, or nullptr
	int n[3];
	long long N;
	Gas gas;
	double len[3];
	double inv_len[3];
	double area[3];
	double cfl;
	Speed_Max* red;                  // [3], ring by step phase
	Clock* clock;                    // [3]
	Status* status;
	int phase;
	double max_dt;                   // >= 0: cap of dt; < 0: the cap is t_end - t
	double t_end;
	int kchunk;                      // z planes per face-solve block
	int fchunk;                      // z planes per face-field block
	// bounded grids (one layer of boundary cells outside a bounded dimension's walls)
	int ext[3];                      // 1 along a bounded dimension, 0 along a periodic one
	int E[3];                        // cells along each dimension, the layer included (N = E0 E1 E2)
	int value_dim, value_side;       // the VALUE side (value_dim -1: none)
	const Inflow_Table* inflow;      // its time-stamped states, in device memory
};

__device__ __forceinline__ long long wrap_index(const Stag_Params& P, int i, int j, int k)
{
	i = i < 0 ? i + P.n[0] : (i >= P.n[0] ? i - P.n[0] : i);
	j = j < 0 ? j + P.n[1] : (j >= P.n[1] ? j - P.n[1] : j);
	k = k < 0 ? k + P.n[2] : (k >= P.n[2] ? k - P.n[2] : k);
	return (long long)i + (long long)P.n[0] * ((long long)j + (long long)P.n[1] * k);
}

__device__ __forceinline__ void cell_coords(const Stag_Params& P, const long long c, int& i, int& j, int& k)
{
	i = int(c % P.n[0]);
	j = int((c / P.n[0]) % P.n[1]);
	k = int(c / ((long long)P.n[0] * P.n[1]));
}

__device__ __forceinline__ void record_failure(const Stag_Params& P, const uint32_t flag, const long long cell,
                                               const int axis)
{
	atomicOr(&P.status->flags, flag);
	const unsigned long long key = ((unsigned long long)(cell * 3 + axis) << 8) | flag;
	atomicMin(&P.status->first, key);
}

/*
The fast speed of a side with the total field (own + background, in the face
frame), as get_fast_magnetosonic_speed with a background field
(mhd/common.hpp:433-490), and its check.
*/
__device__ __forceinline__ void with_background(Side& s, const double bg[3], const Gas& g)
{
	const double t0 = s.b0 + bg[0], t1 = s.b1 + bg[1], t2 = s.b2 + bg[2];
	const double t2s = t0 * t0 + t1 * t1 + t2 * t2;
	const double cs2 = g.gamma * s.p * s.rinv;
	if (t2s > 0.0) {
		const double va2 = t2s * g.inv_mu0 * s.rinv;
		const double sum2 = cs2 + va2;
		const double to_sqrt = cs2 * cs2 + va2 * va2 + 2.0 * cs2 * va2 * (1.0 - 2.0 * (t0 * t0 / t2s));
		if (s.bad == 0 and not (is_normal(sum2) and to_sqrt > 0.0 and is_normal(to_sqrt))) {
			s.bad = PAMHD_FLAG_WAVE_SPEED;
		}
		s.cf = sqrt(0.5 * (sum2 + sqrt(fmax(to_sqrt, 0.0))));
	} else {
		s.cf = sqrt(fmax(cs2, 0.0));
	}
}

/*
The face solves as tiles: a block of STX x STY threads owns a column of cells
and marches it in z through a chunk of planes.  Each plane's cells, with the
-x column and -y row next to the tile, are read and derived once into a
shared-memory record (state, 1/rho, pressure, fast speed along each axis,
validity per axis) instead of once per face; every cell then solves its three
-d faces from the records, the -z face against the previous plane's record.
Three record slots rotate over the planes, so one barrier per plane keeps a
plane's stores apart from the reads of the plane two before it.
*/
constexpr int STX = 32, STY = 8;            // 256 threads, two blocks per SM (one for Roe)
constexpr int SW = STX + 1;                 // a record row: the -x halo at column 0
constexpr int SCELLS = SW * (STY + 1);      // record rows: the -y halo at row 0
constexpr int SREC = 13;                    // rho, mom xyz, E, B xyz, 1/rho, p, c_f xyz
constexpr int SSLOT = SREC * SCELLS;        // doubles of one slot
constexpr int SSLOTS = 3;
constexpr size_t SMEM_FACES = SSLOTS * (SSLOT * sizeof(double) + SCELLS * sizeof(uint32_t));

/*
Read cell c from HBM and derive its record into slot position r, with the
fast speeds along the axes its faces in the tile need (a halo cell only
along the axis of the face it shares with the tile).
*/
template <bool CX, bool CY, bool CZ>
__device__ __forceinline__ void stage_cell(const Stag_Params& P, double* rec, uint32_t* bad, const int r,
                                           const long long c)
{
	double U[8];
	#pragma unroll
	for (int v = 0; v < 8; v++) U[v] = __ldg(P.U + v * P.N + c);
	const Derived d = derive<CX, CY, CZ>(U[0], U[1], U[2], U[3], U[4], U[5], U[6], U[7], P.gas);
	#pragma unroll
	for (int v = 0; v < 8; v++) rec[v * SCELLS + r] = U[v];
	rec[8 * SCELLS + r] = d.rinv;
	rec[9 * SCELLS + r] = d.p;
	if (CX) rec[10 * SCELLS + r] = d.cf[0];
	if (CY) rec[11 * SCELLS + r] = d.cf[1];
	if (CZ) rec[12 * SCELLS + r] = d.cf[2];
	// one byte of flags per face direction: the reference checks the fast speed of each face
	// along that face's normal, so a failed speed belongs to the failing directions only (with
	// one axis derived, d.bad is that axis's)
	uint32_t packed = d.bad | (d.bad << 8) | (d.bad << 16);
	if (CX and CY and CZ and d.bad == PAMHD_FLAG_WAVE_SPEED) {
		packed = derive<true, false, false>(U[0], U[1], U[2], U[3], U[4], U[5], U[6], U[7], P.gas).bad
			| (derive<false, true, false>(U[0], U[1], U[2], U[3], U[4], U[5], U[6], U[7], P.gas).bad << 8)
			| (derive<false, false, true>(U[0], U[1], U[2], U[3], U[4], U[5], U[6], U[7], P.gas).bad << 16);
	}
	bad[r] = packed;
}

// the cell at slot position r seen from a face normal to axis A (as side_of<A>)
template <int A>
__device__ __forceinline__ Side side_rec(const double* rec, const uint32_t* bad, const int r)
{
	Side s;
	s.rho = rec[r];
	rotate<A>(rec[SCELLS + r], rec[2 * SCELLS + r], rec[3 * SCELLS + r], s.m0, s.m1, s.m2);
	s.E = rec[4 * SCELLS + r];
	rotate<A>(rec[5 * SCELLS + r], rec[6 * SCELLS + r], rec[7 * SCELLS + r], s.b0, s.b1, s.b2);
	s.rinv = rec[8 * SCELLS + r];
	s.p = rec[9 * SCELLS + r];
	s.cf = rec[(10 + A) * SCELLS + r];
	s.v0 = s.m0 * s.rinv;
	s.v1 = s.m1 * s.rinv;
	s.v2 = s.m2 * s.rinv;
	s.bad = (bad[r] >> (8 * A)) & 0xffu;
	return s;
}

// the -A face of cell c between its -A neighbour m (left) and c (right); BG: with the face's
// background field (Rusanov and HLL use it; the reference's HLLD and Roe ignore it)
template <int SOLVER, int A, bool BG>
__device__ __forceinline__ void solve_minus_face(const Stag_Params& P, Side L, Side R, const long long c,
                                                 const long long m, double& smax, bool& zero)
{
	double G[8];
	uint32_t flag = 0;
	double s;
	if (BG) {
		double b[3];
		rotate<A>(P.bg[(3 * A) * P.N + c], P.bg[(3 * A + 1) * P.N + c], P.bg[(3 * A + 2) * P.N + c],
		          b[0], b[1], b[2]);
		with_background(L, b, P.gas);
		with_background(R, b, P.gas);
		flag = L.bad | R.bad;
		if (flag & PAMHD_FLAG_DENSITY) flag = PAMHD_FLAG_DENSITY;
		else if (flag & PAMHD_FLAG_PRESSURE) flag = PAMHD_FLAG_PRESSURE;
		s = SOLVER == PAMHD_RUSANOV ? flux_rusanov<true>(L, R, P.gas, G, flag, b)
		                            : flux_hll<true>(L, R, P.gas, G, flag, b);
	} else {
		// HLLD in explicitly rounded arithmetic (fused multiply-adds: fewer instructions under
		// -fmad=false); the other solvers as written, in the oracle's operation order
		s = solve_face<SOLVER, SOLVER == PAMHD_HLLD_ATHENA>(L, R, P.gas, G, flag);
	}
	if (flag != 0) record_failure(P, flag, m, A);
	smax = fmax(smax, s);
	zero = zero or not (s > 0.0);
	double out[8];
	out[0] = G[0];
	unrotate<A>(G[1], G[2], G[3], out[1], out[2], out[3]);
	out[4] = G[4];
	unrotate<A>(G[5], G[6], G[7], out[5], out[6], out[7]);
	#pragma unroll
	for (int v = 0; v < 8; v++) P.F[(A * 8 + v) * P.N + c] = out[v];
}

__device__ __forceinline__ double warp_max(double v)
{
	#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
	return v;
}

template <int SOLVER, bool BG>
__global__ void __launch_bounds__(STX * STY, SOLVER == PAMHD_ROE_ATHENA ? 1 : 2) faces_kernel(const Stag_Params P)
{
	extern __shared__ __align__(16) double smem[];
	uint32_t* const bad_base = reinterpret_cast<uint32_t*>(smem + SSLOTS * SSLOT);
	const int tx = threadIdx.x, ty = threadIdx.y;
	// the grid with its boundary layer on a bounded grid (E = n on a periodic one)
	const int nx = P.E[0], ny = P.E[1], nz = P.E[2];
	const int gx0 = blockIdx.x * STX, gy0 = blockIdx.y * STY;
	const int gx = gx0 + tx, gy = gy0 + ty;
	const bool own = gx < nx and gy < ny;
	const int kb = blockIdx.z * P.kchunk;
	const int ke = min(nz, kb + P.kchunk);
	const int ri = (ty + 1) * SW + tx + 1;
	// a layer cell's -d face past the low wall has no cell on its other side
	const bool has_x = not (P.ext[0] and gx == 0), has_y = not (P.ext[1] and gy == 0);
	const long long plane = (long long)nx * ny;
	const long long col = gx + (long long)nx * gy;
	// this thread's halo cell, if any: warp 0 the row below the tile (its y speed), warp 1 the column
	// left of it (its x speed)
	int hr = -1;
	long long hcol = 0;
	if (ty == 0 and gx < nx) {
		hr = tx + 1;
		hcol = gx + (long long)nx * (gy0 == 0 ? ny - 1 : gy0 - 1);
	} else if (ty == 1 and tx < STY and gy0 + tx < ny) {
		hr = (tx + 1) * SW;
		hcol = (gx0 == 0 ? nx - 1 : gx0 - 1) + (long long)nx * (gy0 + tx);
	}
	// the -d neighbours' columns (failure reports name the face's negative cell)
	const long long col_mx = (gx == 0 ? nx - 1 : gx - 1) + (long long)nx * gy;
	const long long col_my = gx + (long long)nx * (gy == 0 ? ny - 1 : gy - 1);

	double s0 = 0.0, s1 = 0.0, s2 = 0.0;
	bool zero = false;
	// the plane before the chunk, own cells only: the left sides of the first plane's -z faces
	if (own) stage_cell<false, false, true>(P, smem, bad_base, ri, col + plane * (kb == 0 ? nz - 1 : kb - 1));
	for (int k = kb; k < ke; k++) {
		const int t = k - kb + 1;
		double* const rec = smem + (t % SSLOTS) * SSLOT;
		uint32_t* const bad = bad_base + (t % SSLOTS) * SCELLS;
		const double* const prv = smem + ((t - 1) % SSLOTS) * SSLOT;
		const uint32_t* const pbad = bad_base + ((t - 1) % SSLOTS) * SCELLS;
		const long long kofs = plane * k;
		if (own) stage_cell<true, true, true>(P, rec, bad, ri, col + kofs);
		if (ty == 0) {
			if (hr >= 0) stage_cell<false, true, false>(P, rec, bad, hr, hcol + kofs);
		} else if (hr >= 0) {
			stage_cell<true, false, false>(P, rec, bad, hr, hcol + kofs);
		}
		__syncthreads();
		if (own) {
			const long long c = col + kofs;
			const long long mz = col + plane * (k == 0 ? nz - 1 : k - 1);
			if (has_x) {
				solve_minus_face<SOLVER, 0, BG>(P, side_rec<0>(rec, bad, ri - 1), side_rec<0>(rec, bad, ri), c,
				                                col_mx + kofs, s0, zero);
			}
			if (has_y) {
				solve_minus_face<SOLVER, 1, BG>(P, side_rec<1>(rec, bad, ri - SW), side_rec<1>(rec, bad, ri), c,
				                                col_my + kofs, s1, zero);
			}
			if (not (P.ext[2] and k == 0)) {
				solve_minus_face<SOLVER, 2, BG>(P, side_rec<2>(prv, pbad, ri), side_rec<2>(rec, bad, ri), c, mz,
				                                s2, zero);
			}
		}
	}
	// per-axis maxima of the non-negative speeds, as bit patterns
	s0 = warp_max(s0);
	s1 = warp_max(s1);
	s2 = warp_max(s2);
	const bool any_zero = __any_sync(0xffffffffu, zero);
	if (tx == 0) {
		Speed_Max& r = P.red[(P.phase + 1) % 3];
		atomicMax(&r.smax[0], (unsigned long long)__double_as_longlong(s0));
		atomicMax(&r.smax[1], (unsigned long long)__double_as_longlong(s1));
		atomicMax(&r.smax[2], (unsigned long long)__double_as_longlong(s2));
		if (any_zero) atomicOr(&r.zero, 1u);
	}
}

// dt of the step from the previous step's speeds (solve.hpp:1983-2003, substepping.hpp:331-338)
__device__ __forceinline__ double step_dt(const Stag_Params& P)
{
	const Speed_Max& r = P.red[P.phase];
	bool zero = r.zero != 0;
	double smallest = 1.7976931348623157e308;
	#pragma unroll
	for (int d = 0; d < 3; d++) {
		const double s = __longlong_as_double((long long)r.smax[d]);
		if (not (s > 0.0)) {
			zero = true;
		} else {
			smallest = fmin(smallest, (P.cfl * P.len[d]) / s);
		}
	}
	if (zero) smallest = 0.0;
	const double t = P.clock[P.phase].t;
	const double cap = P.max_dt >= 0.0 ? P.max_dt : P.t_end - t;
	return (cap <= smallest) ? cap : smallest;
}

/*
Change of the normal field of the -D face of a cell, times the face area: the
twelve edge terms of assign_face_dBs_f{x,y,z} that reach the face, in the
order of the oracle (D-directed fluxes one cell away along a and b, then the
a- and b-directed fluxes of the faces sharing an edge with it).
get(axis, comp, ox, oy, oz) is the flux of field component comp through the
-axis face of the cell at offset (ox, oy, oz) from this one.
*/
template <int D, class Get>
__device__ __forceinline__ double face_dB(const Stag_Params& P, const Get& get, const double dt)
{
	constexpr int A = (D + 1) % 3, Bd = (D + 2) % 3;
	const double La = P.len[A], Lb = P.len[Bd];
	auto at = [&](const int axis, const int comp, const int da, const int db, const int dd) {
		int o[3] = {0, 0, 0};
		o[A] += da;
		o[Bd] += db;
		o[D] += dd;
		return get(axis, comp, o[0], o[1], o[2]);
	};
	auto e1 = [&](const int da, const int db, const int dd) { return at(D, A, da, db, dd) * dt * Lb / 4; };
	auto e2 = [&](const int da, const int db, const int dd) { return -(at(D, Bd, da, db, dd) * dt * La / 4); };
	auto e3 = [&](const int da, const int db, const int dd) { return -(at(A, D, da, db, dd) * dt * Lb / 4); };
	auto e4 = [&](const int da, const int db, const int dd) { return at(Bd, D, da, db, dd) * dt * La / 4; };
	double dB = 0;
	dB += e1(+1, 0, 0);
	dB -= e1(-1, 0, 0);
	dB -= e2(0, +1, 0);
	dB += e2(0, -1, 0);
	dB += e3(+1, 0, 0);
	dB += e3(+1, 0, -1);
	dB -= e3(0, 0, 0);
	dB -= e3(0, 0, -1);
	dB -= e4(0, +1, 0);
	dB -= e4(0, +1, -1);
	dB += e4(0, 0, 0);
	dB += e4(0, 0, -1);
	return dB;
}

// get_pressure, mhd/common.hpp:79-118
__device__ __forceinline__ double pressure(const double u[8], const Gas& g)
{
	const double kinetic = 0.5 / u[0] * (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]);
	const double magnetic = 0.5 / g.mu0 * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7]);
	return (u[4] - kinetic - magnetic) * (g.gamma - 1);
}

// update_vol_B with constant thermal pressure for one cell (mhd/solve.hpp:1646-1672)
__device__ __forceinline__ void vol_B_constant_pressure(double u[8], const double mean[3], const Gas& g)
{
	if (u[0] <= 0) return;
	const double p = pressure(u, g);
	u[5] = mean[0];
	u[6] = mean[1];
	u[7] = mean[2];
	const double inv = 1 / u[0];
	const double v0 = u[1] * inv, v1 = u[2] * inv, v2 = u[3] * inv;
	const double kinetic = 0.5 * u[0] * (v0 * v0 + v1 * v1 + v2 * v2);
	const double magnetic = 0.5 / g.mu0 * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7]);
	u[4] = p / (g.gamma - 1) + kinetic + magnetic;
}

// the step's dt, or whether it is skipped: a failed face leaves the state as it was; so does a step past t_end
__device__ __forceinline__ double step_start(const Stag_Params& P, bool& skip)
{
	const Clock c = P.clock[P.phase];
	skip = P.status->flags != 0u or (P.max_dt < 0.0 and c.t >= P.t_end);
	return skip ? 0.0 : step_dt(P);
}

// whether the -D face of cell x is one the step updates: an interior cell's, or a high wall's
template <int D>
__device__ __forceinline__ bool updated_face(const Stag_Params& P, const int x[3])
{
	#pragma unroll
	for (int e = 0; e < 3; e++) {
		const int top = P.n[e] + ((e == D and P.ext[e]) ? 1 : 0);
		if (x[e] < 0 or x[e] >= top) return false;
	}
	return true;
}

/*
Face_B += Face_dB / area for the three -d faces of every cell, as a z-marching
stencil: a block of FTX x FTY threads owns a column of cells; the six
tangential field fluxes (component b of every -a face, a != b) of each plane,
with a one-cell halo in x and y, are staged once in shared memory, and the
twelve terms of each face are read from the planes k - 1, k and k + 1 there.
Four plane slots rotate, so one barrier per plane keeps a plane's stores
apart from the reads of the three planes before it.
*/
constexpr int FTX = 32, FTY = 8;
constexpr int FW = FTX + 2, FH = FTY + 2;
constexpr int FPLANE = 6 * FW * FH;        // doubles of one staged plane
constexpr int FSLOTS = 4;
constexpr size_t SMEM_FIELD = FSLOTS * FPLANE * sizeof(double);

// a thread's share of a staged plane: elements tid + i FTX FTY, i < FPER
constexpr int FPER = (FPLANE + FTX * FTY - 1) / (FTX * FTY);

/*
The six arrays of a staged plane: 2 axis + j holds component (axis + 1 + j)
mod 3 of the -axis faces.  off[i]: the global offset, within its z plane, of
this thread's i-th element (-1 past the plane's end).
*/
__device__ __forceinline__ void plane_offsets(const Stag_Params& P, const int gx0, const int gy0, long long off[FPER])
{
	const int nx = P.E[0], ny = P.E[1];
	const int tid = threadIdx.y * FTX + threadIdx.x;
	#pragma unroll
	for (int i = 0; i < FPER; i++) {
		const int e = tid + i * FTX * FTY;
		off[i] = -1;
		if (e < FPLANE) {
			const int arr = e / (FW * FH);
			const int rem = e - arr * (FW * FH);
			const int row = rem / FW, col = rem - row * FW;
			const int axis = arr >> 1, comp = (axis + 1 + (arr & 1)) % 3;
			const long long x = ((gx0 - 1 + col) % nx + nx) % nx;
			const long long y = ((gy0 - 1 + row) % ny + ny) % ny;
			off[i] = (long long)(axis * 8 + 5 + comp) * P.N + x + nx * y;
		}
	}
}

__device__ __forceinline__ void load_plane(const Stag_Params& P, const long long off[FPER], const int pz, double v[FPER])
{
	const int nz = P.E[2];
	const long long z = (long long)P.E[0] * P.E[1] * (((pz % nz) + nz) % nz);
	#pragma unroll
	for (int i = 0; i < FPER; i++) v[i] = off[i] >= 0 ? P.F[off[i] + z] : 0.0;
}

__device__ __forceinline__ void store_plane(double* slot, const double v[FPER])
{
	const int tid = threadIdx.y * FTX + threadIdx.x;
	#pragma unroll
	for (int i = 0; i < FPER; i++) {
		const int e = tid + i * FTX * FTY;
		if (e < FPLANE) slot[e] = v[i];
	}
}

__global__ void __launch_bounds__(FTX * FTY, 3) field_kernel(const Stag_Params P)
{
	extern __shared__ __align__(16) double fsm[];
	__shared__ double s_dt;
	__shared__ int s_skip;
	const int tx = threadIdx.x, ty = threadIdx.y;
	if (tx == 0 and ty == 0) {
		bool skip;
		s_dt = step_start(P, skip);
		s_skip = skip ? 1 : 0;
	}
	__syncthreads();
	const double dt = s_dt;
	const int nx = P.E[0], ny = P.E[1], nz = P.E[2];
	const int gx0 = blockIdx.x * FTX, gy0 = blockIdx.y * FTY;
	const int gx = gx0 + tx, gy = gy0 + ty;
	const bool own = gx < nx and gy < ny;
	const int kb = blockIdx.z * P.fchunk;
	const int ke = min(nz, kb + P.fchunk);
	const long long plane = (long long)nx * ny;
	const long long col = gx + (long long)nx * gy;
	if (s_skip != 0) {   // the same for the whole block: no barrier is skipped by some threads only
		if (own) {
			for (int k = kb; k < ke; k++) {
				#pragma unroll
				for (int d = 0; d < 3; d++) P.Bo[d * P.N + col + plane * k] = P.B[d * P.N + col + plane * k];
			}
		}
		return;
	}
	long long off[FPER];
	plane_offsets(P, gx0, gy0, off);
	// global plane p sits in slot (p - kb + 1) mod 4; planes kb - 1 .. kb + 1 staged first, the
	// loads of the next plane kept in flight in registers while a plane is computed
	double v[FPER];
	#pragma unroll 1
	for (int t = 0; t < 3; t++) {
		load_plane(P, off, kb - 1 + t, v);
		store_plane(fsm + t * FPLANE, v);
	}
	load_plane(P, off, kb + 2, v);
	for (int k = kb; k < ke; k++) {
		const int t = k - kb + 1;
		__syncthreads();
		if (own) {
			auto get = [&](const int axis, const int comp, const int ox, const int oy, const int oz) {
				const int j = comp == (axis + 1) % 3 ? 0 : 1;
				return fsm[((t + oz) & 3) * FPLANE + (2 * axis + j) * (FW * FH) + (ty + 1 + oy) * FW + tx + 1 + ox];
			};
			const long long c = col + plane * k;
			const double d0 = face_dB<0>(P, get, dt), d1 = face_dB<1>(P, get, dt), d2 = face_dB<2>(P, get, dt);
			const double b0 = P.B[c], b1 = P.B[P.N + c], b2 = P.B[2 * P.N + c];
			// on a bounded grid only the interior cells' faces (the high walls included) change; the
			// layer's are refilled after the step
			const int x[3] = {gx - P.ext[0], gy - P.ext[1], k - P.ext[2]};
			P.Bo[c] = updated_face<0>(P, x) ? b0 + d0 / P.area[0] : b0;
			P.Bo[P.N + c] = updated_face<1>(P, x) ? b1 + d1 / P.area[1] : b1;
			P.Bo[2 * P.N + c] = updated_face<2>(P, x) ? b2 + d2 / P.area[2] : b2;
		}
		// plane k + 2 into its slot (not one of the three the slowest thread may still read), then
		// the loads of plane k + 3
		store_plane(fsm + ((t + 2) & 3) * FPLANE, v);
		if (k + 1 < ke) load_plane(P, off, k + 3, v);
	}
}

/*
The cell update of update_mhd_state (mass, momentum, energy, volume field;
x, then y, then z, each flux slot 0 + dt F as the reference accumulates it),
then update_vol_B twice with the new faces.  Block 0 advances the clock ring.
*/
// two blocks per SM (128 registers, a few spilled): 16 warps with their loads in flight
__global__ void __launch_bounds__(THREADS, 2) cell_kernel(const Stag_Params P)
{
	__shared__ double s_dt;
	__shared__ int s_skip;
	if (threadIdx.x == 0) {
		bool skip;
		const double dt = step_start(P, skip);
		s_dt = dt;
		s_skip = skip ? 1 : 0;
		if (blockIdx.x == 0) {
			const Clock c = P.clock[P.phase];
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
	const bool skip = s_skip != 0;
	const long long N = P.N;
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N; c += stride) {
		if (skip) {
			#pragma unroll
			for (int v = 0; v < 8; v++) P.Uo[v * N + c] = P.U[v * N + c];
			continue;
		}
		int i, j, k;
		cell_coords(P, c, i, j, k);
		const long long up[3] = {wrap_index(P, i + 1, j, k), wrap_index(P, i, j + 1, k), wrap_index(P, i, j, k + 1)};
		// every input read first: 62 independent loads in flight
		double Fm[3][8], Fp[3][8], bm[3], bp[3];
		#pragma unroll
		for (int d = 0; d < 3; d++) {
			#pragma unroll
			for (int v = 0; v < 8; v++) {
				Fm[d][v] = P.F[(d * 8 + v) * N + c];
				Fp[d][v] = P.F[(d * 8 + v) * N + up[d]];
			}
			bm[d] = P.Bo[d * N + c];
			bp[d] = P.Bo[d * N + up[d]];
		}
		auto fm = [&](const int d, const int v) { return 0 + dt * Fm[d][v]; };
		auto fp = [&](const int d, const int v) { return 0 + dt * Fp[d][v]; };
		double u[8];
		#pragma unroll
		for (int v = 0; v < 8; v++) u[v] = P.U[v * N + c];
		#pragma unroll
		for (int d = 0; d < 3; d++) u[0] += (fm(d, 0) - fp(d, 0)) / P.len[d];
		#pragma unroll
		for (int d = 0; d < 3; d++) {
			#pragma unroll
			for (int e = 1; e <= 3; e++) u[e] = u[e] + P.inv_len[d] * (fm(d, e) + (-fp(d, e)));
		}
		#pragma unroll
		for (int d = 0; d < 3; d++) u[4] += (fm(d, 4) - fp(d, 4)) / P.len[d];
		#pragma unroll
		for (int d = 0; d < 3; d++) {
			#pragma unroll
			for (int e = 5; e <= 7; e++) u[e] = u[e] + P.inv_len[d] * (fm(d, e) + (-fp(d, e)));
		}
		const double mean[3] = {0.5 * (bm[0] + bp[0]), 0.5 * (bm[1] + bp[1]), 0.5 * (bm[2] + bp[2])};
		vol_B_constant_pressure(u, mean, P.gas);
		vol_B_constant_pressure(u, mean, P.gas);
		#pragma unroll
		for (int v = 0; v < 8; v++) P.Uo[v * N + c] = u[v];
	}
}

/*
Bounded grids.  The arrays hold the grid with its layer of boundary cells
(E = n + 2 ext cells per dimension, x fastest); periodic dimensions wrap as
above.  The layer follows the reference's solar-wind box (every layer cell a
boundary cell, faces, edges and vertices alike; grid/solar_wind_box.hpp:
268-376): its faces are solved and their speeds enter the timestep, its
cells are refilled from the interior after each step
(apply_boundaries_sw_box, mhd/solar_wind_box.hpp:386-537) and the VALUE
side's plane from its table (apply_solar_wind_boundaries, :227-306).  One
step is five launches:
  faces_kernel          the tiled face solves above over the grid with its
                        layer: every cell's -d faces that have a cell on
                        both sides;
  field_kernel          the tiled face-field stencil above: the new normal
                        field of the interior cells' faces, the walls of
                        bounded dimensions included (the layer's faces are
                        copied and refilled after the step);
and, each a grid-stride loop of one thread per cell,
  bounded_cell_kernel   the interior cells' update, then update_vol_B, the
                        walls' copy sync (sync_magnetic_field: the boundary
                        cell's copy of a wall face is not updated, and the
                        two copies meet about half way), update_vol_B again;
  layer_fill_kernel     the layer from the interior;
  value_fill_kernel     the VALUE plane and the cells on its inner side.
*/
__device__ __forceinline__ int wrap_or_keep(const Stag_Params& P, const int d, const int c)
{
	if (P.ext[d]) return c;
	return c < 0 ? c + P.n[d] : (c >= P.n[d] ? c - P.n[d] : c);
}

// linear index of cell (i, j, k), layer coordinates -1 .. n (periodic dimensions wrap)
__device__ __forceinline__ long long ext_index(const Stag_Params& P, const int i, const int j, const int k)
{
	return (long long)(wrap_or_keep(P, 0, i) + P.ext[0])
		+ (long long)P.E[0] * ((long long)(wrap_or_keep(P, 1, j) + P.ext[1])
		                       + (long long)P.E[1] * (wrap_or_keep(P, 2, k) + P.ext[2]));
}

// coordinates of cell c in 32-bit arithmetic (create keeps N below 2^31)
__device__ __forceinline__ void ext_coords(const Stag_Params& P, const long long c, int x[3])
{
	const unsigned int u = (unsigned int)c, e0 = (unsigned int)P.E[0], e1 = (unsigned int)P.E[1];
	const unsigned int q = u / e0;
	x[0] = int(u - q * e0) - P.ext[0];
	x[1] = int(q % e1) - P.ext[1];
	x[2] = int(q / e1) - P.ext[2];
}

// total energy density from thermal pressure (get_total_energy_density, mhd/common.hpp:258-311)
__device__ __forceinline__ double energy(const double u[8], const double p, const Gas& g)
{
	const double inv = 1 / u[0];
	const double v0 = u[1] * inv, v1 = u[2] * inv, v2 = u[3] * inv;
	const double kinetic = 0.5 * u[0] * (v0 * v0 + v1 * v1 + v2 * v2);
	const double magnetic = 0.5 / g.mu0 * (u[5] * u[5] + u[6] * u[6] + u[7] * u[7]);
	return p / (g.gamma - 1) + kinetic + magnetic;
}

/*
sync_magnetic_field on a wall face (common_functions.hpp:216-251): the
boundary cell's copy `old`, the interior cell's `updated`; the cells in
index order, each visit moving the visitor's copy down by half the
difference and the other's up by as much.  Returns the interior copy.
*/
__device__ __forceinline__ double wall_sync(const double old, const double updated, const bool lo_wall)
{
	if (lo_wall) {
		const double diff1 = old - updated;
		const double g1 = old - diff1 / 2, p1 = updated + diff1 / 2;
		const double diff2 = p1 - g1;
		return p1 - diff2 / 2;
	}
	const double diff1 = updated - old;
	const double p1 = updated - diff1 / 2, g1 = old + diff1 / 2;
	const double diff2 = g1 - p1;
	return p1 + diff2 / 2;
}

// two blocks per SM, as cell_kernel (the loads in flight matter more than a few spilled registers)
__global__ void __launch_bounds__(THREADS, 2) bounded_cell_kernel(const Stag_Params P)
{
	__shared__ double s_dt;
	__shared__ int s_skip;
	if (threadIdx.x == 0) {
		bool skip;
		const double dt = step_start(P, skip);
		s_dt = dt;
		s_skip = skip ? 1 : 0;
		if (blockIdx.x == 0) {
			const Clock c = P.clock[P.phase];
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
	const bool skip = s_skip != 0;
	const long long N = P.N;
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N; c += stride) {
		int x[3];
		ext_coords(P, c, x);
		const bool inside = x[0] >= 0 and x[0] < P.n[0] and x[1] >= 0 and x[1] < P.n[1] and x[2] >= 0
			and x[2] < P.n[2];
		if (skip or not inside) {
			#pragma unroll
			for (int v = 0; v < 8; v++) P.Uo[v * N + c] = P.U[v * N + c];
			continue;
		}
		const long long up[3] = {ext_index(P, x[0] + 1, x[1], x[2]), ext_index(P, x[0], x[1] + 1, x[2]),
		                         ext_index(P, x[0], x[1], x[2] + 1)};
		double Fm[3][8], Fp[3][8], bm[3], bp[3];
		#pragma unroll
		for (int d = 0; d < 3; d++) {
			#pragma unroll
			for (int v = 0; v < 8; v++) {
				Fm[d][v] = P.F[(d * 8 + v) * N + c];
				Fp[d][v] = P.F[(d * 8 + v) * N + up[d]];
			}
			bm[d] = P.Bo[d * N + c];
			bp[d] = P.Bo[d * N + up[d]];
		}
		auto fm = [&](const int d, const int v) { return 0 + dt * Fm[d][v]; };
		auto fp = [&](const int d, const int v) { return 0 + dt * Fp[d][v]; };
		double u[8];
		#pragma unroll
		for (int v = 0; v < 8; v++) u[v] = P.U[v * N + c];
		#pragma unroll
		for (int d = 0; d < 3; d++) u[0] += (fm(d, 0) - fp(d, 0)) / P.len[d];
		#pragma unroll
		for (int d = 0; d < 3; d++) {
			#pragma unroll
			for (int e = 1; e <= 3; e++) u[e] = u[e] + P.inv_len[d] * (fm(d, e) + (-fp(d, e)));
		}
		#pragma unroll
		for (int d = 0; d < 3; d++) u[4] += (fm(d, 4) - fp(d, 4)) / P.len[d];
		#pragma unroll
		for (int d = 0; d < 3; d++) {
			#pragma unroll
			for (int e = 5; e <= 7; e++) u[e] = u[e] + P.inv_len[d] * (fm(d, e) + (-fp(d, e)));
		}
		const double mean1[3] = {0.5 * (bm[0] + bp[0]), 0.5 * (bm[1] + bp[1]), 0.5 * (bm[2] + bp[2])};
		vol_B_constant_pressure(u, mean1, P.gas);
		// the walls' copies (this cell is the only interior cell on each of its walls)
		#pragma unroll
		for (int d = 0; d < 3; d++) {
			if (not P.ext[d]) continue;
			if (x[d] == 0) {
				bm[d] = wall_sync(P.B[d * N + c], bm[d], true);
				P.Bo[d * N + c] = bm[d];
			}
			if (x[d] == P.n[d] - 1) {
				bp[d] = wall_sync(P.B[d * N + up[d]], bp[d], false);
				P.Bo[d * N + up[d]] = bp[d];
			}
		}
		const double mean2[3] = {0.5 * (bm[0] + bp[0]), 0.5 * (bm[1] + bp[1]), 0.5 * (bm[2] + bp[2])};
		vol_B_constant_pressure(u, mean2, P.gas);
		#pragma unroll
		for (int v = 0; v < 8; v++) P.Uo[v * N + c] = u[v];
	}
}

/*
The layer from the interior (apply_boundaries_sw_box, mhd/solar_wind_box.hpp:
386-537), into the arrays U, B: each layer cell from the interior cell it
touches through a face, an edge or a vertex; its faces from that cell's,
mirrored across the walls it lies behind; volume field the face means;
total energy from the source cell's thermal pressure.  Reads interior cells
and the faces they hold only, writes layer cells and the faces they hold, so
the threads never meet.  check: skip when the step was skipped.
*/
__global__ void __launch_bounds__(THREADS) layer_fill_kernel(const Stag_Params P, double* U, double* B,
                                                             const bool check)
{
	if (check) {
		bool skip;
		step_start(P, skip);
		if (skip) return;
	}
	const long long N = P.N;
	// the layer's cells only, enumerated as the planes below and above the box (along a bounded z),
	// then the rows in front and behind between them (bounded y), then the columns left and right
	const long long nz_planes = P.ext[2] ? 2ll * P.E[0] * P.E[1] : 0;
	const long long ny_rows = P.ext[1] ? 2ll * P.E[0] * P.n[2] : 0;
	const long long nx_cols = P.ext[0] ? 2ll * P.n[1] * P.n[2] : 0;
	const long long count = nz_planes + ny_rows + nx_cols;
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < count; t += stride) {
		int x[3], s[3];
		if (t < nz_planes) {
			const long long r = t % ((long long)P.E[0] * P.E[1]);
			x[0] = int(r % P.E[0]) - P.ext[0];
			x[1] = int(r / P.E[0]) - P.ext[1];
			x[2] = t < nz_planes / 2 ? -1 : P.n[2];
		} else if (t < nz_planes + ny_rows) {
			const long long u = t - nz_planes, r = u % ((long long)P.E[0] * P.n[2]);
			x[0] = int(r % P.E[0]) - P.ext[0];
			x[1] = u < ny_rows / 2 ? -1 : P.n[1];
			x[2] = int(r / P.E[0]);
		} else {
			const long long u = t - nz_planes - ny_rows, r = u % ((long long)P.n[1] * P.n[2]);
			x[0] = u < nx_cols / 2 ? -1 : P.n[0];
			x[1] = int(r % P.n[1]);
			x[2] = int(r / P.n[1]);
		}
		const long long c = ext_index(P, x[0], x[1], x[2]);
		bool shell[3];
		#pragma unroll
		for (int d = 0; d < 3; d++) {
			shell[d] = x[d] < 0 or x[d] >= P.n[d];
			s[d] = x[d] < 0 ? 0 : (x[d] >= P.n[d] ? P.n[d] - 1 : x[d]);
		}
		const long long src = ext_index(P, s[0], s[1], s[2]);
		double u[8];
		#pragma unroll
		for (int v = 0; v < 8; v++) u[v] = U[v * N + src];
		const double p = pressure(u, P.gas);
		#pragma unroll
		for (int e = 0; e < 3; e++) {
			int o[3] = {s[0], s[1], s[2]};
			o[e] += 1;
			const double lo = B[e * N + src], hi = B[e * N + ext_index(P, o[0], o[1], o[2])];
			int f[3] = {s[0], s[1], s[2]};
			f[e] = (shell[e] and x[e] < 0) ? 1 : x[e];
			const long long fi = ext_index(P, f[0], f[1], f[2]);
			if (fi != c) B[e * N + c] = B[e * N + fi];
			u[5 + e] = shell[e] ? 0.5 * (hi + lo) : 0.5 * (lo + hi);
		}
		u[4] = energy(u, p, P.gas);
		#pragma unroll
		for (int v = 0; v < 8; v++) U[v * N + c] = u[v];
	}
}

__device__ __forceinline__ const double* table_state(const Inflow_Table& T, const double t)
{
	int i = 0;
	while (i < T.count and t >= T.times[i]) i++;
	return T.states + 8 * i;
}

/*
The VALUE plane (apply_solar_wind_boundaries, mhd/solar_wind_box.hpp:227-306)
at the time in clock slot tslot: its cells take the table's state, every
face of theirs its field; each cell on the plane's inner side gets the
state's normal field on the face it shares with the plane, half of each of
its two faces along that dimension as its volume field component, and its
total energy from its thermal pressure before the change.  One thread per
plane cell.
*/
__global__ void __launch_bounds__(THREADS) value_fill_kernel(const Stag_Params P, double* U, double* B,
                                                             const int tslot, const bool check)
{
	if (check) {
		bool skip;
		step_start(P, skip);
		if (skip) return;
	}
	const int d = P.value_dim, a = (d + 1) % 3, b = (d + 2) % 3;
	const bool lo = P.value_side == 0;
	const double* v = table_state(*P.inflow, P.clock[tslot].t);
	const long long N = P.N, count = (long long)P.E[a] * P.E[b];
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < count; t += stride) {
		int x[3];
		x[d] = lo ? -1 : P.n[d];
		x[a] = int(t % P.E[a]) - P.ext[a];
		x[b] = int(t / P.E[a]) - P.ext[b];
		const long long c = ext_index(P, x[0], x[1], x[2]);
		#pragma unroll
		for (int k = 0; k < 8; k++) U[k * N + c] = v[k];
		#pragma unroll
		for (int e = 0; e < 3; e++) B[e * N + c] = v[5 + e];
		int q[3] = {x[0], x[1], x[2]};
		q[d] = lo ? 0 : P.n[d] - 1;
		const long long qi = ext_index(P, q[0], q[1], q[2]);
		q[d] += 1;
		const long long qu = ext_index(P, q[0], q[1], q[2]);
		const long long shared = lo ? qi : qu, other = lo ? qu : qi;
		double u[8];
		#pragma unroll
		for (int k = 0; k < 8; k++) u[k] = U[k * N + qi];
		const double p = pressure(u, P.gas);
		B[d * N + shared] = v[5 + d];
		u[5 + d] = B[d * N + shared] / 2 + B[d * N + other] / 2;
		u[4] = energy(u, p, P.gas);
		#pragma unroll
		for (int k = 0; k < 8; k++) U[k * N + qi] = u[k];
	}
}

// interior cells and faces between the packed arrays of the ABI and the layered ones
__global__ void __launch_bounds__(THREADS) bounded_pack_kernel(const Stag_Params P, double* U, double* B,
                                                               double* packed, const bool to_packed)
{
	const long long cells = (long long)P.n[0] * P.n[1] * P.n[2];
	long long fcount[3], total = 8 * cells;
	#pragma unroll
	for (int d = 0; d < 3; d++) {
		fcount[d] = cells / P.n[d] * (P.n[d] + P.ext[d]);
		total += fcount[d];
	}
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += stride) {
		double* dev;
		if (t < 8 * cells) {
			const int v = int(t / cells);
			const long long r = t - v * cells;
			const int i = int(r % P.n[0]), j = int((r / P.n[0]) % P.n[1]), k = int(r / ((long long)P.n[0] * P.n[1]));
			dev = U + v * P.N + ext_index(P, i, j, k);
		} else {
			long long r = t - 8 * cells;
			int d = 0;
			while (r >= fcount[d]) r -= fcount[d++];
			int ext[3] = {P.n[0], P.n[1], P.n[2]};
			ext[d] += P.ext[d];
			const int i = int(r % ext[0]), j = int((r / ext[0]) % ext[1]), k = int(r / ((long long)ext[0] * ext[1]));
			dev = B + d * P.N + ext_index(P, i, j, k);
		}
		if (to_packed) packed[t] = *dev;
		else *dev = packed[t];
	}
}

// the face kernels' shared memory above the default 48 KB, once per kernel
template <int SOLVER>
int allow_face_smem()
{
	constexpr bool USES_BG = SOLVER == PAMHD_RUSANOV or SOLVER == PAMHD_HLL_ATHENA;
	if (cudaFuncSetAttribute(faces_kernel<SOLVER, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                         int(SMEM_FACES)) != cudaSuccess) {
		return PAMHD_ERR_CUDA;
	}
	if (USES_BG and cudaFuncSetAttribute(faces_kernel<SOLVER, USES_BG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
	                                     int(SMEM_FACES)) != cudaSuccess) {
		return PAMHD_ERR_CUDA;
	}
	return PAMHD_OK;
}

template <int SOLVER>
int launch_pair(const Stag_Params& P, const int grid, cudaStream_t stream)
{
	constexpr bool USES_BG = SOLVER == PAMHD_RUSANOV or SOLVER == PAMHD_HLL_ATHENA;
	const dim3 tiles((P.E[0] + STX - 1) / STX, (P.E[1] + STY - 1) / STY, (P.E[2] + P.kchunk - 1) / P.kchunk);
	const dim3 block(STX, STY);
	if (USES_BG and P.bg != nullptr) {
		faces_kernel<SOLVER, USES_BG><<<tiles, block, SMEM_FACES, stream>>>(P);
	} else {
		faces_kernel<SOLVER, false><<<tiles, block, SMEM_FACES, stream>>>(P);
	}
	if (cudaGetLastError() != cudaSuccess) return PAMHD_ERR_CUDA;
	const dim3 field_tiles((P.E[0] + FTX - 1) / FTX, (P.E[1] + FTY - 1) / FTY, (P.E[2] + P.fchunk - 1) / P.fchunk);
	field_kernel<<<field_tiles, dim3(FTX, FTY), SMEM_FIELD, stream>>>(P);
	if (cudaGetLastError() != cudaSuccess) return PAMHD_ERR_CUDA;
	cell_kernel<<<grid, THREADS, 0, stream>>>(P);
	return cudaGetLastError() == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

// the five launches of a step on a bounded grid
template <int SOLVER>
int launch_bounded(const Stag_Params& P, const int grid, cudaStream_t stream)
{
	// the tiled face solves and face-field stencil over the grid with its layer, then the cell
	// update with the walls' copy sync, the layer and the inflow plane
	const dim3 tiles((P.E[0] + STX - 1) / STX, (P.E[1] + STY - 1) / STY, (P.E[2] + P.kchunk - 1) / P.kchunk);
	faces_kernel<SOLVER, false><<<tiles, dim3(STX, STY), SMEM_FACES, stream>>>(P);
	const dim3 field_tiles((P.E[0] + FTX - 1) / FTX, (P.E[1] + FTY - 1) / FTY, (P.E[2] + P.fchunk - 1) / P.fchunk);
	field_kernel<<<field_tiles, dim3(FTX, FTY), SMEM_FIELD, stream>>>(P);
	bounded_cell_kernel<<<grid, THREADS, 0, stream>>>(P);
	layer_fill_kernel<<<grid, THREADS, 0, stream>>>(P, P.Uo, P.Bo, true);
	if (P.value_dim >= 0) {
		const long long count = (long long)P.E[(P.value_dim + 1) % 3] * P.E[(P.value_dim + 2) % 3];
		value_fill_kernel<<<int((count + THREADS - 1) / THREADS), THREADS, 0, stream>>>(
			P, P.Uo, P.Bo, (P.phase + 1) % 3, true);
	}
	return cudaGetLastError() == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

int check(const cudaError_t e)
{
	return e == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

#define PAMHD_TRY(expr) do { const int rc_ = (expr); if (rc_ != PAMHD_OK) return rc_; } while (0)

} // namespace

struct pamhd_stag {
	pamhd_cfg cfg;
	int device = 0;
	cudaStream_t stream = nullptr;
	long long N = 0;
	double* U[2] = {nullptr, nullptr};
	double* B[2] = {nullptr, nullptr};
	double* F = nullptr;
	double* bg = nullptr;        // background field, 9 x N, allocated by set_background
	Speed_Max* red = nullptr;
	Clock* clock = nullptr;
	Status* status = nullptr;
	int cur = 0;
	long long steps = 0;         // launched steps since set_state (the ring phase)
	int grid = 0;
	bool loaded = false;
	bool bounded = false;        // a layer of boundary cells outside some walls
	long long packed = 0;        // doubles of the ABI's state arrays (cells and faces)
	double* stage = nullptr;     // device staging of those arrays (bounded grids)
	Inflow_Table* table = nullptr;   // the VALUE side's table in device memory
	double* table_data = nullptr;    // its timestamps and states
	Stag_Params base;
};

namespace {

Stag_Params params_of(const pamhd_stag& x, const double max_dt, const double t_end)
{
	Stag_Params P = x.base;
	P.U = x.U[x.cur];
	P.Uo = x.U[x.cur ^ 1];
	P.B = x.B[x.cur];
	P.Bo = x.B[x.cur ^ 1];
	P.phase = int(x.steps % 3);
	P.max_dt = max_dt;
	P.t_end = t_end;
	return P;
}

int issue(pamhd_stag& x, const double max_dt, const double t_end)
{
	const Stag_Params P = params_of(x, max_dt, t_end);
	int rc = PAMHD_ERR_ARGUMENT;
	if (x.bounded) {
		switch (x.cfg.solver) {
		case PAMHD_RUSANOV: rc = launch_bounded<PAMHD_RUSANOV>(P, x.grid, x.stream); break;
		case PAMHD_HLL_ATHENA: rc = launch_bounded<PAMHD_HLL_ATHENA>(P, x.grid, x.stream); break;
		case PAMHD_HLLD_ATHENA: rc = launch_bounded<PAMHD_HLLD_ATHENA>(P, x.grid, x.stream); break;
		case PAMHD_ROE_ATHENA: rc = launch_bounded<PAMHD_ROE_ATHENA>(P, x.grid, x.stream); break;
		default: break;
		}
	} else {
		switch (x.cfg.solver) {
		case PAMHD_RUSANOV: rc = launch_pair<PAMHD_RUSANOV>(P, x.grid, x.stream); break;
		case PAMHD_HLL_ATHENA: rc = launch_pair<PAMHD_HLL_ATHENA>(P, x.grid, x.stream); break;
		case PAMHD_HLLD_ATHENA: rc = launch_pair<PAMHD_HLLD_ATHENA>(P, x.grid, x.stream); break;
		case PAMHD_ROE_ATHENA: rc = launch_pair<PAMHD_ROE_ATHENA>(P, x.grid, x.stream); break;
		default: break;
		}
	}
	if (rc != PAMHD_OK) return rc;
	x.cur ^= 1;
	x.steps++;
	return PAMHD_OK;
}

int reset_ring(pamhd_stag& x)
{
	Speed_Max r[3] = {};
	r[0].zero = 1u;   // no speeds yet: the first step's dt is 0 unless capped lower
	const Clock c[3] = {};
	const Status s{0u, 0u, ~0ull};
	PAMHD_TRY(check(cudaMemcpyAsync(x.red, r, sizeof r, cudaMemcpyHostToDevice, x.stream)));
	PAMHD_TRY(check(cudaMemcpyAsync(x.clock, c, sizeof c, cudaMemcpyHostToDevice, x.stream)));
	PAMHD_TRY(check(cudaMemcpyAsync(x.status, &s, sizeof s, cudaMemcpyHostToDevice, x.stream)));
	x.steps = 0;
	return check(cudaStreamSynchronize(x.stream));
}

// a dimension with a layer of boundary cells: not periodic, two cells or more
bool bounded_dim(const pamhd_cfg& c, const int d)
{
	return c.n[d] > 1 and not (c.bc_lo[d] == PAMHD_BC_PERIODIC and c.bc_hi[d] == PAMHD_BC_PERIODIC);
}

int validate_stag(const pamhd_cfg& c)
{
	if (c.solver != PAMHD_RUSANOV and c.solver != PAMHD_HLL_ATHENA and c.solver != PAMHD_HLLD_ATHENA
		and c.solver != PAMHD_ROE_ATHENA) {
		return PAMHD_ERR_ARGUMENT;
	}
	int values = 0;
	long long N = 1;
	for (int d = 0; d < 3; d++) {
		if (c.n[d] < 1 or not (c.cell_length[d] > 0.0)) return PAMHD_ERR_ARGUMENT;
		const int kinds[2] = {c.bc_lo[d], c.bc_hi[d]};
		for (const int k: kinds) {
			if (k != PAMHD_BC_PERIODIC and k != PAMHD_BC_COPY and k != PAMHD_BC_VALUE) return PAMHD_ERR_ARGUMENT;
			if (k == PAMHD_BC_VALUE) values++;
		}
		// periodic on both sides or on neither; a dimension of one cell is its own (periodic) neighbour
		if ((kinds[0] == PAMHD_BC_PERIODIC) != (kinds[1] == PAMHD_BC_PERIODIC)) return PAMHD_ERR_ARGUMENT;
		if (c.n[d] == 1 and kinds[0] != PAMHD_BC_PERIODIC) return PAMHD_ERR_ARGUMENT;
		N *= c.n[d] + (bounded_dim(c, d) ? 2 : 0);
	}
	if (values > 1) return PAMHD_ERR_ARGUMENT;   // one inflow side, as the solar-wind box's
	if (not (c.adiabatic_index > 1.0) or not (c.vacuum_permeability > 0.0) or not (c.time_step_factor > 0.0)) {
		return PAMHD_ERR_ARGUMENT;
	}
	if (N > (1ll << 31)) return PAMHD_ERR_ARGUMENT;
	if ((c.n[1] + STY - 1) / STY > 65535) return PAMHD_ERR_ARGUMENT;   // rows of face tiles: the grid's y extent
	return PAMHD_OK;
}

// the VALUE side's table: count timestamps, count + 1 states of 8 doubles (host memory)
int upload_table(pamhd_stag& x, const int32_t count, const double* times, const double* states)
{
	const size_t nt = size_t(count), ns = 8 * (size_t(count) + 1);
	double* data = nullptr;
	PAMHD_TRY(check(cudaMalloc(&data, (nt + ns) * sizeof(double))));
	Inflow_Table t;
	t.times = data;
	t.states = data + nt;
	t.count = count;
	if ((nt > 0 and cudaMemcpy(data, times, nt * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
		or cudaMemcpy(data + nt, states, ns * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess
		or cudaMemcpy(x.table, &t, sizeof t, cudaMemcpyHostToDevice) != cudaSuccess) {
		cudaFree(data);
		return PAMHD_ERR_CUDA;
	}
	cudaFree(x.table_data);
	x.table_data = data;
	return PAMHD_OK;
}

// the layer (and the VALUE plane) of the current state from its interior, at the current time
int fill_layer(pamhd_stag& x)
{
	Stag_Params P = params_of(x, -1.0, 0.0);
	double* U = x.U[x.cur];
	double* B = x.B[x.cur];
	layer_fill_kernel<<<x.grid, THREADS, 0, x.stream>>>(P, U, B, false);
	if (P.value_dim >= 0) {
		const long long count = (long long)P.E[(P.value_dim + 1) % 3] * P.E[(P.value_dim + 2) % 3];
		value_fill_kernel<<<int((count + THREADS - 1) / THREADS), THREADS, 0, x.stream>>>(P, U, B, P.phase, false);
	}
	return check(cudaGetLastError());
}

// doubles of one array of the ABI: cell variable v (face < 0) or the faces normal to axis `face`
size_t packed_length(const pamhd_cfg& c, const int v, const int face)
{
	(void)v;
	size_t len = 1;
	for (int d = 0; d < 3; d++) len *= size_t(c.n[d] + ((d == face and bounded_dim(c, d)) ? 1 : 0));
	return len;
}

} // namespace

extern "C" {

int pamhd_gpu_staggered_create(const pamhd_cfg* cfg, pamhd_stag** out)
{
	if (cfg == nullptr or out == nullptr) return PAMHD_ERR_ARGUMENT;
	*out = nullptr;
	PAMHD_TRY(validate_stag(*cfg));
	pamhd_stag* x = new (std::nothrow) pamhd_stag;
	if (x == nullptr) return PAMHD_ERR_ARGUMENT;
	x->cfg = *cfg;
	x->device = cfg->device;
	int ext[3];
	x->N = 1;
	x->packed = 8ll * cfg->n[0] * cfg->n[1] * cfg->n[2];
	for (int d = 0; d < 3; d++) {
		ext[d] = bounded_dim(*cfg, d) ? 1 : 0;
		x->bounded = x->bounded or ext[d] != 0;
		x->N *= cfg->n[d] + 2 * ext[d];
		x->packed += (long long)cfg->n[0] * cfg->n[1] * cfg->n[2] / cfg->n[d] * (cfg->n[d] + ext[d]);
	}
	auto fail = [&](const int rc) {
		pamhd_gpu_staggered_destroy(x);
		return rc;
	};
	if (cudaSetDevice(x->device) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	if (cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	const size_t n = size_t(x->N);
	if (cudaMalloc(&x->U[0], 8 * n * sizeof(double)) != cudaSuccess
		or cudaMalloc(&x->U[1], 8 * n * sizeof(double)) != cudaSuccess
		or cudaMalloc(&x->B[0], 3 * n * sizeof(double)) != cudaSuccess
		or cudaMalloc(&x->B[1], 3 * n * sizeof(double)) != cudaSuccess
		or cudaMalloc(&x->F, 24 * n * sizeof(double)) != cudaSuccess
		or cudaMalloc(&x->red, 3 * sizeof(Speed_Max)) != cudaSuccess
		or cudaMalloc(&x->clock, 3 * sizeof(Clock)) != cudaSuccess
		or cudaMalloc(&x->status, sizeof(Status)) != cudaSuccess) {
		return fail(PAMHD_ERR_CUDA);
	}
	if (x->bounded and cudaMalloc(&x->stage, size_t(x->packed) * sizeof(double)) != cudaSuccess) {
		return fail(PAMHD_ERR_CUDA);
	}
	int sms = 0;
	if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, x->device) != cudaSuccess) {
		return fail(PAMHD_ERR_CUDA);
	}
	const long long blocks = (x->N + THREADS - 1) / THREADS;
	x->grid = int(blocks < 8ll * sms ? blocks : 8ll * sms);
	int rc = PAMHD_ERR_ARGUMENT;
	switch (cfg->solver) {
	case PAMHD_RUSANOV: rc = allow_face_smem<PAMHD_RUSANOV>(); break;
	case PAMHD_HLL_ATHENA: rc = allow_face_smem<PAMHD_HLL_ATHENA>(); break;
	case PAMHD_HLLD_ATHENA: rc = allow_face_smem<PAMHD_HLLD_ATHENA>(); break;
	case PAMHD_ROE_ATHENA: rc = allow_face_smem<PAMHD_ROE_ATHENA>(); break;
	default: break;
	}
	if (rc != PAMHD_OK) return fail(rc);
	Stag_Params& P = x->base;
	P = Stag_Params{};
	// z chunks so that the face tiles fill the SMs about six times over
	// (over the grid with its boundary layer on a bounded grid)
	int E[3];
	for (int d = 0; d < 3; d++) E[d] = cfg->n[d] + 2 * ext[d];
	const long long tiles = (long long)((E[0] + STX - 1) / STX) * ((E[1] + STY - 1) / STY);
	const long long chunks = std::max(1ll, std::min((long long)E[2], 18ll * sms / tiles));
	P.kchunk = int((E[2] + chunks - 1) / chunks);
	const long long ftiles = (long long)((E[0] + FTX - 1) / FTX) * ((E[1] + FTY - 1) / FTY);
	const long long fchunks = std::max(1ll, std::min((long long)E[2], 12ll * sms / ftiles));
	P.fchunk = int((E[2] + fchunks - 1) / fchunks);
	if (cudaFuncSetAttribute(field_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM_FIELD))
		!= cudaSuccess) {
		return fail(PAMHD_ERR_CUDA);
	}
	for (int d = 0; d < 3; d++) {
		P.n[d] = cfg->n[d];
		P.len[d] = cfg->cell_length[d];
		P.inv_len[d] = 1 / cfg->cell_length[d];
	}
	P.area[0] = cfg->cell_length[1] * cfg->cell_length[2];
	P.area[1] = cfg->cell_length[0] * cfg->cell_length[2];
	P.area[2] = cfg->cell_length[0] * cfg->cell_length[1];
	P.N = x->N;
	P.gas.gamma = cfg->adiabatic_index;
	P.gas.mu0 = cfg->vacuum_permeability;
	P.gas.inv_mu0 = 1.0 / cfg->vacuum_permeability;
	P.gas.sqrt_mu0 = std::sqrt(cfg->vacuum_permeability);
	P.gas.inv_sqrt_mu0 = 1.0 / P.gas.sqrt_mu0;
	P.cfl = cfg->time_step_factor;
	P.F = x->F;
	P.red = x->red;
	P.clock = x->clock;
	P.status = x->status;
	P.value_dim = -1;
	for (int d = 0; d < 3; d++) {
		P.ext[d] = ext[d];
		P.E[d] = cfg->n[d] + 2 * ext[d];
		if (ext[d] and (cfg->bc_lo[d] == PAMHD_BC_VALUE or cfg->bc_hi[d] == PAMHD_BC_VALUE)) {
			P.value_dim = d;
			P.value_side = cfg->bc_lo[d] == PAMHD_BC_VALUE ? 0 : 1;
		}
	}
	if (P.value_dim >= 0) {
		// a constant table: the configured state until pamhd_gpu_staggered_set_inflow gives one
		if (cudaMalloc(&x->table, sizeof(Inflow_Table)) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
		const double* v = P.value_side == 0 ? cfg->value_lo[P.value_dim] : cfg->value_hi[P.value_dim];
		if (upload_table(*x, 0, nullptr, v) != PAMHD_OK) return fail(PAMHD_ERR_CUDA);
		P.inflow = x->table;
	}
	if (cudaMemsetAsync(x->U[0], 0, 8 * n * sizeof(double), x->stream) != cudaSuccess
		or cudaMemsetAsync(x->B[0], 0, 3 * n * sizeof(double), x->stream) != cudaSuccess) {
		return fail(PAMHD_ERR_CUDA);
	}
	if (reset_ring(*x) != PAMHD_OK) return fail(PAMHD_ERR_CUDA);
	*out = x;
	return PAMHD_OK;
}

int pamhd_gpu_staggered_destroy(pamhd_stag* x)
{
	if (x == nullptr) return PAMHD_OK;
	cudaSetDevice(x->device);
	if (x->stream != nullptr) cudaStreamSynchronize(x->stream);
	cudaFree(x->U[0]);
	cudaFree(x->U[1]);
	cudaFree(x->B[0]);
	cudaFree(x->B[1]);
	cudaFree(x->F);
	cudaFree(x->bg);
	cudaFree(x->red);
	cudaFree(x->clock);
	cudaFree(x->status);
	cudaFree(x->stage);
	cudaFree(x->table);
	cudaFree(x->table_data);
	if (x->stream != nullptr) cudaStreamDestroy(x->stream);
	delete x;
	return PAMHD_OK;
}

int pamhd_gpu_staggered_set_state(pamhd_stag* x, const double* const cells[8], const double* const faces[3])
{
	if (x == nullptr or cells == nullptr or faces == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int v = 0; v < 8; v++) if (cells[v] == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int d = 0; d < 3; d++) if (faces[d] == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	const size_t n = size_t(x->N);
	x->cur = 0;
	if (x->bounded) {
		// the caller's arrays into the staging buffer, from there into the layered arrays; then the
		// layer from the interior at time 0
		size_t at = 0;
		for (int v = 0; v < 8; v++) {
			const size_t len = packed_length(x->cfg, v, -1);
			PAMHD_TRY(check(cudaMemcpyAsync(x->stage + at, cells[v], len * sizeof(double), cudaMemcpyHostToDevice,
			                                x->stream)));
			at += len;
		}
		for (int d = 0; d < 3; d++) {
			const size_t len = packed_length(x->cfg, 0, d);
			PAMHD_TRY(check(cudaMemcpyAsync(x->stage + at, faces[d], len * sizeof(double), cudaMemcpyHostToDevice,
			                                x->stream)));
			at += len;
		}
		PAMHD_TRY(reset_ring(*x));
		const Stag_Params P = params_of(*x, -1.0, 0.0);
		bounded_pack_kernel<<<x->grid, THREADS, 0, x->stream>>>(P, x->U[0], x->B[0], x->stage, false);
		PAMHD_TRY(check(cudaGetLastError()));
		PAMHD_TRY(fill_layer(*x));
		PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
		x->loaded = true;
		return PAMHD_OK;
	}
	// one copy per array straight from the caller's memory (at full speed when it is pinned)
	for (int v = 0; v < 8; v++) {
		PAMHD_TRY(check(cudaMemcpyAsync(x->U[0] + v * n, cells[v], n * sizeof(double), cudaMemcpyHostToDevice,
		                                x->stream)));
	}
	for (int d = 0; d < 3; d++) {
		PAMHD_TRY(check(cudaMemcpyAsync(x->B[0] + d * n, faces[d], n * sizeof(double), cudaMemcpyHostToDevice,
		                                x->stream)));
	}
	PAMHD_TRY(reset_ring(*x));
	x->loaded = true;
	return PAMHD_OK;
}

int pamhd_gpu_staggered_set_inflow(pamhd_stag* x, const int32_t dim, const int32_t side, const int32_t count,
                                   const double* times, const double* states)
{
	if (x == nullptr or dim < 0 or dim > 2 or (side != 0 and side != 1) or count < 0) return PAMHD_ERR_ARGUMENT;
	if ((count > 0 and times == nullptr) or states == nullptr) return PAMHD_ERR_ARGUMENT;
	if (x->base.value_dim != dim or x->base.value_side != side) return PAMHD_ERR_ARGUMENT;
	for (int i = 0; i < count; i++) {
		if (not std::isfinite(times[i]) or (i > 0 and not (times[i] > times[i - 1]))) return PAMHD_ERR_ARGUMENT;
	}
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	PAMHD_TRY(upload_table(*x, count, times, states));
	// the plane of the current state at the current time
	if (x->loaded) {
		PAMHD_TRY(fill_layer(*x));
		PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	}
	return PAMHD_OK;
}

int pamhd_gpu_staggered_set_background(pamhd_stag* x, const double* const bg[9])
{
	if (x == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	if (bg == nullptr) {
		x->base.bg = nullptr;
		return PAMHD_OK;
	}
	for (int k = 0; k < 9; k++) if (bg[k] == nullptr) return PAMHD_ERR_ARGUMENT;
	if (x->bounded) return PAMHD_ERR_ARGUMENT;   // a background field on periodic grids only
	const size_t n = size_t(x->N);
	if (x->bg == nullptr) PAMHD_TRY(check(cudaMalloc(&x->bg, 9 * n * sizeof(double))));
	for (int k = 0; k < 9; k++) {
		PAMHD_TRY(check(cudaMemcpy(x->bg + k * n, bg[k], n * sizeof(double), cudaMemcpyHostToDevice)));
	}
	x->base.bg = x->bg;
	return PAMHD_OK;
}

int pamhd_gpu_staggered_get_state(pamhd_stag* x, double* const cells[8], double* const faces[3])
{
	if (x == nullptr or cells == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int v = 0; v < 8; v++) if (cells[v] == nullptr) return PAMHD_ERR_ARGUMENT;
	if (faces != nullptr) {
		for (int d = 0; d < 3; d++) if (faces[d] == nullptr) return PAMHD_ERR_ARGUMENT;
	}
	if (not x->loaded) return PAMHD_ERR_STATE;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	const size_t n = size_t(x->N);
	if (x->bounded) {
		const Stag_Params P = params_of(*x, -1.0, 0.0);
		bounded_pack_kernel<<<x->grid, THREADS, 0, x->stream>>>(P, x->U[x->cur], x->B[x->cur], x->stage, true);
		PAMHD_TRY(check(cudaGetLastError()));
		size_t at = 0;
		for (int v = 0; v < 8; v++) {
			const size_t len = packed_length(x->cfg, v, -1);
			PAMHD_TRY(check(cudaMemcpyAsync(cells[v], x->stage + at, len * sizeof(double), cudaMemcpyDeviceToHost,
			                                x->stream)));
			at += len;
		}
		for (int d = 0; faces != nullptr and d < 3; d++) {
			const size_t len = packed_length(x->cfg, 0, d);
			PAMHD_TRY(check(cudaMemcpyAsync(faces[d], x->stage + at, len * sizeof(double), cudaMemcpyDeviceToHost,
			                                x->stream)));
			at += len;
		}
		return check(cudaStreamSynchronize(x->stream));
	}
	for (int v = 0; v < 8; v++) {
		PAMHD_TRY(check(cudaMemcpyAsync(cells[v], x->U[x->cur] + v * n, n * sizeof(double), cudaMemcpyDeviceToHost,
		                                x->stream)));
	}
	if (faces != nullptr) {
		for (int d = 0; d < 3; d++) {
			PAMHD_TRY(check(cudaMemcpyAsync(faces[d], x->B[x->cur] + d * n, n * sizeof(double),
			                                cudaMemcpyDeviceToHost, x->stream)));
		}
	}
	return check(cudaStreamSynchronize(x->stream));
}

int pamhd_gpu_staggered_sync(pamhd_stag* x)
{
	if (x == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	Status s;
	PAMHD_TRY(check(cudaMemcpy(&s, x->status, sizeof s, cudaMemcpyDeviceToHost)));
	return s.flags != 0u ? PAMHD_ERR_PHYSICS : PAMHD_OK;
}

int pamhd_gpu_staggered_step(pamhd_stag* x, const double max_dt, double* dt_taken)
{
	if (x == nullptr or not (max_dt >= 0.0)) return PAMHD_ERR_ARGUMENT;
	if (not x->loaded) return PAMHD_ERR_STATE;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(issue(*x, max_dt, 0.0));
	const int rc = pamhd_gpu_staggered_sync(x);
	if (dt_taken != nullptr) {
		Clock c;
		PAMHD_TRY(check(cudaMemcpy(&c, x->clock + (x->steps % 3), sizeof c, cudaMemcpyDeviceToHost)));
		*dt_taken = rc == PAMHD_OK ? c.dt : 0.0;
	}
	return rc;
}

int pamhd_gpu_staggered_steps(pamhd_stag* x, const int32_t nsteps, const double t_end)
{
	if (x == nullptr or nsteps < 0 or not (t_end == t_end)) return PAMHD_ERR_ARGUMENT;
	if (not x->loaded) return PAMHD_ERR_STATE;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	for (int32_t s = 0; s < nsteps; s++) PAMHD_TRY(issue(*x, -1.0, t_end));
	return PAMHD_OK;
}

int pamhd_gpu_staggered_time(pamhd_stag* x, double* time, int64_t* steps, double* last_dt)
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

int pamhd_gpu_staggered_status(pamhd_stag* x, uint32_t* flags, int32_t cell[3], int32_t* dir)
{
	if (x == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	Status s;
	PAMHD_TRY(check(cudaMemcpy(&s, x->status, sizeof s, cudaMemcpyDeviceToHost)));
	if (flags != nullptr) *flags = s.flags;
	if (s.flags != 0u and s.first != ~0ull) {
		const long long key = (long long)(s.first >> 8);
		const long long c = key / 3;
		// the face's negative cell, in layer coordinates (-1 .. n along a bounded dimension)
		const int* E = x->base.E;
		const int* ext = x->base.ext;
		if (cell != nullptr) {
			cell[0] = int32_t(c % E[0]) - ext[0];
			cell[1] = int32_t((c / E[0]) % E[1]) - ext[1];
			cell[2] = int32_t(c / ((long long)E[0] * E[1])) - ext[2];
		}
		if (dir != nullptr) *dir = int32_t(key % 3) + 1;
	} else {
		if (cell != nullptr) cell[0] = cell[1] = cell[2] = -1;
		if (dir != nullptr) *dir = 0;
	}
	return PAMHD_OK;
}

int pamhd_gpu_staggered_get_stream(pamhd_stag* x, void** stream)
{
	if (x == nullptr or stream == nullptr) return PAMHD_ERR_ARGUMENT;
	*stream = static_cast<void*>(x->stream);
	return PAMHD_OK;
}

} // extern "C"
