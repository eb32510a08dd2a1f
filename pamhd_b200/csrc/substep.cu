/*
The cell-centred step with local time stepping (the reference's timestep()
with substeps, mhd/solve.hpp:1837-1924 and substepping.hpp) on uniform
grids periodic in every dimension, behind pamhd_gpu_substep_* of
include/pamhd_gpu.h.  Dimensions of one cell are inactive.

Every cell advances with a period of 2^k substeps of one common substep
length.  A step is planned on the device in one batch of launches, read back
once (the substep count and length), and its substeps launched from the host:
  limits_kernel    each cell's CFL limit from the last face speeds
                   (minimize_timestep, mhd/solve.hpp:1933-2007), the smallest
                   limit and the smallest limit / 2^min over cells
                   (substepping.hpp:312-353), reduced per warp, then one
                   atomicMin per warp on the bits of the non-negative doubles;
  exponent_kernel  floor(log2(min(limit, max_dt) / substep)) capped by the
                   cell's largest exponent (substepping.hpp:364-390);
  restrict_kernel  a cell's exponent at most one above any face or edge
                   neighbour's, repeated until nothing changes (the largest
                   such assignment, which the reference's in-place passes reach
                   too, substepping.hpp:104-176): one pass in the batch, the
                   periods taken on the guess that it changed nothing, and
                   more passes (each read back) only where it did;
  period_kernel,   periods 2^k and their largest value; each cell's smallest
  reach_kernel     period among itself and its face and edge neighbours, M;
then for every substep s:
  faces_kernel     cells with s % M == 0 solve their +d faces and add
                   (substep M) F to both sides' flux slots (get_fluxes,
                   mhd/solve.hpp:254-392), a slot's first contribution
                   since its cell's last update added to zero instead of
                   to the slot's old value;
  update_kernel    cells whose period divides s apply their slots
                   (update_mhd_state, mhd/solve.hpp:1543-1587); the slots
                   are not cleared (the reference zeroes them, :1596-1602),
                   the faces kernel starts them afresh instead.
Layout: state 8 x N, flux slots 6 x 8 x N (each cell's -x, +x, -y, +y, -z,
+z), the speed of every cell's -d face 3 x N, exponents and periods
N int32, x fastest, no ghosts.  One host round trip per step for the plan
(the host needs the substep count to launch the substeps).  Compiled without
FMA contraction; the update follows the oracle's operation order.
*/
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "pamhd_gpu.h"
#include "step.cuh"

using namespace pamhd_b200;

namespace {

constexpr int THREADS = 256;
constexpr int MAX_RESTRICT_PASSES = 64;

struct Plan {
	unsigned long long smallest;   // bits of the smallest CFL limit
	unsigned long long ret;        // bits of the smallest limit / 2^min
	unsigned long long substep;    // bits of the step's substep length (written by exponent_kernel)
	unsigned int max_period;
	unsigned int changed;
	unsigned int bad_exponents;
	unsigned int pad;
};

struct Sub_Params {
	double* U;                 // 8 x N
	double* slot;              // 6 x 8 x N
	double* speed;             // 3 x N
	const int32_t* user_min;   // N
	const int32_t* user_max;   // N
	int32_t* S;                // N exponents
	int32_t* S2;               // N (restriction buffer)
	int32_t* P;                // N periods
	int32_t* M;                // N smallest period of the neighbourhood
	double* T;                 // N CFL limits
	Plan* plan;
	Status* status;
	int n[3];
	int active[3];
	long long N;
	Gas gas;
	double len[3];
	double inv_len[3];
	double cfl;
	int min_offset;            // the smallest user minimum when it is above 0
};

__device__ __forceinline__ long long wrap(const Sub_Params& P, int i, int j, int k)
{
	i = i < 0 ? i + P.n[0] : (i >= P.n[0] ? i - P.n[0] : i);
	j = j < 0 ? j + P.n[1] : (j >= P.n[1] ? j - P.n[1] : j);
	k = k < 0 ? k + P.n[2] : (k >= P.n[2] ? k - P.n[2] : k);
	return (long long)i + (long long)P.n[0] * ((long long)j + (long long)P.n[1] * k);
}

__device__ __forceinline__ void coords(const Sub_Params& P, const long long c, int& i, int& j, int& k)
{
	i = int(c % P.n[0]);
	j = int((c / P.n[0]) % P.n[1]);
	k = int(c / ((long long)P.n[0] * P.n[1]));
}

// calls body(neighbour) for the face and edge neighbours of cell (i, j, k) in the active dimensions
template <class Body>
__device__ __forceinline__ void for_neighbours(const Sub_Params& P, const int i, const int j, const int k, Body body)
{
	for (int dz = -1; dz <= 1; dz++) {
		if (dz != 0 and not P.active[2]) continue;
		for (int dy = -1; dy <= 1; dy++) {
			if (dy != 0 and not P.active[1]) continue;
			for (int dx = -1; dx <= 1; dx++) {
				if (dx != 0 and not P.active[0]) continue;
				const int nonzero = (dx != 0) + (dy != 0) + (dz != 0);
				if (nonzero == 0 or nonzero == 3) continue;
				body(wrap(P, i + dx, j + dy, k + dz));
			}
		}
	}
}

__device__ __forceinline__ unsigned long long bits(const double x)
{
	return (unsigned long long)__double_as_longlong(x);
}

__device__ __forceinline__ double warp_min(double v)
{
	#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
	return v;
}

// each cell's CFL limit (0 when a face speed is <= 0), the smallest limit and limit / 2^min
// (reduced per warp, then one atomicMin per warp on the bits of the non-negative doubles)
__global__ void limits_kernel(const Sub_Params P)
{
	double smallest = DBL_MAX, ret = DBL_MAX;
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < P.N; c += stride) {
		int i, j, k;
		coords(P, c, i, j, k);
		double t = DBL_MAX;
		bool zero = false;
		for (int d = 0; d < 3; d++) {
			if (not P.active[d]) continue;
			const long long up = wrap(P, i + (d == 0), j + (d == 1), k + (d == 2));
			const double vs[2] = {P.speed[d * P.N + up], P.speed[d * P.N + c]};   // +d face, -d face
			for (int f = 0; f < 2; f++) {
				const double v = vs[f];
				if (v <= 0) zero = true;
				else t = fmin(P.cfl * P.len[d] / v, t);
			}
		}
		if (zero) t = 0.0;
		P.T[c] = t;
		const int smin = P.user_min[c] - P.min_offset;
		smallest = fmin(smallest, t);
		ret = fmin(ret, t / (1 << smin));
	}
	smallest = warp_min(smallest);
	ret = warp_min(ret);
	if ((threadIdx.x & 31) == 0) {
		atomicMin(&P.plan->smallest, bits(smallest));
		atomicMin(&P.plan->ret, bits(ret));
	}
}

/*
The substep and the exponents (substepping.hpp:312-390): when max_dt is at
most the smallest limit, every exponent is 0 and the substep is max_dt; else
the substep is the smallest limit / 2^min and each cell's largest exponent is
capped by floor(log2(min(limit, max_dt) / substep)).
*/
__global__ void exponent_kernel(const Sub_Params P, const double max_dt)
{
	const double smallest = __longlong_as_double((long long)P.plan->smallest);
	const double ret = __longlong_as_double((long long)P.plan->ret);
	const bool capped = max_dt <= smallest;
	if (blockIdx.x == 0 and threadIdx.x == 0) {
		P.plan->substep = (unsigned long long)__double_as_longlong(capped ? max_dt : ret);
	}
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < P.N; c += stride) {
		if (capped) {
			P.S[c] = 0;
			continue;
		}
		const double dt = P.T[c];
		int smin = P.user_min[c] - P.min_offset, smax = P.user_max[c];
		if (dt > 0) {
			const int step = max(0, int(floor(log2(fmin(dt, max_dt) / ret))));
			if (smax > step) smax = step;
			if (smin > smax) atomicOr(&P.plan->bad_exponents, 1u);
		} else {
			smax = 0;
		}
		P.S[c] = smax;
	}
}

__global__ void restrict_kernel(const Sub_Params P, const int32_t* __restrict__ in, int32_t* __restrict__ out)
{
	unsigned int changed = 0u;
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < P.N; c += stride) {
		int i, j, k;
		coords(P, c, i, j, k);
		int s = in[c];
		for_neighbours(P, i, j, k, [&](const long long m) { s = min(s, in[m] + 1); });
		out[c] = s;
		if (s != in[c]) changed = 1u;
	}
	if (__any_sync(0xffffffffu, changed != 0u) and (threadIdx.x & 31) == 0) atomicOr(&P.plan->changed, 1u);
}

__global__ void period_kernel(const Sub_Params P)
{
	unsigned int largest = 0u;
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < P.N; c += stride) {
		const int p = 1 << P.S[c];
		P.P[c] = p;
		largest = max(largest, (unsigned int)p);
	}
	largest = __reduce_max_sync(0xffffffffu, largest);
	if ((threadIdx.x & 31) == 0) atomicMax(&P.plan->max_period, largest);
}

__global__ void reach_kernel(const Sub_Params P)
{
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < P.N; c += stride) {
		int i, j, k;
		coords(P, c, i, j, k);
		int m = P.P[c];
		for_neighbours(P, i, j, k, [&](const long long q) { m = min(m, P.P[q]); });
		P.M[c] = m;
	}
}

template <int SOLVER, int A>
__device__ __forceinline__ void plus_face(const Sub_Params& P, const long long c, const int i, const int j,
                                          const int k, const double Uc[8], const Derived& dc, const double min_dt,
                                          const bool fresh_plus, const int sub, const int m)
{
	const long long up = wrap(P, i + (A == 0), j + (A == 1), k + (A == 2));
	double* const plus = P.slot + (size_t(2 * A + 1) * 8) * P.N + c;   // the cell's +A slot
	double* const minus = P.slot + (size_t(2 * A) * 8) * P.N + up;     // the neighbour's -A slot
	/*
	A slot holds the contributions since its cell's last update.  The face is
	solved every m substeps and m divides the periods of both its cells, so its
	first contribution after a cell's update comes at substep sub with (sub - m) a
	multiple of that cell's period: there the slot starts from zero instead of
	being read (the update does not clear it).  The slots are read before the
	solve, so that their latency overlaps its arithmetic.
	*/
	const bool fresh_minus = (sub - m) % P.P[up] == 0;
	double pv[8], mv[8];
	#pragma unroll
	for (int v = 0; v < 8; v++) {
		pv[v] = fresh_plus ? 0.0 : plus[v * P.N];
		mv[v] = fresh_minus ? 0.0 : minus[v * P.N];
	}
	double Uu[8];
	#pragma unroll
	for (int v = 0; v < 8; v++) Uu[v] = P.U[v * P.N + up];
	const Derived du = derive<A == 0, A == 1, A == 2>(Uu[0], Uu[1], Uu[2], Uu[3], Uu[4], Uu[5], Uu[6], Uu[7], P.gas);
	const Side L = side_of<A>(Uc, dc), R = side_of<A>(Uu, du);
	double G[8];
	uint32_t flag = 0;
	// HLLD in explicitly rounded arithmetic, as in the cell-centred step
	const double s = solve_face<SOLVER, SOLVER == PAMHD_HLLD_ATHENA>(L, R, P.gas, G, flag);
	if (flag != 0) {
		atomicOr(&P.status->flags, flag);
		atomicMin(&P.status->first, ((unsigned long long)(c * 3 + A) << 8) | flag);
		return;
	}
	P.speed[A * P.N + up] = s;
	double F[8];
	F[0] = G[0];
	unrotate<A>(G[1], G[2], G[3], F[1], F[2], F[3]);
	F[4] = G[4];
	unrotate<A>(G[5], G[6], G[7], F[5], F[6], F[7]);
	#pragma unroll
	for (int v = 0; v < 8; v++) {
		plus[v * P.N] = pv[v] + min_dt * F[v];
		minus[v * P.N] = mv[v] + min_dt * F[v];
	}
}

template <int SOLVER>
__global__ void __launch_bounds__(128, 3) faces_kernel(const Sub_Params P, const int s)
{
	if (P.status->flags != 0u) return;   // a face of an earlier substep failed: the step stops there
	const double substep = __longlong_as_double((long long)P.plan->substep);
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < P.N; c += stride) {
		const int m = P.M[c];
		if (s % m != 0) continue;
		int i, j, k;
		coords(P, c, i, j, k);
		double Uc[8];
		#pragma unroll
		for (int v = 0; v < 8; v++) Uc[v] = P.U[v * P.N + c];
		const Derived dc = derive<true, true, true>(Uc[0], Uc[1], Uc[2], Uc[3], Uc[4], Uc[5], Uc[6], Uc[7], P.gas);
		const double min_dt = substep * m;
		const bool fresh = (s - m) % P.P[c] == 0;
		if (P.active[0]) plus_face<SOLVER, 0>(P, c, i, j, k, Uc, dc, min_dt, fresh, s, m);
		if (P.active[1]) plus_face<SOLVER, 1>(P, c, i, j, k, Uc, dc, min_dt, fresh, s, m);
		if (P.active[2]) plus_face<SOLVER, 2>(P, c, i, j, k, Uc, dc, min_dt, fresh, s, m);
	}
}

// two blocks per SM (128 registers, a few spilled): 16 warps with their loads in flight
__global__ void __launch_bounds__(THREADS, 2) update_kernel(const Sub_Params P, const int s)
{
	if (P.status->flags != 0u) return;
	const long long N = P.N;
	const long long stride = (long long)gridDim.x * blockDim.x;
	for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N; c += stride) {
		if (s % P.P[c] != 0) continue;
		// every slot read first: 48 independent loads in flight
		double sl_[6][8];
		#pragma unroll
		for (int sl = 0; sl < 6; sl++) {
			#pragma unroll
			for (int v = 0; v < 8; v++) sl_[sl][v] = P.slot[(size_t(sl) * 8 + v) * N + c];
		}
		auto f = [&](const int sl, const int v) -> double { return sl_[sl][v]; };
		double u[8];
		#pragma unroll
		for (int v = 0; v < 8; v++) u[v] = P.U[v * N + c];
		#pragma unroll
		for (int d = 0; d < 3; d++) {
			if (P.active[d]) u[0] += (f(2 * d, 0) - f(2 * d + 1, 0)) / P.len[d];
		}
		#pragma unroll
		for (int d = 0; d < 3; d++) {
			if (not P.active[d]) continue;
			#pragma unroll
			for (int e = 1; e <= 3; e++) u[e] = u[e] + P.inv_len[d] * (f(2 * d, e) + (-f(2 * d + 1, e)));
		}
		#pragma unroll
		for (int d = 0; d < 3; d++) {
			if (P.active[d]) u[4] += (f(2 * d, 4) - f(2 * d + 1, 4)) / P.len[d];
		}
		#pragma unroll
		for (int d = 0; d < 3; d++) {
			if (not P.active[d]) continue;
			#pragma unroll
			for (int e = 5; e <= 7; e++) u[e] = u[e] + P.inv_len[d] * (f(2 * d, e) + (-f(2 * d + 1, e)));
		}
		#pragma unroll
		for (int v = 0; v < 8; v++) P.U[v * N + c] = u[v];
	}
}

int check(const cudaError_t e)
{
	return e == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

#define PAMHD_TRY(expr) do { const int rc_ = (expr); if (rc_ != PAMHD_OK) return rc_; } while (0)

} // namespace

struct pamhd_sub {
	pamhd_cfg cfg;
	int device = 0;
	cudaStream_t stream = nullptr;
	long long N = 0;
	double* U = nullptr;
	double* slot = nullptr;
	double* speed = nullptr;
	int32_t* ints = nullptr;     // user_min, user_max, S, S2, P, M
	double* T = nullptr;
	Plan* plan = nullptr;
	Status* status = nullptr;
	int grid = 0;
	bool loaded = false;
	int32_t last_substeps = 0;
	Sub_Params base;
};

namespace {

template <class K, class... Args>
int launch(const pamhd_sub& x, K kernel, Args... args)
{
	kernel<<<x.grid, THREADS, 0, x.stream>>>(args...);
	return check(cudaGetLastError());
}

int faces(const pamhd_sub& x, const int s)
{
	const int g = 2 * x.grid;
	switch (x.cfg.solver) {
	case PAMHD_RUSANOV: faces_kernel<PAMHD_RUSANOV><<<g, 128, 0, x.stream>>>(x.base, s); break;
	case PAMHD_HLL_ATHENA: faces_kernel<PAMHD_HLL_ATHENA><<<g, 128, 0, x.stream>>>(x.base, s); break;
	case PAMHD_HLLD_ATHENA: faces_kernel<PAMHD_HLLD_ATHENA><<<g, 128, 0, x.stream>>>(x.base, s); break;
	case PAMHD_ROE_ATHENA: faces_kernel<PAMHD_ROE_ATHENA><<<g, 128, 0, x.stream>>>(x.base, s); break;
	default: return PAMHD_ERR_ARGUMENT;
	}
	return check(cudaGetLastError());
}

int read_plan(pamhd_sub& x, Plan& p)
{
	PAMHD_TRY(check(cudaMemcpyAsync(&p, x.plan, sizeof p, cudaMemcpyDeviceToHost, x.stream)));
	return check(cudaStreamSynchronize(x.stream));
}

double from_bits(const unsigned long long b)
{
	double d;
	std::memcpy(&d, &b, sizeof d);
	return d;
}

} // namespace

extern "C" {

int pamhd_gpu_substep_create(const pamhd_cfg* cfg, pamhd_sub** out)
{
	if (cfg == nullptr or out == nullptr) return PAMHD_ERR_ARGUMENT;
	*out = nullptr;
	if (cfg->solver != PAMHD_RUSANOV and cfg->solver != PAMHD_HLL_ATHENA and cfg->solver != PAMHD_HLLD_ATHENA
		and cfg->solver != PAMHD_ROE_ATHENA) {
		return PAMHD_ERR_ARGUMENT;
	}
	int active = 0;
	for (int d = 0; d < 3; d++) {
		if (cfg->n[d] < 1 or not (cfg->cell_length[d] > 0.0)) return PAMHD_ERR_ARGUMENT;
		if (cfg->bc_lo[d] != PAMHD_BC_PERIODIC or cfg->bc_hi[d] != PAMHD_BC_PERIODIC) return PAMHD_ERR_ARGUMENT;
		active += cfg->n[d] > 1;
	}
	if (active == 0 or not (cfg->adiabatic_index > 1.0) or not (cfg->vacuum_permeability > 0.0)
		or not (cfg->time_step_factor > 0.0)) {
		return PAMHD_ERR_ARGUMENT;
	}
	const long long N = (long long)cfg->n[0] * cfg->n[1] * cfg->n[2];
	if (N > (1ll << 30)) return PAMHD_ERR_ARGUMENT;
	pamhd_sub* x = new (std::nothrow) pamhd_sub;
	if (x == nullptr) return PAMHD_ERR_ARGUMENT;
	x->cfg = *cfg;
	x->device = cfg->device;
	x->N = N;
	auto fail = [&](const int rc) {
		pamhd_gpu_substep_destroy(x);
		return rc;
	};
	if (cudaSetDevice(x->device) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	if (cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	const size_t n = size_t(N);
	if (cudaMalloc(&x->U, 8 * n * sizeof(double)) != cudaSuccess
		or cudaMalloc(&x->slot, 48 * n * sizeof(double)) != cudaSuccess
		or cudaMalloc(&x->speed, 3 * n * sizeof(double)) != cudaSuccess
		or cudaMalloc(&x->ints, 6 * n * sizeof(int32_t)) != cudaSuccess
		or cudaMalloc(&x->T, n * sizeof(double)) != cudaSuccess
		or cudaMalloc(&x->plan, sizeof(Plan)) != cudaSuccess
		or cudaMalloc(&x->status, sizeof(Status)) != cudaSuccess) {
		return fail(PAMHD_ERR_CUDA);
	}
	if (cudaMemsetAsync(x->ints, 0, 6 * n * sizeof(int32_t), x->stream) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	int sms = 0;
	if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, x->device) != cudaSuccess) {
		return fail(PAMHD_ERR_CUDA);
	}
	const long long blocks = (N + THREADS - 1) / THREADS;
	x->grid = int(blocks < 8ll * sms ? blocks : 8ll * sms);
	Sub_Params& P = x->base;
	std::memset(&P, 0, sizeof P);
	P.U = x->U;
	P.slot = x->slot;
	P.speed = x->speed;
	P.user_min = x->ints;
	P.user_max = x->ints + n;
	P.S = x->ints + 2 * n;
	P.S2 = x->ints + 3 * n;
	P.P = x->ints + 4 * n;
	P.M = x->ints + 5 * n;
	P.T = x->T;
	P.plan = x->plan;
	P.status = x->status;
	for (int d = 0; d < 3; d++) {
		P.n[d] = cfg->n[d];
		P.active[d] = cfg->n[d] > 1;
		P.len[d] = cfg->cell_length[d];
		P.inv_len[d] = 1 / cfg->cell_length[d];
	}
	P.N = N;
	P.gas.gamma = cfg->adiabatic_index;
	P.gas.mu0 = cfg->vacuum_permeability;
	P.gas.inv_mu0 = 1.0 / cfg->vacuum_permeability;
	P.gas.sqrt_mu0 = std::sqrt(cfg->vacuum_permeability);
	P.gas.inv_sqrt_mu0 = 1.0 / P.gas.sqrt_mu0;
	P.cfl = cfg->time_step_factor;
	P.min_offset = 0;
	if (cudaStreamSynchronize(x->stream) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	*out = x;
	return PAMHD_OK;
}

int pamhd_gpu_substep_destroy(pamhd_sub* x)
{
	if (x == nullptr) return PAMHD_OK;
	cudaSetDevice(x->device);
	if (x->stream != nullptr) cudaStreamSynchronize(x->stream);
	cudaFree(x->U);
	cudaFree(x->slot);
	cudaFree(x->speed);
	cudaFree(x->ints);
	cudaFree(x->T);
	cudaFree(x->plan);
	cudaFree(x->status);
	if (x->stream != nullptr) cudaStreamDestroy(x->stream);
	delete x;
	return PAMHD_OK;
}

int pamhd_gpu_substep_set_state(pamhd_sub* x, const double* const cells[8])
{
	if (x == nullptr or cells == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int v = 0; v < 8; v++) if (cells[v] == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	const size_t n = size_t(x->N);
	for (int v = 0; v < 8; v++) {
		PAMHD_TRY(check(cudaMemcpyAsync(x->U + v * n, cells[v], n * sizeof(double), cudaMemcpyHostToDevice,
		                                x->stream)));
	}
	// no face speeds yet (the first step is the reference's dt = 0 priming step); the flux slots
	// need no clearing: each is written afresh before it is read
	PAMHD_TRY(check(cudaMemsetAsync(x->speed, 0, 3 * n * sizeof(double), x->stream)));
	const Status s{0u, 0u, ~0ull};
	PAMHD_TRY(check(cudaMemcpyAsync(x->status, &s, sizeof s, cudaMemcpyHostToDevice, x->stream)));
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	x->loaded = true;
	return PAMHD_OK;
}

int pamhd_gpu_substep_get_state(pamhd_sub* x, double* const cells[8])
{
	if (x == nullptr or cells == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int v = 0; v < 8; v++) if (cells[v] == nullptr) return PAMHD_ERR_ARGUMENT;
	if (not x->loaded) return PAMHD_ERR_STATE;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	const size_t n = size_t(x->N);
	for (int v = 0; v < 8; v++) {
		PAMHD_TRY(check(cudaMemcpyAsync(cells[v], x->U + v * n, n * sizeof(double), cudaMemcpyDeviceToHost,
		                                x->stream)));
	}
	return check(cudaStreamSynchronize(x->stream));
}

int pamhd_gpu_substep_set_exponents(pamhd_sub* x, const int32_t* mins, const int32_t* maxs)
{
	if (x == nullptr or mins == nullptr or maxs == nullptr) return PAMHD_ERR_ARGUMENT;
	const size_t n = size_t(x->N);
	int lowest = 1 << 30;
	for (size_t c = 0; c < n; c++) {
		if (mins[c] < 0 or maxs[c] < 0 or mins[c] > 30 or maxs[c] > 30) return PAMHD_ERR_ARGUMENT;
		lowest = mins[c] < lowest ? mins[c] : lowest;
	}
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(check(cudaMemcpyAsync(x->ints, mins, n * sizeof(int32_t), cudaMemcpyHostToDevice, x->stream)));
	PAMHD_TRY(check(cudaMemcpyAsync(x->ints + n, maxs, n * sizeof(int32_t), cudaMemcpyHostToDevice, x->stream)));
	x->base.min_offset = lowest > 0 ? lowest : 0;
	return check(cudaStreamSynchronize(x->stream));
}

int pamhd_gpu_substep_step(pamhd_sub* x, const double max_dt, double* dt_taken, int32_t* substeps)
{
	if (x == nullptr or not (max_dt >= 0.0)) return PAMHD_ERR_ARGUMENT;
	if (not x->loaded) return PAMHD_ERR_STATE;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	const Sub_Params& P = x->base;
	Plan p{~0ull, ~0ull, 0ull, 0u, 0u, 0u, 0u};
	PAMHD_TRY(check(cudaMemcpyAsync(x->plan, &p, sizeof p, cudaMemcpyHostToDevice, x->stream)));
	/*
	The plan in one batch and one read-back: limits, substep and exponents, one
	restriction pass (S -> S2), and the periods and their reach taken from S on
	the guess that the pass changed nothing (then S2 equals S).  When it did,
	the passes continue from S2 until nothing changes and the periods are
	taken again.
	*/
	PAMHD_TRY(launch(*x, limits_kernel, P));
	PAMHD_TRY(launch(*x, exponent_kernel, P, max_dt));
	PAMHD_TRY(launch(*x, restrict_kernel, P, static_cast<const int32_t*>(P.S), P.S2));
	PAMHD_TRY(launch(*x, period_kernel, P));
	PAMHD_TRY(launch(*x, reach_kernel, P));
	PAMHD_TRY(read_plan(*x, p));
	if (p.bad_exponents != 0u) return PAMHD_ERR_ARGUMENT;
	if (p.changed != 0u) {
		// restrict_substepping_period: passes until no exponent changes
		int32_t* in = P.S2;
		int32_t* out = P.S;
		for (int pass = 1;; pass++) {
			if (pass == MAX_RESTRICT_PASSES) return PAMHD_ERR_TIMEOUT;
			const unsigned int zero = 0u;
			PAMHD_TRY(check(cudaMemcpyAsync(&x->plan->changed, &zero, sizeof zero, cudaMemcpyHostToDevice,
			                                x->stream)));
			PAMHD_TRY(launch(*x, restrict_kernel, P, static_cast<const int32_t*>(in), out));
			PAMHD_TRY(read_plan(*x, p));
			std::swap(in, out);
			if (p.changed == 0u) break;
		}
		if (in != P.S) {
			PAMHD_TRY(check(cudaMemcpyAsync(P.S, in, size_t(x->N) * sizeof(int32_t), cudaMemcpyDeviceToDevice,
			                                x->stream)));
		}
		const unsigned int zero = 0u;
		PAMHD_TRY(check(cudaMemcpyAsync(&x->plan->max_period, &zero, sizeof zero, cudaMemcpyHostToDevice,
		                                x->stream)));
		PAMHD_TRY(launch(*x, period_kernel, P));
		PAMHD_TRY(launch(*x, reach_kernel, P));
		PAMHD_TRY(read_plan(*x, p));
	}
	const double substep = from_bits(p.substep);
	const int steps = int(p.max_period);
	double total = 0;
	for (int s = 1; s <= steps; s++) {
		total += substep;
		PAMHD_TRY(faces(*x, s));
		PAMHD_TRY(launch(*x, update_kernel, P, s));
	}
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	Status st;
	PAMHD_TRY(check(cudaMemcpy(&st, x->status, sizeof st, cudaMemcpyDeviceToHost)));
	x->last_substeps = steps;
	if (dt_taken != nullptr) *dt_taken = total;
	if (substeps != nullptr) *substeps = steps;
	return st.flags != 0u ? PAMHD_ERR_PHYSICS : PAMHD_OK;
}

int pamhd_gpu_substep_periods(pamhd_sub* x, int32_t* periods)
{
	if (x == nullptr or periods == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(check(cudaMemcpyAsync(periods, x->base.P, size_t(x->N) * sizeof(int32_t), cudaMemcpyDeviceToHost,
	                                x->stream)));
	return check(cudaStreamSynchronize(x->stream));
}

int pamhd_gpu_substep_status(pamhd_sub* x, uint32_t* flags, int32_t cell[3], int32_t* dir)
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

} // extern "C"
