/*
Discrete adjoint of the step map on the GPU, with checkpoint-and-recompute.

The step is U_{n+1} = U_n + dt_n / d_len sum over faces of +-F(U_L, U_R)
(mhd/solve.hpp:1543-1587 and the fluxes of :217-392); the adjoint runs on
the forward run's dt schedule, frozen (dt_n is a constant of the
linearisation).  With lambda = dJ/dU_{n+1}, one reverse step is

  phi_f  = dt_n / d_len (lambda_R - lambda_L)      (cotangent of F_f; ghosts have lambda 0)
  g_L, g_R = (dF/dU_L)^T phi_f, (dF/dU_R)^T phi_f  (face_vjp, adjoint_face.cuh)
  lambda_n = lambda + sum over the cell's faces of its g,
             a ghost's g going to the cell it is made from (periodic image,
             COPY source) or, for VALUE sides, to the inflow-state gradient.

Kernels: faces_vjp_kernel (one launch for every active axis: one thread
per face, one solver VJP instance for every axis; writes g_L and g_R as 16
arrays per axis, x fastest, so that reads and writes are coalesced), gather_kernel (one thread per cell, sums
its faces in a fixed order: deterministic), value_side_kernel (sums the
ghost gradients of VALUE sides, one block per side, fixed order; launched
only when the grid has a VALUE side).

Driver (pamhd_gpu_adjoint): the forward run stores the state every K
steps and keeps every state of the last two segments (they fill the two
segment buffers, so no recompute is needed for them); the reverse sweep steps
lambda back through each segment while the segment before it is
recomputed from its checkpoint on a second stream (same kernels, so the
same bits), into the other of two segment buffers.  Memory: ceil(N/K)
checkpoints + 2 (K - 1) state copies, kept by the context between calls.
*/
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "adjoint_face.cuh"
#include "context.cuh"

namespace pamhd_b200 {
int launch_fill_ghosts_values(const Step_Params& P, double* state, const double lo[3][8], const double hi[3][8],
                              cudaStream_t stream);
}

namespace {

using pamhd_b200::adjoint::Gas_Adj;

struct Adj_Params {
	const double* U;      // state at step n, ghosts valid
	const double* lam;    // dJ/dU_{n+1}, padded layout, ghosts zero
	double* lam_out;      // dJ/dU_n
	double* G[3];         // per axis: 16 arrays of nf[d] doubles, g_L then g_R in the state's variable order
	long long nf[3];      // faces per axis
	Layout L;
	Gas_Adj gas;
	double dt;
	double inv_len[3];
	int active[3];
	int periodic[3];
	int bc_lo[3];
	int bc_hi[3];
};

__host__ __device__ inline long long faces_of(const Layout& L, const int d)
{
	const int e = (d + 1) % 3, f = (d + 2) % 3;
	return (long long)(L.n[d] + 1) * L.n[e] * L.n[f];
}

/*
Index of the face of axis D whose lower cell is (c0, c1, c2): c_D runs over
-1 .. n_D - 1, the other coordinates over the interior; x fastest, so that
the faces of consecutive threads are consecutive in memory.
*/
template <int D>
__device__ __forceinline__ long long face_at(const Layout& L, const int c0, const int c1, const int c2)
{
	constexpr int s0 = D == 0, s1 = D == 1, s2 = D == 2;
	const long long N0 = L.n[0] + s0, N1 = L.n[1] + s1;
	return (c0 + s0) + N0 * ((c1 + s1) + N1 * (long long)(c2 + s2));
}

/*
Cotangents of every face of every active axis in one launch: one thread per
face.  The faces of axis d are numbered as face_at<d> numbers them (lower
cell c with c_d from -1 to n_d - 1, the other coordinates interior, x
fastest), one axis after another, so consecutive threads read consecutive
cells and write consecutive entries of the 16 arrays of their axis.  The
axis is a run-time value (the rotation into the face frame a permutation
of the variables read and written), so the kernel holds one instance of
the solver's VJP.  A ghost cell has lambda 0; its g goes to the cell it is
made from in gather_kernel.
*/
template <int SOLVER>
__global__ void __launch_bounds__(128) faces_vjp_kernel(const Adj_Params A)
{
	const long long n0 = A.active[0] ? A.nf[0] : 0, n1 = A.active[1] ? A.nf[1] : 0;
	const long long n2 = A.active[2] ? A.nf[2] : 0;
	const long long count = n0 + n1 + n2;
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < count;
	     t += (long long)gridDim.x * blockDim.x) {
		const int D = t < n0 ? 0 : (t < n0 + n1 ? 1 : 2);
		const long long idx = t - (D == 0 ? 0 : (D == 1 ? n0 : n0 + n1));
		const int E = D == 2 ? 0 : D + 1, F = D == 0 ? 2 : D - 1;
		const long long N0 = A.L.n[0] + (D == 0), N1 = A.L.n[1] + (D == 1);
		int c[3];
		c[0] = int(idx % N0) - (D == 0);
		c[1] = int((idx / N0) % N1) - (D == 1);
		c[2] = int(idx / (N0 * N1)) - (D == 2);
		int r[3] = {c[0], c[1], c[2]};
		r[D] += 1;
		const long long oL = A.L.offset(c[0], c[1], c[2]), oR = A.L.offset(r[0], r[1], r[2]);
		const bool lam_l = c[D] >= 0, lam_r = r[D] <= A.L.n[D] - 1;
		const double scale = A.dt * A.inv_len[D];
		const int perm[8] = {0, 1 + D, 1 + E, 1 + F, 4, 5 + D, 5 + E, 5 + F};
		double uL[8], uR[8], phi[8];
		#pragma unroll
		for (int v = 0; v < 8; v++) {
			const long long o = perm[v] * A.L.var;
			uL[v] = A.U[o + oL];
			uR[v] = A.U[o + oR];
			const double ll = lam_l ? A.lam[o + oL] : 0.0;
			const double lr = lam_r ? A.lam[o + oR] : 0.0;
			phi[v] = scale * (lr - ll);
		}
		double gL[8], gR[8];
		pamhd_b200::adjoint::face_vjp<SOLVER>(uL, uR, A.gas, phi, gL, gR);
		double* G = A.G[D];
		const long long nf = A.nf[D];
		#pragma unroll
		for (int v = 0; v < 8; v++) {
			G[perm[v] * nf + idx] = gL[v];
			G[(8 + perm[v]) * nf + idx] = gR[v];
		}
	}
}

// adds to acc the cotangents that axis D's faces give the interior cell c, ghosts included
template <int D>
__device__ __forceinline__ void gather_axis(const Adj_Params& A, const int* c, double* acc)
{
	const double* G = A.G[D];
	const long long nf = A.nf[D];
	const int nd = A.L.n[D];
	int m[3] = {c[0], c[1], c[2]};
	m[D] -= 1;
	// the cell is the right side of its -D face and the left side of its +D face
	const long long i_minus = face_at<D>(A.L, m[0], m[1], m[2]);
	const long long i_plus = face_at<D>(A.L, c[0], c[1], c[2]);
	#pragma unroll
	for (int v = 0; v < 8; v++) acc[v] += G[(8 + v) * nf + i_minus] + G[v * nf + i_plus];
	// ghosts made from this cell: a periodic image, or a COPY ghost (equal to its source cell in
	// exact arithmetic: identity Jacobian)
	const bool first = c[D] == 0, last = c[D] == nd - 1;
	const bool from_lo = A.periodic[D] ? last : (first and A.bc_lo[D] == PAMHD_BC_COPY);
	const bool from_hi = A.periodic[D] ? first : (last and A.bc_hi[D] == PAMHD_BC_COPY);
	if (from_lo) {   // the ghost at -1 is this cell: left side of the face with lower cell -1
		int g[3] = {c[0], c[1], c[2]};
		g[D] = -1;
		const long long i = face_at<D>(A.L, g[0], g[1], g[2]);
		#pragma unroll
		for (int v = 0; v < 8; v++) acc[v] += G[v * nf + i];
	}
	if (from_hi) {   // the ghost at n is this cell: right side of the face with lower cell n - 1
		int g[3] = {c[0], c[1], c[2]};
		g[D] = nd - 1;
		const long long i = face_at<D>(A.L, g[0], g[1], g[2]);
		#pragma unroll
		for (int v = 0; v < 8; v++) acc[v] += G[(8 + v) * nf + i];
	}
}

// lambda_n = lambda_{n+1} + the cotangents of each interior cell's faces, summed in a fixed order
__global__ void gather_kernel(const Adj_Params A)
{
	const long long n = (long long)A.L.n[0] * A.L.n[1] * A.L.n[2];
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
		int c[3];
		c[0] = int(t % A.L.n[0]);
		c[1] = int((t / A.L.n[0]) % A.L.n[1]);
		c[2] = int(t / ((long long)A.L.n[0] * A.L.n[1]));
		const long long o = A.L.offset(c[0], c[1], c[2]);
		double acc[8];
		#pragma unroll
		for (int v = 0; v < 8; v++) acc[v] = A.lam[v * A.L.var + o];
		if (A.active[0]) gather_axis<0>(A, c, acc);
		if (A.active[1]) gather_axis<1>(A, c, acc);
		if (A.active[2]) gather_axis<2>(A, c, acc);
		#pragma unroll
		for (int v = 0; v < 8; v++) A.lam_out[v * A.L.var + o] = acc[v];
	}
}

template <int D>
__device__ __forceinline__ const double* value_ghost_cotangent(const Adj_Params& A, const int side, const int ce,
                                                               const int cf, long long& stride)
{
	constexpr int E = (D + 1) % 3, F = (D + 2) % 3;
	int c[3];
	c[D] = side ? A.L.n[D] - 1 : -1;
	c[E] = ce;
	c[F] = cf;
	stride = A.nf[D];
	return A.G[D] + (side ? 8 * stride : 0) + face_at<D>(A.L, c[0], c[1], c[2]);
}

// block (d, side): adds the cotangents of the VALUE ghosts of that side into acc[d][side][8]
__global__ void value_side_kernel(const Adj_Params A, double* acc)
{
	__shared__ double red[8][256];
	const int d = blockIdx.x / 2, side = blockIdx.x % 2;
	const bool on = A.active[d] and not A.periodic[d] and (side ? A.bc_hi[d] : A.bc_lo[d]) == PAMHD_BC_VALUE;
	double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
	if (on) {
		const int e = (d + 1) % 3;
		const long long m = (long long)A.L.n[e] * A.L.n[(d + 2) % 3];
		for (long long t = threadIdx.x; t < m; t += blockDim.x) {
			const int ce = int(t % A.L.n[e]), cf = int(t / A.L.n[e]);
			long long stride = 0;
			const double* g = d == 0 ? value_ghost_cotangent<0>(A, side, ce, cf, stride)
			                : d == 1 ? value_ghost_cotangent<1>(A, side, ce, cf, stride)
			                         : value_ghost_cotangent<2>(A, side, ce, cf, stride);
			for (int v = 0; v < 8; v++) s[v] += g[v * stride];
		}
	}
	for (int v = 0; v < 8; v++) red[v][threadIdx.x] = s[v];
	__syncthreads();
	for (int w = blockDim.x / 2; w > 0; w >>= 1) {
		if ((int)threadIdx.x < w) {
			for (int v = 0; v < 8; v++) red[v][threadIdx.x] += red[v][threadIdx.x + w];
		}
		__syncthreads();
	}
	if (threadIdx.x == 0 and on) {
		for (int v = 0; v < 8; v++) acc[(2 * d + side) * 8 + v] += red[v][0];
	}
}

int check(const cudaError_t e)
{
	return e == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

#define PAMHD_TRY(expr) do { const int rc_ = (expr); if (rc_ != PAMHD_OK) return rc_; } while (0)

int launch_vjp(const Adj_Params& A, const int solver, cudaStream_t stream)
{
	long long count = 0;
	for (int d = 0; d < 3; d++) count += A.active[d] ? A.nf[d] : 0;
	int blocks = int(std::min<long long>(65535, (count + 127) / 128));
	// no more blocks than fit at once: the loop over faces then ends without a partial last wave
	{
		int device = 0, sms = 0, per_sm = 0;
		cudaError_t e = cudaGetDevice(&device);
		if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
		if (e == cudaSuccess) {
			switch (solver) {
			case PAMHD_RUSANOV: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, faces_vjp_kernel<PAMHD_RUSANOV>, 128, 0); break;
			case PAMHD_HLL_ATHENA: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, faces_vjp_kernel<PAMHD_HLL_ATHENA>, 128, 0); break;
			case PAMHD_HLLD_ATHENA: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, faces_vjp_kernel<PAMHD_HLLD_ATHENA>, 128, 0); break;
			default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, faces_vjp_kernel<PAMHD_ROE_ATHENA>, 128, 0); break;
			}
		}
		if (e != cudaSuccess) return PAMHD_ERR_CUDA;
		if (per_sm > 0) blocks = std::max(1, std::min(blocks, per_sm * sms));
	}
	switch (solver) {
	case PAMHD_RUSANOV: faces_vjp_kernel<PAMHD_RUSANOV><<<blocks, 128, 0, stream>>>(A); break;
	case PAMHD_HLL_ATHENA: faces_vjp_kernel<PAMHD_HLL_ATHENA><<<blocks, 128, 0, stream>>>(A); break;
	case PAMHD_HLLD_ATHENA: faces_vjp_kernel<PAMHD_HLLD_ATHENA><<<blocks, 128, 0, stream>>>(A); break;
	case PAMHD_ROE_ATHENA: faces_vjp_kernel<PAMHD_ROE_ATHENA><<<blocks, 128, 0, stream>>>(A); break;
	default: return PAMHD_ERR_ARGUMENT;
	}
	return check(cudaGetLastError());
}

// one forward step of the context with a prescribed dt (the context's own buffers and clock)
int forward_step(pamhd_ctx& x, const double dt)
{
	Step_Params P = x.base;
	P.in = x.state[x.cur];
	P.out = x.state[x.cur ^ 1];
	P.phase = int(x.steps % 3);
	P.forced_dt = dt;
	if (x.needs_boundary_speeds) PAMHD_TRY(launch_boundary_speeds(P, x.cfg.solver, x.stream));
	PAMHD_TRY(launch_step(P, x.cfg.solver, x.stream));
	x.cur ^= 1;
	x.steps++;
	return PAMHD_OK;
}

struct Device_Buffer {
	double* p = nullptr;
	size_t len = 0;
	~Device_Buffer() { cudaFree(p); }
	// grows to at least n doubles (contents not kept)
	int reserve(const size_t n)
	{
		if (n <= len) return PAMHD_OK;
		cudaFree(p);
		p = nullptr;
		len = 0;
		PAMHD_TRY(check(cudaMalloc(&p, n * sizeof(double))));
		len = n;
		return PAMHD_OK;
	}
};

} // namespace

/*
Device memory of the adjoint, kept by the context between calls so that
repeated gradients do not allocate: checkpoints, two buffers of recompute
states, the two cotangent copies, per-axis face cotangents, VALUE-side sums
and the reduction ring of the recompute steps.  Grows when a call needs
more.  The recompute of a segment runs on its own stream, overlapping the
reverse sweep of the segment after it.
*/
struct Adjoint_Work {
	Device_Buffer ck, seg[2], lam[2], G[3], acc, scratch;
	int seg_ready[2] = {0, 0};  // recompute states whose VALUE ghosts are filled
	cudaStream_t side = nullptr;
	cudaEvent_t forward_done = nullptr, recomputed[2] = {nullptr, nullptr}, swept[2] = {nullptr, nullptr};

	int init(const int device)
	{
		if (side != nullptr) return PAMHD_OK;
		PAMHD_TRY(check(cudaSetDevice(device)));
		PAMHD_TRY(check(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking)));
		for (cudaEvent_t* e: {&forward_done, &recomputed[0], &recomputed[1], &swept[0], &swept[1]}) {
			PAMHD_TRY(check(cudaEventCreateWithFlags(e, cudaEventDisableTiming)));
		}
		return PAMHD_OK;
	}
	~Adjoint_Work()
	{
		if (side != nullptr) cudaStreamSynchronize(side);
		for (cudaEvent_t e: {forward_done, recomputed[0], recomputed[1], swept[0], swept[1]}) {
			if (e != nullptr) cudaEventDestroy(e);
		}
		if (side != nullptr) cudaStreamDestroy(side);
	}
};

namespace pamhd_b200 {
void release_adjoint(pamhd_ctx& x)
{
	delete x.adjoint;
	x.adjoint = nullptr;
}
}

namespace {

} // namespace

extern "C" {

int pamhd_gpu_steps_dt(pamhd_ctx* x, const int32_t nsteps, const double* dts)
{
	if (x == nullptr or nsteps < 0 or (nsteps > 0 and dts == nullptr)) return PAMHD_ERR_ARGUMENT;
	if (not x->loaded or x->half) return PAMHD_ERR_STATE;
	for (int n = 0; n < nsteps; n++) {
		if (not (dts[n] >= 0.0)) return PAMHD_ERR_ARGUMENT;
	}
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	for (int n = 0; n < nsteps; n++) PAMHD_TRY(forward_step(*x, dts[n]));
	return PAMHD_OK;
}

int pamhd_gpu_adjoint(pamhd_ctx* x, const int32_t nsteps, const int32_t every, const double* const user_seed[8],
                      double* const user_grad[8], double* grad_value, const double* dt_in, double* dt_out)
{
	if (x == nullptr or nsteps < 1 or every < 1 or user_seed == nullptr or user_grad == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int v = 0; v < 8; v++) if (user_seed[v] == nullptr or user_grad[v] == nullptr) return PAMHD_ERR_ARGUMENT;
	// the caller's arrays in the internal component order (see Axis_Map)
	const double* seed[8];
	double* grad[8];
	for (int v = 0; v < 8; v++) {
		seed[v] = user_seed[x->map.user_var(v)];
		grad[v] = user_grad[x->map.user_var(v)];
	}
	if (x->cfg.bc_lo[2] == PAMHD_BC_EXTERNAL or x->cfg.bc_hi[2] == PAMHD_BC_EXTERNAL) return PAMHD_ERR_ARGUMENT;
	// the inflow-state gradient is of one constant state per side
	if (x->base.inflow != nullptr) return PAMHD_ERR_ARGUMENT;
	if (not x->loaded or x->half) return PAMHD_ERR_STATE;
	if (dt_in != nullptr) {
		for (int n = 0; n < nsteps; n++) if (not (dt_in[n] >= 0.0)) return PAMHD_ERR_ARGUMENT;
	}
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	const Layout& L = x->L;
	const size_t state_len = size_t(8) * L.var;
	const int nck = (nsteps + every - 1) / every;
	const int seg_len = std::min(every, nsteps);
	if (nsteps > x->hist_len) return PAMHD_ERR_ARGUMENT;
	if (x->adjoint == nullptr) {
		x->adjoint = new (std::nothrow) Adjoint_Work;
		if (x->adjoint == nullptr) return PAMHD_ERR_ARGUMENT;
	}
	Adjoint_Work& W = *x->adjoint;
	PAMHD_TRY(W.init(x->device));
	const size_t scratch_bytes = 3 * sizeof(Speed_Max) + 3 * sizeof(Clock) + sizeof(Status);
	PAMHD_TRY(W.ck.reserve(state_len * size_t(nck)));
	for (int b = 0; b < 2; b++) {
		if (seg_len > 1 and W.seg[b].len < state_len * size_t(seg_len - 1)) {
			PAMHD_TRY(W.seg[b].reserve(state_len * size_t(seg_len - 1)));
			W.seg_ready[b] = 0;
		}
	}
	PAMHD_TRY(W.lam[0].reserve(state_len));
	PAMHD_TRY(W.lam[1].reserve(state_len));
	PAMHD_TRY(W.acc.reserve(48));
	PAMHD_TRY(W.scratch.reserve((scratch_bytes + 7) / 8));
	Adj_Params A;
	A.L = L;
	A.gas.gamma = x->base.gas.gamma;
	A.gas.inv_mu0 = x->base.gas.inv_mu0;
	A.gas.sqrt_mu0 = x->base.gas.sqrt_mu0;
	A.gas.inv_sqrt_mu0 = x->base.gas.inv_sqrt_mu0;
	bool any_value = false;
	for (int d = 0; d < 3; d++) {
		A.inv_len[d] = x->base.inv_len[d];
		A.active[d] = x->base.active[d];
		A.periodic[d] = x->base.periodic[d];
		A.bc_lo[d] = x->base.bc_lo[d];
		A.bc_hi[d] = x->base.bc_hi[d];
		A.G[d] = nullptr;
		A.nf[d] = 0;
		if (A.active[d]) {
			A.nf[d] = faces_of(L, d);
			PAMHD_TRY(W.G[d].reserve(16 * size_t(A.nf[d])));
			A.G[d] = W.G[d].p;
			if (not A.periodic[d] and (A.bc_lo[d] == PAMHD_BC_VALUE or A.bc_hi[d] == PAMHD_BC_VALUE)) any_value = true;
		}
	}

	// ---- forward run with checkpoints
	{
		Control c;
		c.max_dt = -1.0;
		c.t_end = 1.0e300;
		PAMHD_TRY(check(cudaMemcpyAsync(x->control, &c, sizeof c, cudaMemcpyHostToDevice, x->stream)));
		x->control_max_dt = c.max_dt;
		x->control_t_end = c.t_end;
	}
	// VALUE ghosts are constant and the step kernel never writes them: fill each recompute state once
	for (int b = 0; b < 2; b++) {
		for (int i = W.seg_ready[b]; i < seg_len - 1; i++) {
			PAMHD_TRY(launch_fill_ghosts_values(x->base, W.seg[b].p + state_len * size_t(i), x->cfg.value_lo,
			                                    x->cfg.value_hi, x->stream));
		}
		W.seg_ready[b] = std::max(W.seg_ready[b], seg_len - 1);
	}
	std::vector<double> dts(nsteps);
	const int last = nck - 1;
	// the segments from kept on fill the two segment buffers as they are made instead of being
	// recomputed: the last two (the buffers hold two segments)
	const int kept = std::max(0, last - 1);
	for (int n = 0; n < nsteps; n++) {
		if (n % every == 0) {
			PAMHD_TRY(check(cudaMemcpyAsync(W.ck.p + state_len * size_t(n / every), x->state[x->cur],
			                                state_len * sizeof(double), cudaMemcpyDeviceToDevice, x->stream)));
		}
		PAMHD_TRY(forward_step(*x, dt_in != nullptr ? dt_in[n] : -1.0));
		// state n + 1, inside segment n / every (not the next checkpoint)
		const int sn = n / every;
		if (sn >= kept and n + 1 < std::min(nsteps, (sn + 1) * every)) {
			PAMHD_TRY(check(cudaMemcpyAsync(W.seg[sn & 1].p + state_len * size_t(n - sn * every), x->state[x->cur],
			                                state_len * sizeof(double), cudaMemcpyDeviceToDevice, x->stream)));
		}
	}
	PAMHD_TRY(check(cudaEventRecord(W.forward_done, x->stream)));
	{
		std::vector<double> hist(x->hist_len);
		PAMHD_TRY(check(cudaMemcpyAsync(hist.data(), x->dt_hist, x->hist_len * sizeof(double),
		                                cudaMemcpyDeviceToHost, x->stream)));
		Status s;
		PAMHD_TRY(check(cudaMemcpyAsync(&s, x->status, sizeof s, cudaMemcpyDeviceToHost, x->stream)));
		PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
		if (s.flags != 0) return PAMHD_ERR_PHYSICS;
		for (int n = 0; n < nsteps; n++) dts[n] = hist[(x->steps - nsteps + n) % x->hist_len];
	}
	if (dt_out != nullptr) std::copy(dts.begin(), dts.end(), dt_out);

	// ---- reverse sweep
	PAMHD_TRY(check(cudaMemsetAsync(W.acc.p, 0, 48 * sizeof(double), x->stream)));
	PAMHD_TRY(check(cudaMemsetAsync(W.lam[0].p, 0, state_len * sizeof(double), x->stream)));
	PAMHD_TRY(check(cudaMemsetAsync(W.lam[1].p, 0, state_len * sizeof(double), x->stream)));
	const size_t cells = size_t(L.n[0]) * L.n[1] * L.n[2];
	for (int v = 0; v < 8; v++) {
		PAMHD_TRY(check(cudaMemcpyAsync(x->staging, seed[v], cells * sizeof(double), cudaMemcpyHostToDevice,
		                                x->stream)));
		PAMHD_TRY(launch_scatter(x->staging, W.lam[0].p + v * L.var, L, x->stream));
	}
	PAMHD_TRY(check(cudaStreamWaitEvent(W.side, W.forward_done, 0)));
	PAMHD_TRY(check(cudaMemsetAsync(W.scratch.p, 0, scratch_bytes, W.side)));
	Step_Params R = x->base;
	R.red = reinterpret_cast<Speed_Max*>(W.scratch.p);
	R.clock = reinterpret_cast<Clock*>(reinterpret_cast<char*>(W.scratch.p) + 3 * sizeof(Speed_Max));
	R.status = reinterpret_cast<Status*>(reinterpret_cast<char*>(W.scratch.p) + 3 * sizeof(Speed_Max)
	                                     + 3 * sizeof(Clock));
	R.dt_hist = nullptr;
	R.phase = 0;
	// state i of segment s: its checkpoint (i = 0) or entry i - 1 of segment buffer s & 1
	auto state_of = [&](const int s, const int i) -> const double* {
		return i == 0 ? W.ck.p + state_len * size_t(s) : W.seg[s & 1].p + state_len * size_t(i - 1);
	};
	// segment s recomputed on the side stream, once the sweep two segments later freed its buffer
	auto recompute = [&](const int s) -> int {
		const int start = s * every, end = std::min(nsteps, start + every);
		PAMHD_TRY(check(cudaStreamWaitEvent(W.side, W.swept[s & 1], 0)));
		for (int i = 1; i < end - start; i++) {
			R.in = state_of(s, i - 1);
			R.out = const_cast<double*>(state_of(s, i));
			R.forced_dt = dts[start + i - 1];
			PAMHD_TRY(launch_step(R, x->cfg.solver, W.side));
		}
		return check(cudaEventRecord(W.recomputed[s & 1], W.side));
	};
	int li = 0;
	for (int s = nck - 1; s >= 0; s--) {
		const int start = s * every, end = std::min(nsteps, start + every);
		if (s >= 1 and s - 1 < kept) PAMHD_TRY(recompute(s - 1));
		if (s < kept) PAMHD_TRY(check(cudaStreamWaitEvent(x->stream, W.recomputed[s & 1], 0)));
		std::vector<const double*> states(end - start);
		for (int i = 0; i < end - start; i++) states[i] = state_of(s, i);
		for (int n = end - 1; n >= start; n--) {
			A.U = states[n - start];
			A.dt = dts[n];
			A.lam = W.lam[li].p;
			A.lam_out = W.lam[li ^ 1].p;
			PAMHD_TRY(launch_vjp(A, x->cfg.solver, x->stream));
			gather_kernel<<<int(std::min<size_t>(65535, (cells + 255) / 256)), 256, 0, x->stream>>>(A);
			if (any_value) value_side_kernel<<<6, 256, 0, x->stream>>>(A, W.acc.p);
			PAMHD_TRY(check(cudaGetLastError()));
			li ^= 1;
		}
		PAMHD_TRY(check(cudaEventRecord(W.swept[s & 1], x->stream)));
	}
	for (int v = 0; v < 8; v++) {
		PAMHD_TRY(launch_gather(W.lam[li].p + v * L.var, x->staging, L, x->stream));
		PAMHD_TRY(check(cudaMemcpyAsync(grad[v], x->staging, cells * sizeof(double), cudaMemcpyDeviceToHost,
		                                x->stream)));
	}
	double internal_value[48];
	if (grad_value != nullptr) {
		PAMHD_TRY(check(cudaMemcpyAsync(internal_value, W.acc.p, 48 * sizeof(double), cudaMemcpyDeviceToHost,
		                                x->stream)));
	}
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	if (grad_value != nullptr) {
		// [dimension][side][variable] in the caller's axes and component order
		for (int d = 0; d < 3; d++) {
			for (int side = 0; side < 2; side++) {
				for (int v = 0; v < 8; v++) {
					grad_value[(2 * x->map.perm[d] + side) * 8 + x->map.user_var(v)] = internal_value[(2 * d + side) * 8 + v];
				}
			}
		}
	}
	return PAMHD_OK;
}

} // extern "C"
