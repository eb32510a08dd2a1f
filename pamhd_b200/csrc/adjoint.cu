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

Kernels: face_vjp_kernel (one thread per face of one axis, writes g_L and
g_R of every face), gather_kernel (one thread per cell, sums its faces in
a fixed order: deterministic), value_side_kernel (sums the ghost gradients
of VALUE sides, one block per side, fixed order).

Driver (pamhd_gpu_adjoint): the forward run stores the state every K
steps; the reverse sweep recomputes each segment of K states from its
checkpoint (same kernels, so the same bits) and steps lambda back through
it.  Memory: ceil(N/K) + K - 1 state copies.
*/
#include <cuda_runtime.h>

#include <algorithm>
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
	double* G[3];         // per axis: 16 values per face (g_L, g_R)
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

// face of axis d whose lower cell has coordinate l along d
__device__ inline long long face_index(const Layout& L, const int d, const int l, const int ce, const int cf)
{
	const int e = (d + 1) % 3;
	return (long long)(l + 1) + (long long)(L.n[d] + 1) * (ce + (long long)L.n[e] * cf);
}

template <int SOLVER>
__global__ void face_vjp_kernel(const Adj_Params A, const int d)
{
	const int e = (d + 1) % 3, f = (d + 2) % 3;
	const long long count = faces_of(A.L, d);
	for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < count;
	     t += (long long)gridDim.x * blockDim.x) {
		const int l = int(t % (A.L.n[d] + 1)) - 1;
		const long long rest = t / (A.L.n[d] + 1);
		int c[3];
		c[d] = l;
		c[e] = int(rest % A.L.n[e]);
		c[f] = int(rest / A.L.n[e]);
		const long long oL = A.L.offset(c[0], c[1], c[2]);
		c[d] = l + 1;
		const long long oR = A.L.offset(c[0], c[1], c[2]);
		const int a0 = d, a1 = e, a2 = f;
		double UL[8], UR[8], phi[8];
		const double scale = A.dt * A.inv_len[d];
		const int perm[8] = {0, 1 + a0, 1 + a1, 1 + a2, 4, 5 + a0, 5 + a1, 5 + a2};
		const bool in_l = l >= 0, in_r = l + 1 <= A.L.n[d] - 1;
		#pragma unroll
		for (int v = 0; v < 8; v++) {
			const long long vo = perm[v] * A.L.var;
			UL[v] = A.U[vo + oL];
			UR[v] = A.U[vo + oR];
			const double lr = in_r ? A.lam[vo + oR] : 0.0;
			const double ll = in_l ? A.lam[vo + oL] : 0.0;
			phi[v] = scale * (lr - ll);
		}
		double gL[8], gR[8];
		pamhd_b200::adjoint::face_vjp<SOLVER>(UL, UR, A.gas, phi, gL, gR);
		double* out = A.G[d] + 16 * t;
		#pragma unroll
		for (int v = 0; v < 8; v++) {
			out[perm[v]] = gL[v];
			out[8 + perm[v]] = gR[v];
		}
	}
}

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
		for (int d = 0; d < 3; d++) {
			if (not A.active[d]) continue;
			const int e = (d + 1) % 3, f = (d + 2) % 3;
			const int nd = A.L.n[d];
			const double* G = A.G[d];
			// the cell is the right side of its -d face and the left side of its +d face
			const double* minus = G + 16 * face_index(A.L, d, c[d] - 1, c[e], c[f]);
			const double* plus = G + 16 * face_index(A.L, d, c[d], c[e], c[f]);
			#pragma unroll
			for (int v = 0; v < 8; v++) acc[v] += minus[8 + v] + plus[v];
			// ghosts made from this cell
			const bool first = c[d] == 0, last = c[d] == nd - 1;
			if (A.periodic[d]) {
				if (last) {   // ghost -1 is this cell
					const double* g = G + 16 * face_index(A.L, d, -1, c[e], c[f]);
					for (int v = 0; v < 8; v++) acc[v] += g[v];
				}
				if (first) {  // ghost n is this cell
					const double* g = G + 16 * face_index(A.L, d, nd - 1, c[e], c[f]);
					for (int v = 0; v < 8; v++) acc[v] += g[8 + v];
				}
			} else {
				// a COPY ghost equals its source cell in exact arithmetic: identity Jacobian
				if (first and A.bc_lo[d] == PAMHD_BC_COPY) {
					const double* g = G + 16 * face_index(A.L, d, -1, c[e], c[f]);
					for (int v = 0; v < 8; v++) acc[v] += g[v];
				}
				if (last and A.bc_hi[d] == PAMHD_BC_COPY) {
					const double* g = G + 16 * face_index(A.L, d, nd - 1, c[e], c[f]);
					for (int v = 0; v < 8; v++) acc[v] += g[8 + v];
				}
			}
		}
		#pragma unroll
		for (int v = 0; v < 8; v++) A.lam_out[v * A.L.var + o] = acc[v];
	}
}

// block (d, side): adds the gradients of the VALUE ghosts of that side into acc[d][side][8]
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
			const double* g = A.G[d] + 16 * face_index(A.L, d, side ? A.L.n[d] - 1 : -1, ce, cf) + (side ? 8 : 0);
			for (int v = 0; v < 8; v++) s[v] += g[v];
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
	for (int d = 0; d < 3; d++) {
		if (not A.active[d]) continue;
		const long long count = faces_of(A.L, d);
		const int blocks = int(std::min<long long>(4096, (count + 127) / 128));
		switch (solver) {
		case PAMHD_RUSANOV: face_vjp_kernel<PAMHD_RUSANOV><<<blocks, 128, 0, stream>>>(A, d); break;
		case PAMHD_HLL_ATHENA: face_vjp_kernel<PAMHD_HLL_ATHENA><<<blocks, 128, 0, stream>>>(A, d); break;
		case PAMHD_HLLD_ATHENA: face_vjp_kernel<PAMHD_HLLD_ATHENA><<<blocks, 128, 0, stream>>>(A, d); break;
		default: return PAMHD_ERR_ARGUMENT;
		}
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
	~Device_Buffer() { cudaFree(p); }
	int alloc(const size_t n) { return check(cudaMalloc(&p, n * sizeof(double))); }
};

} // namespace

extern "C" {

int pamhd_gpu_steps_dt(pamhd_ctx* x, const int32_t nsteps, const double* dts)
{
	if (x == nullptr or nsteps < 0 or (nsteps > 0 and dts == nullptr)) return PAMHD_ERR_ARGUMENT;
	if (not x->loaded) return PAMHD_ERR_STATE;
	for (int n = 0; n < nsteps; n++) {
		if (not (dts[n] >= 0.0)) return PAMHD_ERR_ARGUMENT;
	}
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	for (int n = 0; n < nsteps; n++) PAMHD_TRY(forward_step(*x, dts[n]));
	return PAMHD_OK;
}

int pamhd_gpu_adjoint(pamhd_ctx* x, const int32_t nsteps, const int32_t every, const double* const seed[8],
                      double* const grad[8], double* grad_value, const double* dt_in, double* dt_out)
{
	if (x == nullptr or nsteps < 1 or every < 1 or seed == nullptr or grad == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int v = 0; v < 8; v++) if (seed[v] == nullptr or grad[v] == nullptr) return PAMHD_ERR_ARGUMENT;
	if (x->cfg.solver == PAMHD_ROE_ATHENA) return PAMHD_ERR_ARGUMENT;  // no Roe adjoint
	if (not x->loaded) return PAMHD_ERR_STATE;
	if (dt_in != nullptr) {
		for (int n = 0; n < nsteps; n++) if (not (dt_in[n] >= 0.0)) return PAMHD_ERR_ARGUMENT;
	}
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	const Layout& L = x->L;
	const size_t state_len = size_t(8) * L.var;
	const int nck = (nsteps + every - 1) / every;

	// ---- forward run with checkpoints
	std::vector<Device_Buffer> ck(nck);
	for (auto& b: ck) PAMHD_TRY(b.alloc(state_len));
	{
		Control c;
		c.max_dt = -1.0;
		c.t_end = 1.0e300;
		PAMHD_TRY(check(cudaMemcpyAsync(x->control, &c, sizeof c, cudaMemcpyHostToDevice, x->stream)));
		PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	}
	std::vector<double> dts(nsteps);
	for (int n = 0; n < nsteps; n++) {
		if (n % every == 0) {
			PAMHD_TRY(check(cudaMemcpyAsync(ck[n / every].p, x->state[x->cur], state_len * sizeof(double),
			                                cudaMemcpyDeviceToDevice, x->stream)));
		}
		PAMHD_TRY(forward_step(*x, dt_in != nullptr ? dt_in[n] : -1.0));
	}
	{
		std::vector<double> hist(x->hist_len);
		PAMHD_TRY(check(cudaMemcpyAsync(hist.data(), x->dt_hist, x->hist_len * sizeof(double),
		                                cudaMemcpyDeviceToHost, x->stream)));
		Status s;
		PAMHD_TRY(check(cudaMemcpyAsync(&s, x->status, sizeof s, cudaMemcpyDeviceToHost, x->stream)));
		PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
		if (s.flags != 0) return PAMHD_ERR_PHYSICS;
		if (nsteps > x->hist_len) return PAMHD_ERR_ARGUMENT;
		for (int n = 0; n < nsteps; n++) dts[n] = hist[(x->steps - nsteps + n) % x->hist_len];
	}
	if (dt_out != nullptr) std::copy(dts.begin(), dts.end(), dt_out);

	// ---- reverse sweep
	Device_Buffer lam[2], G[3], seg_store, acc, scratch;
	PAMHD_TRY(lam[0].alloc(state_len));
	PAMHD_TRY(lam[1].alloc(state_len));
	Adj_Params A;
	A.L = L;
	A.gas.gamma = x->base.gas.gamma;
	A.gas.inv_mu0 = x->base.gas.inv_mu0;
	A.gas.sqrt_mu0 = x->base.gas.sqrt_mu0;
	A.gas.inv_sqrt_mu0 = x->base.gas.inv_sqrt_mu0;
	for (int d = 0; d < 3; d++) {
		A.inv_len[d] = x->base.inv_len[d];
		A.active[d] = x->base.active[d];
		A.periodic[d] = x->base.periodic[d];
		A.bc_lo[d] = x->base.bc_lo[d];
		A.bc_hi[d] = x->base.bc_hi[d];
		A.G[d] = nullptr;
		if (A.active[d]) {
			PAMHD_TRY(G[d].alloc(16 * size_t(faces_of(L, d))));
			A.G[d] = G[d].p;
		}
	}
	PAMHD_TRY(acc.alloc(6 * 8));
	PAMHD_TRY(check(cudaMemsetAsync(acc.p, 0, 48 * sizeof(double), x->stream)));
	PAMHD_TRY(check(cudaMemsetAsync(lam[0].p, 0, state_len * sizeof(double), x->stream)));
	PAMHD_TRY(check(cudaMemsetAsync(lam[1].p, 0, state_len * sizeof(double), x->stream)));
	const size_t cells = size_t(L.n[0]) * L.n[1] * L.n[2];
	for (int v = 0; v < 8; v++) {
		PAMHD_TRY(check(cudaMemcpyAsync(x->staging, seed[v], cells * sizeof(double), cudaMemcpyHostToDevice,
		                                x->stream)));
		PAMHD_TRY(launch_scatter(x->staging, lam[0].p + v * L.var, L, x->stream));
	}
	// recompute buffers: K - 1 states after each checkpoint, and a scratch ring for the recompute steps
	const int seg_len = std::min(every, nsteps);
	if (seg_len > 1) {
		PAMHD_TRY(seg_store.alloc(state_len * size_t(seg_len - 1)));
		// VALUE ghosts are constant: the step kernel never writes them
		for (int i = 0; i < seg_len - 1; i++) {
			PAMHD_TRY(launch_fill_ghosts_values(x->base, seg_store.p + state_len * size_t(i), x->cfg.value_lo,
			                                    x->cfg.value_hi, x->stream));
		}
	}
	const size_t scratch_bytes = 3 * sizeof(Speed_Max) + 3 * sizeof(Clock) + sizeof(Status);
	PAMHD_TRY(scratch.alloc((scratch_bytes + 7) / 8));
	PAMHD_TRY(check(cudaMemsetAsync(scratch.p, 0, scratch_bytes, x->stream)));
	Step_Params R = x->base;
	R.red = reinterpret_cast<Speed_Max*>(scratch.p);
	R.clock = reinterpret_cast<Clock*>(reinterpret_cast<char*>(scratch.p) + 3 * sizeof(Speed_Max));
	R.status = reinterpret_cast<Status*>(reinterpret_cast<char*>(scratch.p) + 3 * sizeof(Speed_Max) + 3 * sizeof(Clock));
	R.dt_hist = nullptr;
	R.phase = 0;
	int li = 0;
	for (int s = nck - 1; s >= 0; s--) {
		const int start = s * every, end = std::min(nsteps, start + every);
		std::vector<const double*> states(end - start);
		states[0] = ck[s].p;
		for (int i = 1; i < end - start; i++) {
			double* dst = seg_store.p + state_len * size_t(i - 1);
			R.in = states[i - 1];
			R.out = dst;
			R.forced_dt = dts[start + i - 1];
			PAMHD_TRY(launch_step(R, x->cfg.solver, x->stream));
			states[i] = dst;
		}
		for (int n = end - 1; n >= start; n--) {
			A.U = states[n - start];
			A.dt = dts[n];
			A.lam = lam[li].p;
			A.lam_out = lam[li ^ 1].p;
			PAMHD_TRY(launch_vjp(A, x->cfg.solver, x->stream));
			gather_kernel<<<int(std::min<size_t>(4096, (cells + 255) / 256)), 256, 0, x->stream>>>(A);
			value_side_kernel<<<6, 256, 0, x->stream>>>(A, acc.p);
			PAMHD_TRY(check(cudaGetLastError()));
			li ^= 1;
		}
	}
	for (int v = 0; v < 8; v++) {
		PAMHD_TRY(launch_gather(lam[li].p + v * L.var, x->staging, L, x->stream));
		PAMHD_TRY(check(cudaMemcpyAsync(grad[v], x->staging, cells * sizeof(double), cudaMemcpyDeviceToHost,
		                                x->stream)));
	}
	if (grad_value != nullptr) {
		PAMHD_TRY(check(cudaMemcpyAsync(grad_value, acc.p, 48 * sizeof(double), cudaMemcpyDeviceToHost,
		                                x->stream)));
	}
	return check(cudaStreamSynchronize(x->stream));
}

} // extern "C"
