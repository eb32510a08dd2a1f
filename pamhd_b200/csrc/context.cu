/*
Host side of the C ABI in include/pamhd_gpu.h: the context (device
buffers, stream, CUDA graph) and every exported entry point.

A context owns two copies of the state (ping-pong: a step reads one and
writes the other), a three-slot ring of speed reductions and clocks, the
error status and a dt history, all on one device and one stream.  Steps
are issued without host synchronisation; because the kernel parameters of
a step depend only on the step index modulo 6 (state parity x ring phase),
six consecutive steps are captured once into a CUDA graph and replayed.
*/
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "context.cuh"

using namespace pamhd_b200;

namespace {

constexpr int GRAPH_STEPS = 6;

int check(const cudaError_t e)
{
	return e == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

#define PAMHD_TRY(expr) do { const int rc_ = (expr); if (rc_ != PAMHD_OK) return rc_; } while (0)

void set_params(pamhd_ctx& x)
{
	x.needs_boundary_speeds = grid_params(x.cfg, x.L, x.base);
	Step_Params& P = x.base;
	P.red = x.red;
	P.clock = x.clock;
	P.status = x.status;
	P.control = x.control;
	P.dt_hist = x.dt_hist;
	P.hist_len = x.hist_len;
}

Step_Params params_for(const pamhd_ctx& x, const long long step, const int cur)
{
	Step_Params P = x.base;
	P.in = x.state[cur];
	P.out = x.state[cur ^ 1];
	P.phase = int(step % 3);
	return P;
}

int issue_step(pamhd_ctx& x)
{
	const Step_Params P = params_for(x, x.steps, x.cur);
	if (x.needs_boundary_speeds) PAMHD_TRY(launch_boundary_speeds(P, x.cfg.solver, x.stream));
	PAMHD_TRY(launch_step(P, x.cfg.solver, x.stream));
	x.cur ^= 1;
	x.steps++;
	return PAMHD_OK;
}

// one part of a step: 1 the first and last z planes (and the boundary speeds), 2 the rest and the
// step's end; the two launches read the same state and fold into the same reduction slot
int issue_step_part(pamhd_ctx& x, const int part)
{
	Step_Params P = params_for(x, x.steps, x.cur);
	P.kpart = part;
	if (part == 1 and x.needs_boundary_speeds) PAMHD_TRY(launch_boundary_speeds(P, x.cfg.solver, x.stream));
	PAMHD_TRY(launch_step(P, x.cfg.solver, x.stream));
	if (part == 2) {
		x.cur ^= 1;
		x.steps++;
	}
	return PAMHD_OK;
}

} // namespace

int pamhd_b200::context_issue_step(pamhd_ctx& x)
{
	return issue_step(x);
}

namespace {

int reset_run_state(pamhd_ctx& x)
{
	PAMHD_TRY(check(cudaMemsetAsync(x.red, 0, 3 * sizeof(Speed_Max), x.stream)));
	PAMHD_TRY(check(cudaMemsetAsync(x.clock, 0, 3 * sizeof(Clock), x.stream)));
	Status s;
	s.flags = 0;
	s.fail_step = 0;
	s.first = ~0ull;
	PAMHD_TRY(check(cudaMemcpyAsync(x.status, &s, sizeof s, cudaMemcpyHostToDevice, x.stream)));
	x.steps = 0;
	x.cur = 0;
	x.half = 0;
	return PAMHD_OK;
}

int read_status(pamhd_ctx& x, Status& s)
{
	PAMHD_TRY(check(cudaMemcpyAsync(&s, x.status, sizeof s, cudaMemcpyDeviceToHost, x.stream)));
	return check(cudaStreamSynchronize(x.stream));
}

int set_control(pamhd_ctx& x, const double max_dt, const double t_end)
{
	x.control_max_dt = max_dt;
	x.control_t_end = t_end;
	Control c;
	c.max_dt = max_dt;
	c.t_end = t_end;
	PAMHD_TRY(check(cudaMemcpyAsync(x.control, &c, sizeof c, cudaMemcpyHostToDevice, x.stream)));
	// the copy reads from this stack variable: wait for it
	return check(cudaStreamSynchronize(x.stream));
}

// ghost states of the VALUE sides at time t: the configured values, or the time-stamped inflow
void values_at(const pamhd_ctx& x, const double t, double lo[3][8], double hi[3][8])
{
	for (int d = 0; d < 3; d++) {
		for (int side = 0; side < 2; side++) {
			double* out = side == 0 ? lo[d] : hi[d];
			const double* v = side == 0 ? x.cfg.value_lo[d] : x.cfg.value_hi[d];
			const std::vector<double>& times = x.inflow_times[d][side];
			const std::vector<double>& states = x.inflow_states[d][side];
			if (not states.empty()) {
				size_t i = 0;
				while (i < times.size() and t >= times[i]) i++;
				v = states.data() + 8 * i;
			}
			for (int k = 0; k < 8; k++) out[k] = v[k];
		}
	}
}

// ghosts of both state copies after set_state (simulation time 0)
int fill_ghosts(pamhd_ctx& x)
{
	const Step_Params P = x.base;
	double lo[3][8], hi[3][8];
	values_at(x, 0.0, lo, hi);
	PAMHD_TRY(launch_fill_ghosts_values(P, x.state[0], lo, hi, x.stream));
	return launch_fill_ghosts_values(P, x.state[1], lo, hi, x.stream);
}

int capture_graph(pamhd_ctx& x)
{
	if (x.graph != nullptr) return PAMHD_OK;
	cudaGraph_t g = nullptr;
	PAMHD_TRY(check(cudaStreamBeginCapture(x.stream, cudaStreamCaptureModeThreadLocal)));
	const long long steps0 = x.steps;
	const int cur0 = x.cur;
	int rc = PAMHD_OK;
	for (int s = 0; s < GRAPH_STEPS and rc == PAMHD_OK; s++) rc = issue_step(x);
	x.steps = steps0;
	x.cur = cur0;
	const cudaError_t e = cudaStreamEndCapture(x.stream, &g);
	if (rc != PAMHD_OK or e != cudaSuccess) {
		if (g != nullptr) cudaGraphDestroy(g);
		return rc != PAMHD_OK ? rc : PAMHD_ERR_CUDA;
	}
	const cudaError_t ie = cudaGraphInstantiate(&x.graph, g, 0);
	cudaGraphDestroy(g);
	return check(ie);
}

} // namespace

extern "C" {

int pamhd_gpu_abi_version(void)
{
	return PAMHD_GPU_ABI_VERSION;
}

const char* pamhd_gpu_errstr(const int code)
{
	switch (code) {
	case PAMHD_OK: return "ok";
	case PAMHD_ERR_ARGUMENT: return "invalid argument or configuration";
	case PAMHD_ERR_CUDA: return "CUDA runtime error";
	case PAMHD_ERR_PHYSICS: return "a face met an invalid state (see pamhd_gpu_status)";
	case PAMHD_ERR_STATE: return "call made in the wrong order";
	case PAMHD_ERR_TIMEOUT: return "a bounded device wait expired";
	case PAMHD_ERR_TOO_LARGE: return "request larger than the fixed scratch of a no-alloc entry point; split it";
	case PAMHD_ERR_IO: return "a file could not be opened, read or written";
	default: return "unknown error";
	}
}

int pamhd_gpu_create(const pamhd_cfg* cfg, pamhd_ctx** out)
{
	if (cfg == nullptr or out == nullptr) return PAMHD_ERR_ARGUMENT;
	*out = nullptr;
	const Axis_Map map = axis_map(*cfg);
	if (not map.identity()) {
		// slab cuts are z sides of grids with the usual axes
		for (int d = 0; d < 3; d++) {
			if (cfg->bc_lo[d] == PAMHD_BC_EXTERNAL or cfg->bc_hi[d] == PAMHD_BC_EXTERNAL) return PAMHD_ERR_ARGUMENT;
		}
	}
	const pamhd_cfg internal = relabelled(*cfg, map);
	PAMHD_TRY(validate(internal));
	// the step's launch: rows of tiles along y and z chunks within a grid dimension's 65535 blocks
	if (internal.n[1] > 1) {
		const int rows = step_tile_rows(internal.solver);
		if ((internal.n[1] + rows - 1) / rows > 65535) return PAMHD_ERR_ARGUMENT;
	}
	if (internal.n[2] > 16 * 65535) return PAMHD_ERR_ARGUMENT;
	pamhd_ctx* x = new (std::nothrow) pamhd_ctx;
	if (x == nullptr) return PAMHD_ERR_ARGUMENT;
	x->cfg = internal;
	x->map = map;
	x->device = cfg->device;
	x->L = make_layout(internal);
	auto fail = [&](const int rc) {
		pamhd_gpu_destroy(x);
		return rc;
	};
	if (cudaSetDevice(x->device) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	if (cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	const size_t state_bytes = size_t(8) * x->L.var * sizeof(double);
	const size_t cells = size_t(x->L.n[0]) * x->L.n[1] * x->L.n[2];
	if (cudaMalloc(&x->state[0], state_bytes) != cudaSuccess
		or cudaMalloc(&x->state[1], state_bytes) != cudaSuccess
		or cudaMalloc(&x->red, 3 * sizeof(Speed_Max)) != cudaSuccess
		or cudaMalloc(&x->clock, 3 * sizeof(Clock)) != cudaSuccess
		or cudaMalloc(&x->status, sizeof(Status)) != cudaSuccess
		or cudaMalloc(&x->control, sizeof(Control)) != cudaSuccess
		or cudaMalloc(&x->dt_hist, x->hist_len * sizeof(double)) != cudaSuccess
		or cudaMalloc(&x->staging, cells * sizeof(double)) != cudaSuccess
		or cudaMalloc(&x->partial, 8 * x->partial_blocks * sizeof(double)) != cudaSuccess) {
		return fail(PAMHD_ERR_CUDA);
	}
	if (cudaMemsetAsync(x->state[0], 0, state_bytes, x->stream) != cudaSuccess
		or cudaMemsetAsync(x->state[1], 0, state_bytes, x->stream) != cudaSuccess
		or cudaMemsetAsync(x->dt_hist, 0, x->hist_len * sizeof(double), x->stream) != cudaSuccess) {
		return fail(PAMHD_ERR_CUDA);
	}
	set_params(*x);
	// kernel attributes are set here, outside any stream capture
	if (prepare_step_kernels(cfg->solver, cfg->n[1] > 1) != PAMHD_OK) return fail(PAMHD_ERR_CUDA);
	if (reset_run_state(*x) != PAMHD_OK) return fail(PAMHD_ERR_CUDA);
	if (cudaStreamSynchronize(x->stream) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	*out = x;
	return PAMHD_OK;
}

int pamhd_gpu_destroy(pamhd_ctx* x)
{
	if (x == nullptr) return PAMHD_OK;
	cudaSetDevice(x->device);
	if (x->stream != nullptr) cudaStreamSynchronize(x->stream);
	if (x->graph != nullptr) cudaGraphExecDestroy(x->graph);
	release_adjoint(*x);
	for (int d = 0; d < 3; d++) {
		cudaFree(x->inflow_dev[d][0]);
		cudaFree(x->inflow_dev[d][1]);
	}
	cudaFree(x->inflow_tables);
	cudaFree(x->state[0]);
	cudaFree(x->state[1]);
	cudaFree(x->red);
	cudaFree(x->clock);
	cudaFree(x->status);
	cudaFree(x->control);
	cudaFree(x->dt_hist);
	cudaFree(x->staging);
	cudaFree(x->partial);
	if (x->stream != nullptr) cudaStreamDestroy(x->stream);
	delete x;
	return PAMHD_OK;
}

static int set_state_impl(pamhd_ctx* x, const double* const user[8], const cudaMemcpyKind kind)
{
	if (x == nullptr or user == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int v = 0; v < 8; v++) if (user[v] == nullptr) return PAMHD_ERR_ARGUMENT;
	const double* soa[8];
	for (int v = 0; v < 8; v++) soa[v] = user[x->map.user_var(v)];
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	const size_t bytes = size_t(x->L.n[0]) * x->L.n[1] * x->L.n[2] * sizeof(double);
	for (int v = 0; v < 8; v++) {
		PAMHD_TRY(check(cudaMemcpyAsync(x->staging, soa[v], bytes, kind, x->stream)));
		PAMHD_TRY(launch_scatter(x->staging, x->state[0] + v * x->L.var, x->L, x->stream));
	}
	PAMHD_TRY(fill_ghosts(*x));
	PAMHD_TRY(reset_run_state(*x));
	x->loaded = true;
	return check(cudaStreamSynchronize(x->stream));
}

static int get_state_impl(pamhd_ctx* x, double* const user[8], const cudaMemcpyKind kind)
{
	if (x == nullptr or user == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int v = 0; v < 8; v++) if (user[v] == nullptr) return PAMHD_ERR_ARGUMENT;
	double* soa[8];
	for (int v = 0; v < 8; v++) soa[v] = user[x->map.user_var(v)];
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	const size_t bytes = size_t(x->L.n[0]) * x->L.n[1] * x->L.n[2] * sizeof(double);
	for (int v = 0; v < 8; v++) {
		PAMHD_TRY(launch_gather(x->state[x->cur] + v * x->L.var, x->staging, x->L, x->stream));
		PAMHD_TRY(check(cudaMemcpyAsync(soa[v], x->staging, bytes, kind, x->stream)));
	}
	return check(cudaStreamSynchronize(x->stream));
}

int pamhd_gpu_set_state(pamhd_ctx* x, const double* const soa[8])
{
	return set_state_impl(x, soa, cudaMemcpyHostToDevice);
}

int pamhd_gpu_get_state(pamhd_ctx* x, double* const soa[8])
{
	return get_state_impl(x, soa, cudaMemcpyDeviceToHost);
}

int pamhd_gpu_set_state_device(pamhd_ctx* x, const double* const soa[8])
{
	return set_state_impl(x, soa, cudaMemcpyDeviceToDevice);
}

int pamhd_gpu_get_state_device(pamhd_ctx* x, double* const soa[8])
{
	return get_state_impl(x, soa, cudaMemcpyDeviceToDevice);
}

int pamhd_gpu_step(pamhd_ctx* x, const double max_dt, double* dt_taken, double* max_signal)
{
	if (x == nullptr) return PAMHD_ERR_ARGUMENT;
	if (not x->loaded or x->half) return PAMHD_ERR_STATE;
	if (not (max_dt >= 0.0)) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(set_control(*x, max_dt, 0.0));
	PAMHD_TRY(issue_step(*x));
	// the step's clock and speed reduction sit in ring slot (steps after it) mod 3
	Clock c;
	PAMHD_TRY(check(cudaMemcpyAsync(&c, x->clock + x->steps % 3, sizeof c, cudaMemcpyDeviceToHost, x->stream)));
	Speed_Max r;
	PAMHD_TRY(check(cudaMemcpyAsync(&r, x->red + x->steps % 3, sizeof r, cudaMemcpyDeviceToHost, x->stream)));
	Status s;
	PAMHD_TRY(read_status(*x, s));
	if (dt_taken != nullptr) *dt_taken = c.dt;
	if (max_signal != nullptr) {
		// internal axis a holds the caller's axis map.perm[a]; the maxima are non-negative doubles
		for (int a = 0; a < 3; a++) {
			double v = 0.0;
			if (x->base.active[a]) std::memcpy(&v, &r.smax[a], sizeof v);
			max_signal[x->map.perm[a]] = v;
		}
	}
	return s.flags != 0 ? PAMHD_ERR_PHYSICS : PAMHD_OK;
}

int pamhd_gpu_steps(pamhd_ctx* x, const int32_t nsteps, const double t_end)
{
	if (x == nullptr or nsteps < 0) return PAMHD_ERR_ARGUMENT;
	if (not x->loaded or x->half) return PAMHD_ERR_STATE;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(set_control(*x, -1.0, t_end));
	int left = nsteps;
	while (left > 0 and x->steps % GRAPH_STEPS != 0) {
		PAMHD_TRY(issue_step(*x));
		left--;
	}
	if (left >= GRAPH_STEPS) {
		PAMHD_TRY(capture_graph(*x));
		while (left >= GRAPH_STEPS) {
			PAMHD_TRY(check(cudaGraphLaunch(x->graph, x->stream)));
			x->steps += GRAPH_STEPS;  // the state parity is unchanged after an even number of steps
			left -= GRAPH_STEPS;
		}
	}
	while (left > 0) {
		PAMHD_TRY(issue_step(*x));
		left--;
	}
	return PAMHD_OK;
}

int pamhd_gpu_step_part(pamhd_ctx* x, const int32_t part, const double t_end)
{
	if (x == nullptr or (part != 1 and part != 2)) return PAMHD_ERR_ARGUMENT;
	if (not x->loaded) return PAMHD_ERR_STATE;
	if (x->base.active[2] == 0) return PAMHD_ERR_ARGUMENT;  // needs z planes
	if ((part == 1) == (x->half != 0)) return PAMHD_ERR_STATE;  // parts 1 and 2 alternate
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	if (part == 1 and (x->control_max_dt != -1.0 or x->control_t_end != t_end)) {
		PAMHD_TRY(set_control(*x, -1.0, t_end));
	}
	PAMHD_TRY(issue_step_part(*x, part));
	x->half = part == 1 ? 1 : 0;
	return PAMHD_OK;
}

int pamhd_gpu_set_inflow(pamhd_ctx* x, const int32_t user_dim, const int32_t side, const int32_t count,
                         const double* times, const double* user_states)
{
	if (x == nullptr or user_dim < 0 or user_dim > 2 or (side != 0 and side != 1) or count < 0) {
		return PAMHD_ERR_ARGUMENT;
	}
	if ((count > 0 and times == nullptr) or user_states == nullptr) return PAMHD_ERR_ARGUMENT;
	// the internal axis and component order
	int dim = 0;
	while (x->map.perm[dim] != user_dim) dim++;
	std::vector<double> internal(8 * (size_t(count) + 1));
	for (size_t i = 0; i <= size_t(count); i++) {
		for (int v = 0; v < 8; v++) internal[8 * i + v] = user_states[8 * i + x->map.user_var(v)];
	}
	const double* states = internal.data();
	if ((side == 0 ? x->cfg.bc_lo[dim] : x->cfg.bc_hi[dim]) != PAMHD_BC_VALUE or x->cfg.n[dim] < 2) {
		return PAMHD_ERR_ARGUMENT;
	}
	for (int i = 0; i < count; i++) {
		if (not std::isfinite(times[i]) or (i > 0 and not (times[i] > times[i - 1]))) return PAMHD_ERR_ARGUMENT;
	}
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	const size_t nt = size_t(count), ns = 8 * (size_t(count) + 1);
	double* dev = nullptr;
	PAMHD_TRY(check(cudaMalloc(&dev, (nt + ns) * sizeof(double))));
	if (nt > 0 and cudaMemcpy(dev, times, nt * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
		cudaFree(dev);
		return PAMHD_ERR_CUDA;
	}
	if (cudaMemcpy(dev + nt, states, ns * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
		cudaFree(dev);
		return PAMHD_ERR_CUDA;
	}
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	cudaFree(x->inflow_dev[dim][side]);
	x->inflow_dev[dim][side] = dev;
	x->inflow_times[dim][side].assign(times, times + nt);
	x->inflow_states[dim][side].assign(states, states + ns);
	if (x->inflow_tables == nullptr) {
		PAMHD_TRY(check(cudaMalloc(&x->inflow_tables, 6 * sizeof(Inflow_Table))));
		PAMHD_TRY(check(cudaMemset(x->inflow_tables, 0, 6 * sizeof(Inflow_Table))));
	}
	const Inflow_Table table{dev, dev + nt, count};
	PAMHD_TRY(check(cudaMemcpy(x->inflow_tables + 2 * dim + side, &table, sizeof table, cudaMemcpyHostToDevice)));
	x->base.inflow = x->inflow_tables;
	// the captured steps hold the old parameters
	if (x->graph != nullptr) {
		cudaGraphExecDestroy(x->graph);
		x->graph = nullptr;
	}
	// the current state's ghosts take the value of the current time
	if (x->loaded) {
		Clock c;
		PAMHD_TRY(check(cudaMemcpyAsync(&c, x->clock + x->steps % 3, sizeof c, cudaMemcpyDeviceToHost, x->stream)));
		PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
		double lo[3][8], hi[3][8];
		values_at(*x, c.t, lo, hi);
		PAMHD_TRY(launch_fill_ghosts_values(x->base, x->state[x->cur], lo, hi, x->stream));
		PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	}
	return PAMHD_OK;
}

int pamhd_gpu_halo(pamhd_ctx* x, const int32_t side, const int32_t ghost, double* planes[8], int64_t* count)
{
	if (x == nullptr or planes == nullptr or count == nullptr) return PAMHD_ERR_ARGUMENT;
	if ((side != 0 and side != 1) or (ghost != 0 and ghost != 1)) return PAMHD_ERR_ARGUMENT;
	const Layout& L = x->L;
	if (L.g[2] == 0) return PAMHD_ERR_ARGUMENT;  // no z ghosts: not a slab
	const int k = side == 0 ? (ghost ? -1 : 0) : (ghost ? L.n[2] : L.n[2] - 1);
	const long long first = (long long)(k + L.g[2]) * L.plane;
	// between the two parts of a split step: the state that step writes
	const double* base = x->state[x->half ? x->cur ^ 1 : x->cur];
	for (int v = 0; v < 8; v++) planes[v] = const_cast<double*>(base) + v * L.var + first;
	*count = L.plane;
	return PAMHD_OK;
}

int pamhd_gpu_speed_slot(pamhd_ctx* x, void** slot)
{
	if (x == nullptr or slot == nullptr) return PAMHD_ERR_ARGUMENT;
	static_assert(sizeof(Speed_Max) == 32, "four 64-bit words");
	*slot = static_cast<void*>(x->red + x->steps % 3);
	return PAMHD_OK;
}

int pamhd_gpu_get_stream(pamhd_ctx* x, void** stream)
{
	if (x == nullptr or stream == nullptr) return PAMHD_ERR_ARGUMENT;
	*stream = static_cast<void*>(x->stream);
	return PAMHD_OK;
}

int pamhd_gpu_sync(pamhd_ctx* x)
{
	if (x == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	Status s;
	PAMHD_TRY(read_status(*x, s));
	return s.flags != 0 ? PAMHD_ERR_PHYSICS : PAMHD_OK;
}

int pamhd_gpu_time(pamhd_ctx* x, double* time, int64_t* steps, double* last_dt)
{
	if (x == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	Clock c;
	PAMHD_TRY(check(cudaMemcpyAsync(&c, x->clock + x->steps % 3, sizeof c, cudaMemcpyDeviceToHost, x->stream)));
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	if (time != nullptr) *time = c.t;
	if (steps != nullptr) *steps = c.steps;
	if (last_dt != nullptr) *last_dt = c.dt;
	return PAMHD_OK;
}

int pamhd_gpu_dt_history(pamhd_ctx* x, double* dt, const int32_t count, int32_t* written)
{
	if (x == nullptr or dt == nullptr or count < 0) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	std::vector<double> all(x->hist_len);
	PAMHD_TRY(check(cudaMemcpyAsync(all.data(), x->dt_hist, x->hist_len * sizeof(double),
	                                cudaMemcpyDeviceToHost, x->stream)));
	// the steps the grid took (a grid that stopped at a failure holds its count)
	Clock c;
	PAMHD_TRY(check(cudaMemcpyAsync(&c, x->clock + x->steps % 3, sizeof c, cudaMemcpyDeviceToHost, x->stream)));
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	const long long have = std::min<long long>(c.steps, x->hist_len);
	const long long n = std::min<long long>(have, count);
	for (long long i = 0; i < n; i++) {
		const long long step = c.steps - n + i;
		dt[i] = all[step % x->hist_len];
	}
	if (written != nullptr) *written = int32_t(n);
	return PAMHD_OK;
}

int pamhd_gpu_status(pamhd_ctx* x, uint32_t* flags, int32_t cell[3], int32_t* dir)
{
	if (x == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	Status s;
	PAMHD_TRY(read_status(*x, s));
	if (flags != nullptr) *flags = s.flags;
	int32_t c[3] = {0, 0, 0};
	int32_t d = 0;
	if (s.flags != 0 and s.first != ~0ull) {
		const unsigned long long key = s.first >> 8;
		d = int32_t(key & 3ull);
		unsigned long long lin = key >> 2;
		const Step_Params& P = x->base;
		const unsigned long long nx = x->L.n[0] + 2 * P.ext[0], ny = x->L.n[1] + 2 * P.ext[1];
		c[0] = int32_t(lin % nx) - P.ext[0];
		lin /= nx;
		c[1] = int32_t(lin % ny) - P.ext[1];
		c[2] = int32_t(lin / ny) - P.ext[2];
	}
	// in the caller's axes
	if (cell != nullptr) {
		for (int a = 0; a < 3; a++) cell[x->map.perm[a]] = c[a];
	}
	if (dir != nullptr) *dir = d > 0 ? x->map.perm[d - 1] + 1 : 0;
	return PAMHD_OK;
}

int pamhd_gpu_totals(pamhd_ctx* x, double totals[8])
{
	if (x == nullptr or totals == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(x->device)));
	PAMHD_TRY(launch_totals(x->state[x->cur], x->L, 0.0, x->partial, x->partial_blocks, x->stream));
	std::vector<double> part(8 * x->partial_blocks);
	PAMHD_TRY(check(cudaMemcpyAsync(part.data(), x->partial, part.size() * sizeof(double),
	                                cudaMemcpyDeviceToHost, x->stream)));
	PAMHD_TRY(check(cudaStreamSynchronize(x->stream)));
	const double volume = x->cfg.cell_length[0] * x->cfg.cell_length[1] * x->cfg.cell_length[2];
	for (int v = 0; v < 8; v++) {
		double sum = 0.0, comp = 0.0;
		for (int b = 0; b < x->partial_blocks; b++) {
			const double y = part[8 * b + v] - comp;
			const double t = sum + y;
			comp = (t - sum) - y;
			sum = t;
		}
		totals[x->map.user_var(v)] = sum * volume;
	}
	return PAMHD_OK;
}

int pamhd_gpu_face_flux(const int32_t device, const int32_t solver, const int64_t n, const double* neg,
                        const double* pos, const double* bg, const double adiabatic_index,
                        const double vacuum_permeability, double* flux, double* speed, uint32_t* flags)
{
	if (n < 0 or neg == nullptr or pos == nullptr or flux == nullptr or speed == nullptr or flags == nullptr) {
		return PAMHD_ERR_ARGUMENT;
	}
	if (solver != PAMHD_RUSANOV and solver != PAMHD_HLL_ATHENA and solver != PAMHD_HLLD_ATHENA
		and solver != PAMHD_ROE_ATHENA) {
		return PAMHD_ERR_ARGUMENT;
	}
	if (not (adiabatic_index > 1.0) or not (vacuum_permeability > 0.0)) return PAMHD_ERR_ARGUMENT;
	if (n == 0) return PAMHD_OK;
	PAMHD_TRY(check(cudaSetDevice(device)));
	Gas g;
	g.gamma = adiabatic_index;
	g.mu0 = vacuum_permeability;
	g.inv_mu0 = 1.0 / vacuum_permeability;
	g.sqrt_mu0 = std::sqrt(vacuum_permeability);
	g.inv_sqrt_mu0 = 1.0 / g.sqrt_mu0;
	double *dn = nullptr, *dp = nullptr, *db = nullptr, *df = nullptr, *ds = nullptr;
	uint32_t* dg = nullptr;
	int rc = PAMHD_OK;
	const size_t s8 = size_t(n) * 8 * sizeof(double);
	if (cudaMalloc(&dn, s8) != cudaSuccess or cudaMalloc(&dp, s8) != cudaSuccess
		or cudaMalloc(&df, s8) != cudaSuccess or cudaMalloc(&ds, n * sizeof(double)) != cudaSuccess
		or cudaMalloc(&dg, n * sizeof(uint32_t)) != cudaSuccess
		or (bg != nullptr and cudaMalloc(&db, size_t(n) * 3 * sizeof(double)) != cudaSuccess)) {
		rc = PAMHD_ERR_CUDA;
	}
	if (rc == PAMHD_OK) {
		rc = check(cudaMemcpy(dn, neg, s8, cudaMemcpyHostToDevice));
		if (rc == PAMHD_OK) rc = check(cudaMemcpy(dp, pos, s8, cudaMemcpyHostToDevice));
		if (rc == PAMHD_OK and bg != nullptr) {
			rc = check(cudaMemcpy(db, bg, size_t(n) * 3 * sizeof(double), cudaMemcpyHostToDevice));
		}
	}
	if (rc == PAMHD_OK) rc = launch_face_flux(solver, n, dn, dp, db, g, df, ds, dg, nullptr);
	if (rc == PAMHD_OK) rc = check(cudaMemcpy(flux, df, s8, cudaMemcpyDeviceToHost));
	if (rc == PAMHD_OK) rc = check(cudaMemcpy(speed, ds, n * sizeof(double), cudaMemcpyDeviceToHost));
	if (rc == PAMHD_OK) rc = check(cudaMemcpy(flags, dg, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
	cudaFree(dn);
	cudaFree(dp);
	cudaFree(db);
	cudaFree(df);
	cudaFree(ds);
	cudaFree(dg);
	if (rc != PAMHD_OK) return rc;
	for (int64_t i = 0; i < n; i++) {
		if (flags[i] != 0) return PAMHD_ERR_PHYSICS;
	}
	return PAMHD_OK;
}

} // extern "C"
