/*
Host side of the batched ensemble (include/pamhd_gpu.h, pamhd_gpu_batch_*):
independent uniform boxes of uneven sizes advanced together, one kernel
launch per step for the whole ensemble, each box with its own CFL
timestep, and multi-step runs replayed from one CUDA graph.

Device data: every box has its own two state copies (ping-pong), a
three-slot speed reduction ring, clock ring, status and dt history, laid
out back to back in shared allocations.  The work-item table lists
(box, tile, z chunk) for all boxes, largest boxes first; the persistent
batched kernel walks it with a grid stride.

The autotuner (pamhd_gpu_batch_tune) times a few steps of the actual
ensemble for each candidate of (z planes per work item, resident grid
size), keeps the fastest and restores the state it started from.
*/
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "grid_setup.cuh"
#include "step.cuh"

using namespace pamhd_b200;

namespace pamhd_b200 {
int launch_fill_ghosts_values(const Step_Params& P, double* state, const double lo[3][8], const double hi[3][8],
                              cudaStream_t stream);
}

struct pamhd_batch {
	int device = 0;
	cudaStream_t stream = nullptr;
	int nboxes = 0;
	int solver = 0;
	bool yact = true;
	std::vector<pamhd_cfg> cfg;
	std::vector<Layout> L;
	std::vector<long long> off;      // doubles from the start of a state buffer to each box
	long long total = 0;             // doubles per state buffer
	double* state[2] = {nullptr, nullptr};
	Speed_Max* red = nullptr;        // 3 per box
	Clock* clock = nullptr;          // 3 per box
	Status* status = nullptr;        // 1 per box
	Control* control = nullptr;
	double* dt_hist = nullptr;       // hist_len per box
	int hist_len = 4096;
	std::vector<Step_Params> params[2];
	Step_Params* d_params[2] = {nullptr, nullptr};
	int4* d_items = nullptr;
	int nitems = 0;                  // work items of the boxes' tiles (the per-step kernel's table)
	int nitems_run = 0;              // the same plus the boundary-face chunks (the persistent run's table)
	int grid = 0;
	int planes_per_item = 32;
	int ty = 1;                      // tile rows of the work items (autotuned when y is active)
	bool needs_boundary = false;
	int largest_plane = 0;
	double* staging = nullptr;
	long long steps = 0;
	int cur = 0;
	bool loaded = false;
	cudaGraphExec_t graph = nullptr;
	// the persistent run (pamhd_gpu_batch_run): scheduler state, per-box items per step and items
	// done, poll limit, resident grid, its graph
	Run_Sync* sync = nullptr;
	int* d_box_items = nullptr;
	unsigned int* d_done = nullptr;
	long long wait_limit = 10000000;
	int run_grid = 0;
	cudaGraphExec_t run_graph = nullptr;
	long long run_key = -1;          // nsteps, state parity and step phase the run graph was captured for
	bool run_graphed = false;        // whether the last run was replayed from a graph
	Axis_Map map{{0, 1, 2}};        // the boxes' axes as the kernels see them
	// time-stamped inflow of VALUE sides, per box and side (index 6 box + 2 dimension + side)
	std::vector<Inflow_Table> inflow;
	Inflow_Table* d_inflow = nullptr;   // the same tables in device memory
	std::vector<double*> inflow_dev;
	std::vector<std::vector<double>> inflow_times, inflow_states;
};

namespace {

constexpr int GRAPH_STEPS = 6;

int check(const cudaError_t e)
{
	return e == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

#define PAMHD_TRY(expr) do { const int rc_ = (expr); if (rc_ != PAMHD_OK) return rc_; } while (0)

long long cells_of(const pamhd_cfg& c)
{
	return (long long)c.n[0] * c.n[1] * c.n[2];
}

// the tile shapes the autotuner chooses among: 32 x 4 and 32 x 8 (32 x 1 when y is inactive)
std::vector<int> tile_choices(const pamhd_batch& b)
{
	if (not b.yact) return {1};
	return {batch_tile_rows(), 8};
}

// ghost states of a box's VALUE sides at time t: configured values or time-stamped inflow
void box_values_at(const pamhd_batch& b, const int box, const double t, double lo[3][8], double hi[3][8])
{
	for (int d = 0; d < 3; d++) {
		for (int side = 0; side < 2; side++) {
			double* out = side == 0 ? lo[d] : hi[d];
			const double* v = side == 0 ? b.cfg[box].value_lo[d] : b.cfg[box].value_hi[d];
			if (not b.inflow.empty()) {
				const size_t k = 6 * size_t(box) + 2 * d + side;
				const std::vector<double>& times = b.inflow_times[k];
				const std::vector<double>& states = b.inflow_states[k];
				if (not states.empty()) {
					size_t i = 0;
					while (i < times.size() and t >= times[i]) i++;
					v = states.data() + 8 * i;
				}
			}
			for (int q = 0; q < 8; q++) out[q] = v[q];
		}
	}
}

// per-box parameters and the work-item table for a given number of z planes per item
int build_work(pamhd_batch& b, const int planes)
{
	b.planes_per_item = planes;
	const int ty = b.ty;
	std::vector<int> order(b.nboxes);
	std::iota(order.begin(), order.end(), 0);
	std::stable_sort(order.begin(), order.end(),
	                 [&](int x, int y) { return cells_of(b.cfg[x]) > cells_of(b.cfg[y]); });
	std::vector<int4> items;
	b.needs_boundary = false;
	b.largest_plane = 0;
	for (int parity = 0; parity < 2; parity++) b.params[parity].resize(b.nboxes);
	for (int i = 0; i < b.nboxes; i++) {
		Step_Params P;
		const bool nb = grid_params(b.cfg[i], b.L[i], P, planes);
		P.kchunk = std::max(1, std::min(planes, b.cfg[i].n[2]));
		b.needs_boundary = b.needs_boundary or nb;
		for (int d = 0; d < 3; d++) {
			for (int e = 0; e < 3; e++) {
				if (e != d) b.largest_plane = std::max(b.largest_plane, b.cfg[i].n[d] * b.cfg[i].n[e]);
			}
		}
		if (b.d_inflow != nullptr) {
			bool any = false;
			for (int k = 0; k < 6; k++) any = any or b.inflow[6 * size_t(i) + k].states != nullptr;
			if (any) P.inflow = b.d_inflow + 6 * size_t(i);
		}
		P.red = b.red + 3 * i;
		P.clock = b.clock + 3 * i;
		P.status = b.status + i;
		P.control = b.control;
		P.dt_hist = b.dt_hist + (long long)b.hist_len * i;
		P.hist_len = b.hist_len;
		for (int parity = 0; parity < 2; parity++) {
			Step_Params Q = P;
			Q.in = b.state[parity] + b.off[i];
			Q.out = b.state[parity ^ 1] + b.off[i];
			b.params[parity][i] = Q;
		}
	}
	for (const int i: order) {
		const pamhd_cfg& c = b.cfg[i];
		const int tiles = ((c.n[0] + 31) / 32) * ((c.n[1] + ty - 1) / ty);
		const int kc = b.params[0][i].kchunk;
		const int chunks = (c.n[2] + kc - 1) / kc;
		for (int z = 0; z < chunks; z++) {
			for (int t = 0; t < tiles; t++) items.push_back(make_int4(i, t, z, 0));
		}
	}
	b.nitems = int(items.size());
	// the persistent run also solves the ghost-ghost faces of non-periodic sides (for their speeds),
	// in chunks: (box, combination, chunk, 1), the combinations numbered as boundary_combos does
	for (const int i: order) {
		const Step_Params& P = b.params[0][i];
		int combo = 0;
		for (int d = 0; d < 3; d++) {
			if (not P.active[d] or P.periodic[d]) continue;
			for (int side = 0; side < 2; side++) {
				if ((side ? P.bc_hi[d] : P.bc_lo[d]) == PAMHD_BC_EXTERNAL) continue;
				for (int e = 0; e < 3; e++) {
					if (e == d or not P.active[e]) continue;
					const int f = 3 - d - e;
					const int ne = (P.periodic[e] or P.bc_hi[e] == PAMHD_BC_EXTERNAL) ? P.L.n[e] : P.L.n[e] - 1;
					const long long count = (long long)ne * P.L.n[f];
					const int chunks = int((count + BOUNDARY_CHUNK - 1) / BOUNDARY_CHUNK);
					for (int k = 0; k < chunks; k++) items.push_back(make_int4(i, combo, k, 1));
					combo++;
				}
			}
		}
	}
	b.nitems_run = int(items.size());
	std::vector<int> per_box(b.nboxes, 0);
	for (const int4& w: items) per_box[w.x]++;
	PAMHD_TRY(check(cudaMemcpy(b.d_box_items, per_box.data(), b.nboxes * sizeof(int), cudaMemcpyHostToDevice)));
	cudaFree(b.d_items);
	b.d_items = nullptr;
	PAMHD_TRY(check(cudaMalloc(&b.d_items, items.size() * sizeof(int4))));
	PAMHD_TRY(check(cudaMemcpy(b.d_items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice)));
	for (int parity = 0; parity < 2; parity++) {
		PAMHD_TRY(check(cudaMemcpy(b.d_params[parity], b.params[parity].data(), b.nboxes * sizeof(Step_Params),
		                           cudaMemcpyHostToDevice)));
	}
	if (b.graph != nullptr) {
		cudaGraphExecDestroy(b.graph);
		b.graph = nullptr;
	}
	if (b.run_graph != nullptr) {
		cudaGraphExecDestroy(b.run_graph);
		b.run_graph = nullptr;
		b.run_key = -1;
	}
	return PAMHD_OK;
}

int reset_run_state(pamhd_batch& b)
{
	PAMHD_TRY(check(cudaMemsetAsync(b.red, 0, 3 * b.nboxes * sizeof(Speed_Max), b.stream)));
	PAMHD_TRY(check(cudaMemsetAsync(b.clock, 0, 3 * b.nboxes * sizeof(Clock), b.stream)));
	std::vector<Status> s(b.nboxes);
	for (auto& x: s) {
		x.flags = 0;
		x.fail_step = 0;
		x.first = ~0ull;
	}
	PAMHD_TRY(check(cudaMemcpyAsync(b.status, s.data(), s.size() * sizeof(Status), cudaMemcpyHostToDevice,
	                                b.stream)));
	PAMHD_TRY(check(cudaStreamSynchronize(b.stream)));
	b.steps = 0;
	b.cur = 0;
	return PAMHD_OK;
}

int issue_step(pamhd_batch& b)
{
	const int phase = int(b.steps % 3);
	if (b.needs_boundary) {
		PAMHD_TRY(launch_batch_boundary_speeds(b.d_params[b.cur], b.nboxes, b.largest_plane, phase, b.solver,
		                                       b.stream));
	}
	PAMHD_TRY(launch_batch_step(b.d_params[b.cur], b.d_items, b.nitems, phase, b.grid, b.solver, b.ty, b.stream));
	b.cur ^= 1;
	b.steps++;
	return PAMHD_OK;
}

int set_control(pamhd_batch& b, const double max_dt, const double t_end)
{
	Control c;
	c.max_dt = max_dt;
	c.t_end = t_end;
	PAMHD_TRY(check(cudaMemcpyAsync(b.control, &c, sizeof c, cudaMemcpyHostToDevice, b.stream)));
	return check(cudaStreamSynchronize(b.stream));
}

int capture_graph(pamhd_batch& b)
{
	if (b.graph != nullptr) return PAMHD_OK;
	cudaGraph_t g = nullptr;
	PAMHD_TRY(check(cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal)));
	const long long steps0 = b.steps;
	const int cur0 = b.cur;
	int rc = PAMHD_OK;
	for (int s = 0; s < GRAPH_STEPS and rc == PAMHD_OK; s++) rc = issue_step(b);
	b.steps = steps0;
	b.cur = cur0;
	const cudaError_t e = cudaStreamEndCapture(b.stream, &g);
	if (rc != PAMHD_OK or e != cudaSuccess) {
		if (g != nullptr) cudaGraphDestroy(g);
		return rc != PAMHD_OK ? rc : PAMHD_ERR_CUDA;
	}
	const cudaError_t ie = cudaGraphInstantiate(&b.graph, g, 0);
	cudaGraphDestroy(g);
	return check(ie);
}

int run_steps(pamhd_batch& b, int left)
{
	while (left > 0 and b.steps % GRAPH_STEPS != 0) {
		PAMHD_TRY(issue_step(b));
		left--;
	}
	if (left >= GRAPH_STEPS) {
		PAMHD_TRY(capture_graph(b));
		while (left >= GRAPH_STEPS) {
			PAMHD_TRY(check(cudaGraphLaunch(b.graph, b.stream)));
			b.steps += GRAPH_STEPS;
			left -= GRAPH_STEPS;
		}
	}
	while (left > 0) {
		PAMHD_TRY(issue_step(b));
		left--;
	}
	return PAMHD_OK;
}

// the resident grid of the persistent run for the current tile shape (one wave: a cooperative launch)
int set_run_grid(pamhd_batch& b)
{
	int per_sm = 0, sms = 0;
	PAMHD_TRY(batch_run_blocks_per_sm(b.solver, b.ty, &per_sm));
	PAMHD_TRY(check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b.device)));
	if (per_sm < 1) return PAMHD_ERR_CUDA;
	b.run_grid = std::max(1, std::min(b.nitems_run, sms * per_sm));
	return PAMHD_OK;
}

int issue_run(pamhd_batch& b, const int nsteps)
{
	if ((long long)nsteps * b.nitems_run >= (1ll << 31)) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaMemsetAsync(b.sync, 0, sizeof(Run_Sync), b.stream)));
	PAMHD_TRY(check(cudaMemsetAsync(b.d_done, 0, b.nboxes * sizeof(unsigned int), b.stream)));
	return launch_batch_run(b.d_params[b.cur], b.d_params[b.cur ^ 1], b.d_items, b.nitems_run, b.d_box_items,
	                        b.d_done, b.nboxes, b.steps, nsteps, b.sync, b.wait_limit, b.run_grid, b.solver, b.ty,
	                        b.stream);
}

/*
nsteps steps in one persistent launch, replayed from a CUDA graph of that one launch (captured
again when nsteps, the state parity or the step phase differ from the captured ones); launched
directly when the capture is refused.
*/
int run_persistent(pamhd_batch& b, const int nsteps)
{
	if (nsteps <= 0) return PAMHD_OK;
	PAMHD_TRY(set_run_grid(b));
	const long long key = (long long)nsteps * 6 + b.cur * 3 + b.steps % 3;
	if (b.run_graph == nullptr or b.run_key != key) {
		if (b.run_graph != nullptr) {
			cudaGraphExecDestroy(b.run_graph);
			b.run_graph = nullptr;
		}
		b.run_key = -1;
		cudaGraph_t g = nullptr;
		bool ok = cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
		const int rc = ok ? issue_run(b, nsteps) : PAMHD_ERR_CUDA;
		if (ok) ok = cudaStreamEndCapture(b.stream, &g) == cudaSuccess and rc == PAMHD_OK;
		if (ok) ok = cudaGraphInstantiate(&b.run_graph, g, 0) == cudaSuccess;
		if (g != nullptr) cudaGraphDestroy(g);
		cudaGetLastError();  // a refused capture leaves no error behind
		if (ok) {
			b.run_key = key;
		} else if (b.run_graph != nullptr) {
			cudaGraphExecDestroy(b.run_graph);
			b.run_graph = nullptr;
		}
	}
	if (b.run_graph != nullptr) {
		PAMHD_TRY(check(cudaGraphLaunch(b.run_graph, b.stream)));
		b.run_graphed = true;
	} else {
		PAMHD_TRY(issue_run(b, nsteps));
		b.run_graphed = false;
	}
	b.steps += nsteps;
	b.cur ^= nsteps & 1;
	return PAMHD_OK;
}

int box_ok(const pamhd_batch* b, const int box)
{
	return (b != nullptr and box >= 0 and box < b->nboxes) ? PAMHD_OK : PAMHD_ERR_ARGUMENT;
}

} // namespace

extern "C" {

int pamhd_gpu_batch_create(const int32_t device, const int32_t nboxes, const pamhd_cfg* user_cfgs, pamhd_batch** out)
{
	if (out == nullptr or user_cfgs == nullptr or nboxes < 1) return PAMHD_ERR_ARGUMENT;
	*out = nullptr;
	// every box with the same active dimensions, relabelled the same way (see Axis_Map)
	const Axis_Map map = axis_map(user_cfgs[0]);
	std::vector<pamhd_cfg> internal(nboxes);
	for (int i = 0; i < nboxes; i++) {
		for (int d = 0; d < 3; d++) {
			if ((user_cfgs[i].n[d] > 1) != (user_cfgs[0].n[d] > 1)) return PAMHD_ERR_ARGUMENT;
			if (user_cfgs[i].bc_lo[d] == PAMHD_BC_EXTERNAL or user_cfgs[i].bc_hi[d] == PAMHD_BC_EXTERNAL) {
				return PAMHD_ERR_ARGUMENT;
			}
		}
		internal[i] = relabelled(user_cfgs[i], map);
		PAMHD_TRY(validate(internal[i]));
		if (internal[i].solver != internal[0].solver) return PAMHD_ERR_ARGUMENT;
	}
	const pamhd_cfg* cfgs = internal.data();
	pamhd_batch* b = new (std::nothrow) pamhd_batch;
	if (b == nullptr) return PAMHD_ERR_ARGUMENT;
	auto fail = [&](const int rc) {
		pamhd_gpu_batch_destroy(b);
		return rc;
	};
	b->device = device;
	b->map = map;
	b->nboxes = nboxes;
	b->solver = cfgs[0].solver;
	b->yact = cfgs[0].n[1] > 1;
	b->cfg.assign(cfgs, cfgs + nboxes);
	long long largest_cells = 0;
	for (int i = 0; i < nboxes; i++) {
		b->L.push_back(make_layout(cfgs[i]));
		b->off.push_back(b->total);
		b->total += 8 * b->L.back().var;
		largest_cells = std::max(largest_cells, cells_of(cfgs[i]));
	}
	if (cudaSetDevice(device) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(PAMHD_ERR_CUDA);
	const size_t bytes = size_t(b->total) * sizeof(double);
	if (cudaMalloc(&b->state[0], bytes) != cudaSuccess or cudaMalloc(&b->state[1], bytes) != cudaSuccess
		or cudaMalloc(&b->red, 3 * nboxes * sizeof(Speed_Max)) != cudaSuccess
		or cudaMalloc(&b->clock, 3 * nboxes * sizeof(Clock)) != cudaSuccess
		or cudaMalloc(&b->status, nboxes * sizeof(Status)) != cudaSuccess
		or cudaMalloc(&b->control, sizeof(Control)) != cudaSuccess
		or cudaMalloc(&b->dt_hist, size_t(b->hist_len) * nboxes * sizeof(double)) != cudaSuccess
		or cudaMalloc(&b->d_params[0], nboxes * sizeof(Step_Params)) != cudaSuccess
		or cudaMalloc(&b->d_params[1], nboxes * sizeof(Step_Params)) != cudaSuccess
		or cudaMalloc(&b->staging, largest_cells * sizeof(double)) != cudaSuccess
		or cudaMalloc(&b->sync, sizeof(Run_Sync)) != cudaSuccess
		or cudaMalloc(&b->d_box_items, nboxes * sizeof(int)) != cudaSuccess
		or cudaMalloc(&b->d_done, nboxes * sizeof(unsigned int)) != cudaSuccess) {
		return fail(PAMHD_ERR_CUDA);
	}
	if (cudaMemset(b->state[0], 0, bytes) != cudaSuccess or cudaMemset(b->state[1], 0, bytes) != cudaSuccess
		or cudaMemset(b->dt_hist, 0, size_t(b->hist_len) * nboxes * sizeof(double)) != cudaSuccess) {
		return fail(PAMHD_ERR_CUDA);
	}
	b->ty = b->yact ? batch_tile_rows() : 1;
	for (const int ty: tile_choices(*b)) {
		if (prepare_batch_kernels(b->solver, ty) != PAMHD_OK) return fail(PAMHD_ERR_CUDA);
		if (prepare_batch_run_kernels(b->solver, ty) != PAMHD_OK) return fail(PAMHD_ERR_CUDA);
	}
	int per_sm = 0;
	if (batch_blocks_per_sm(b->solver, b->ty, &per_sm) != PAMHD_OK or per_sm < 1) return fail(PAMHD_ERR_CUDA);
	int sms = 0;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
	if (build_work(*b, 32) != PAMHD_OK) return fail(PAMHD_ERR_CUDA);
	b->grid = std::min(b->nitems, std::max(1, sms * per_sm));
	if (reset_run_state(*b) != PAMHD_OK) return fail(PAMHD_ERR_CUDA);
	*out = b;
	return PAMHD_OK;
}

int pamhd_gpu_batch_destroy(pamhd_batch* b)
{
	if (b == nullptr) return PAMHD_OK;
	cudaSetDevice(b->device);
	if (b->stream != nullptr) cudaStreamSynchronize(b->stream);
	if (b->graph != nullptr) cudaGraphExecDestroy(b->graph);
	if (b->run_graph != nullptr) cudaGraphExecDestroy(b->run_graph);
	cudaFree(b->sync);
	cudaFree(b->d_box_items);
	cudaFree(b->d_done);
	cudaFree(b->state[0]);
	cudaFree(b->state[1]);
	cudaFree(b->red);
	cudaFree(b->clock);
	cudaFree(b->status);
	cudaFree(b->control);
	cudaFree(b->dt_hist);
	cudaFree(b->d_params[0]);
	cudaFree(b->d_params[1]);
	cudaFree(b->d_items);
	cudaFree(b->staging);
	for (double* p: b->inflow_dev) cudaFree(p);
	cudaFree(b->d_inflow);
	if (b->stream != nullptr) cudaStreamDestroy(b->stream);
	delete b;
	return PAMHD_OK;
}

int pamhd_gpu_batch_set_state(pamhd_batch* b, const int32_t box, const double* const user[8])
{
	PAMHD_TRY(box_ok(b, box));
	if (user == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int v = 0; v < 8; v++) if (user[v] == nullptr) return PAMHD_ERR_ARGUMENT;
	const double* soa[8];
	for (int v = 0; v < 8; v++) soa[v] = user[b->map.user_var(v)];
	PAMHD_TRY(check(cudaSetDevice(b->device)));
	const Layout& L = b->L[box];
	const size_t bytes = size_t(cells_of(b->cfg[box])) * sizeof(double);
	for (int side = 0; side < 2; side++) {
		double* base = b->state[side] + b->off[box];
		if (side == 0) {
			for (int v = 0; v < 8; v++) {
				PAMHD_TRY(check(cudaMemcpyAsync(b->staging, soa[v], bytes, cudaMemcpyHostToDevice, b->stream)));
				PAMHD_TRY(launch_scatter(b->staging, base + v * L.var, L, b->stream));
			}
		}
		double lo[3][8], hi[3][8];
		box_values_at(*b, box, 0.0, lo, hi);
		PAMHD_TRY(launch_fill_ghosts_values(b->params[0][box], base, lo, hi, b->stream));
	}
	b->loaded = true;
	return reset_run_state(*b);
}

int pamhd_gpu_batch_set_inflow(pamhd_batch* b, const int32_t box, const int32_t user_dim, const int32_t side,
                               const int32_t count, const double* times, const double* user_states)
{
	PAMHD_TRY(box_ok(b, box));
	if (user_dim < 0 or user_dim > 2 or (side != 0 and side != 1) or count < 0) return PAMHD_ERR_ARGUMENT;
	if ((count > 0 and times == nullptr) or user_states == nullptr) return PAMHD_ERR_ARGUMENT;
	// the internal axis and component order
	int dim = 0;
	while (b->map.perm[dim] != user_dim) dim++;
	std::vector<double> internal_states(8 * (size_t(count) + 1));
	for (size_t i = 0; i <= size_t(count); i++) {
		for (int v = 0; v < 8; v++) internal_states[8 * i + v] = user_states[8 * i + b->map.user_var(v)];
	}
	const double* states = internal_states.data();
	const pamhd_cfg& c = b->cfg[box];
	if ((side == 0 ? c.bc_lo[dim] : c.bc_hi[dim]) != PAMHD_BC_VALUE or c.n[dim] < 2) return PAMHD_ERR_ARGUMENT;
	for (int i = 0; i < count; i++) {
		if (not std::isfinite(times[i]) or (i > 0 and not (times[i] > times[i - 1]))) return PAMHD_ERR_ARGUMENT;
	}
	PAMHD_TRY(check(cudaSetDevice(b->device)));
	const size_t nt = size_t(count), ns = 8 * (size_t(count) + 1);
	double* dev = nullptr;
	PAMHD_TRY(check(cudaMalloc(&dev, (nt + ns) * sizeof(double))));
	if ((nt > 0 and cudaMemcpy(dev, times, nt * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
		or cudaMemcpy(dev + nt, states, ns * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
		cudaFree(dev);
		return PAMHD_ERR_CUDA;
	}
	PAMHD_TRY(check(cudaStreamSynchronize(b->stream)));
	if (b->inflow.empty()) {
		b->inflow.assign(6 * size_t(b->nboxes), Inflow_Table{nullptr, nullptr, 0});
		b->inflow_dev.assign(6 * size_t(b->nboxes), nullptr);
		b->inflow_times.assign(6 * size_t(b->nboxes), {});
		b->inflow_states.assign(6 * size_t(b->nboxes), {});
		PAMHD_TRY(check(cudaMalloc(&b->d_inflow, 6 * size_t(b->nboxes) * sizeof(Inflow_Table))));
		PAMHD_TRY(check(cudaMemset(b->d_inflow, 0, 6 * size_t(b->nboxes) * sizeof(Inflow_Table))));
	}
	const size_t k = 6 * size_t(box) + 2 * dim + side;
	cudaFree(b->inflow_dev[k]);
	b->inflow_dev[k] = dev;
	b->inflow[k] = Inflow_Table{dev, dev + nt, count};
	b->inflow_times[k].assign(times, times + nt);
	b->inflow_states[k].assign(states, states + ns);
	PAMHD_TRY(check(cudaMemcpy(b->d_inflow + k, &b->inflow[k], sizeof(Inflow_Table), cudaMemcpyHostToDevice)));
	for (int parity = 0; parity < 2; parity++) {
		b->params[parity][box].inflow = b->d_inflow + 6 * size_t(box);
		PAMHD_TRY(check(cudaMemcpy(b->d_params[parity] + box, &b->params[parity][box], sizeof(Step_Params),
		                           cudaMemcpyHostToDevice)));
	}
	if (b->graph != nullptr) {
		cudaGraphExecDestroy(b->graph);
		b->graph = nullptr;
	}
	if (b->loaded) {
		Clock clk;
		PAMHD_TRY(check(cudaMemcpy(&clk, b->clock + 3 * size_t(box) + b->steps % 3, sizeof clk,
		                           cudaMemcpyDeviceToHost)));
		double lo[3][8], hi[3][8];
		box_values_at(*b, box, clk.t, lo, hi);
		PAMHD_TRY(launch_fill_ghosts_values(b->params[b->cur][box], b->state[b->cur] + b->off[box], lo, hi,
		                                    b->stream));
		PAMHD_TRY(check(cudaStreamSynchronize(b->stream)));
	}
	return PAMHD_OK;
}

int pamhd_gpu_batch_get_state(pamhd_batch* b, const int32_t box, double* const user[8])
{
	PAMHD_TRY(box_ok(b, box));
	if (user == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int v = 0; v < 8; v++) if (user[v] == nullptr) return PAMHD_ERR_ARGUMENT;
	double* soa[8];
	for (int v = 0; v < 8; v++) soa[v] = user[b->map.user_var(v)];
	PAMHD_TRY(check(cudaSetDevice(b->device)));
	const Layout& L = b->L[box];
	const size_t bytes = size_t(cells_of(b->cfg[box])) * sizeof(double);
	const double* base = b->state[b->cur] + b->off[box];
	for (int v = 0; v < 8; v++) {
		PAMHD_TRY(launch_gather(base + v * L.var, b->staging, L, b->stream));
		PAMHD_TRY(check(cudaMemcpyAsync(soa[v], b->staging, bytes, cudaMemcpyDeviceToHost, b->stream)));
	}
	return check(cudaStreamSynchronize(b->stream));
}

int pamhd_gpu_batch_steps(pamhd_batch* b, const int32_t nsteps, const double t_end)
{
	if (b == nullptr or nsteps < 0) return PAMHD_ERR_ARGUMENT;
	if (not b->loaded) return PAMHD_ERR_STATE;
	PAMHD_TRY(check(cudaSetDevice(b->device)));
	PAMHD_TRY(set_control(*b, -1.0, t_end));
	return run_steps(*b, nsteps);
}

int pamhd_gpu_batch_run(pamhd_batch* b, const int32_t nsteps, const double t_end)
{
	if (b == nullptr or nsteps < 0) return PAMHD_ERR_ARGUMENT;
	if (not b->loaded) return PAMHD_ERR_STATE;
	PAMHD_TRY(check(cudaSetDevice(b->device)));
	PAMHD_TRY(set_control(*b, -1.0, t_end));
	return run_persistent(*b, nsteps);
}

int pamhd_gpu_batch_set_wait_limit(pamhd_batch* b, const int64_t polls)
{
	if (b == nullptr or polls < 0) return PAMHD_ERR_ARGUMENT;
	b->wait_limit = polls;
	// the limit is a launch argument: a graph captured with the old one is captured again
	if (b->run_graph != nullptr) {
		PAMHD_TRY(check(cudaSetDevice(b->device)));
		PAMHD_TRY(check(cudaStreamSynchronize(b->stream)));
		cudaGraphExecDestroy(b->run_graph);
		b->run_graph = nullptr;
		b->run_key = -1;
	}
	return PAMHD_OK;
}

int pamhd_gpu_batch_run_info(pamhd_batch* b, int32_t* grid, int32_t* items, int32_t* graphed)
{
	if (b == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(b->device)));
	PAMHD_TRY(set_run_grid(*b));
	if (grid != nullptr) *grid = b->run_grid;
	if (items != nullptr) *items = b->nitems_run;
	if (graphed != nullptr) *graphed = b->run_graphed ? 1 : 0;
	return PAMHD_OK;
}

int pamhd_gpu_batch_tune(pamhd_batch* b, const int32_t trial_steps, int32_t* planes_chosen, int32_t* grid_chosen)
{
	if (b == nullptr or trial_steps < 1) return PAMHD_ERR_ARGUMENT;
	if (not b->loaded) return PAMHD_ERR_STATE;
	PAMHD_TRY(check(cudaSetDevice(b->device)));
	PAMHD_TRY(check(cudaStreamSynchronize(b->stream)));
	// keep the state the trials start from
	double* backup = nullptr;
	PAMHD_TRY(check(cudaMalloc(&backup, size_t(b->total) * sizeof(double))));
	int rc = check(cudaMemcpyAsync(backup, b->state[b->cur], size_t(b->total) * sizeof(double),
	                               cudaMemcpyDeviceToDevice, b->stream));
	int sms = 0;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
	float best = 3.0e38f;
	int best_planes = b->planes_per_item, best_grid = b->grid, best_ty = b->ty;
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	if (rc == PAMHD_OK) rc = set_control(*b, -1.0, 1.0e300);
	for (const int ty: tile_choices(*b))
	for (const int planes: {8, 16, 32, 64}) {
		if (rc != PAMHD_OK) break;
		b->ty = ty;
		int per_sm = 0;
		rc = batch_blocks_per_sm(b->solver, ty, &per_sm);
		if (rc == PAMHD_OK) rc = build_work(*b, planes);
		for (const int waves: {1, 2, 0}) {
			if (rc != PAMHD_OK) break;
			b->grid = waves == 0 ? b->nitems : std::min(b->nitems, std::max(1, waves * sms * per_sm));
			rc = check(cudaMemcpyAsync(b->state[b->cur], backup, size_t(b->total) * sizeof(double),
			                           cudaMemcpyDeviceToDevice, b->stream));
			if (rc == PAMHD_OK) rc = issue_step(*b);  // warm-up (and priming after a reset)
			if (rc == PAMHD_OK) rc = check(cudaEventRecord(e0, b->stream));
			for (int s = 0; s < trial_steps and rc == PAMHD_OK; s++) rc = issue_step(*b);
			if (rc == PAMHD_OK) rc = check(cudaEventRecord(e1, b->stream));
			if (rc == PAMHD_OK) rc = check(cudaEventSynchronize(e1));
			float ms = 0.0f;
			if (rc == PAMHD_OK) rc = check(cudaEventElapsedTime(&ms, e0, e1));
			if (rc == PAMHD_OK and ms < best) {
				best = ms;
				best_planes = planes;
				best_grid = b->grid;
				best_ty = ty;
			}
			// the trial steps advanced the state: go back to the starting buffer parity
			if (rc == PAMHD_OK and b->cur != 0) {
				rc = check(cudaMemcpyAsync(b->state[0], b->state[1], size_t(b->total) * sizeof(double),
				                           cudaMemcpyDeviceToDevice, b->stream));
			}
			b->cur = 0;
			if (rc == PAMHD_OK) rc = reset_run_state(*b);
		}
	}
	b->ty = best_ty;
	if (rc == PAMHD_OK) rc = build_work(*b, best_planes);
	b->grid = best_grid;
	if (rc == PAMHD_OK) {
		rc = check(cudaMemcpyAsync(b->state[0], backup, size_t(b->total) * sizeof(double), cudaMemcpyDeviceToDevice,
		                           b->stream));
	}
	if (rc == PAMHD_OK) rc = reset_run_state(*b);
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(backup);
	if (planes_chosen != nullptr) *planes_chosen = best_planes;
	if (grid_chosen != nullptr) *grid_chosen = best_grid;
	return rc;
}

int pamhd_gpu_batch_set_tiling(pamhd_batch* b, const int32_t tile_rows, const int32_t planes, const int32_t grid)
{
	if (b == nullptr or planes < 1 or grid < 1) return PAMHD_ERR_ARGUMENT;
	const std::vector<int> choices = tile_choices(*b);
	if (std::find(choices.begin(), choices.end(), int(tile_rows)) == choices.end()) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(b->device)));
	PAMHD_TRY(check(cudaStreamSynchronize(b->stream)));
	b->ty = tile_rows;
	PAMHD_TRY(build_work(*b, planes));
	b->grid = std::min(b->nitems, int(grid));
	return PAMHD_OK;
}

int pamhd_gpu_batch_tune_run(pamhd_batch* b, const int32_t trial_steps, int32_t* tile_rows_chosen,
                             int32_t* planes_chosen)
{
	if (b == nullptr or trial_steps < 1) return PAMHD_ERR_ARGUMENT;
	if (not b->loaded) return PAMHD_ERR_STATE;
	PAMHD_TRY(check(cudaSetDevice(b->device)));
	PAMHD_TRY(check(cudaStreamSynchronize(b->stream)));
	// keep the state the trials start from
	double* backup = nullptr;
	PAMHD_TRY(check(cudaMalloc(&backup, size_t(b->total) * sizeof(double))));
	int rc = check(cudaMemcpyAsync(backup, b->state[b->cur], size_t(b->total) * sizeof(double),
	                               cudaMemcpyDeviceToDevice, b->stream));
	float best = 3.0e38f;
	int best_planes = b->planes_per_item, best_ty = b->ty;
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	if (rc == PAMHD_OK) rc = set_control(*b, -1.0, 1.0e300);
	for (const int ty: tile_choices(*b))
	for (const int planes: {8, 16, 32, 64}) {
		if (rc != PAMHD_OK) break;
		b->ty = ty;
		rc = build_work(*b, planes);
		if (rc == PAMHD_OK) rc = set_run_grid(*b);
		if (rc == PAMHD_OK) {
			rc = check(cudaMemcpyAsync(b->state[0], backup, size_t(b->total) * sizeof(double),
			                           cudaMemcpyDeviceToDevice, b->stream));
		}
		b->cur = 0;
		if (rc == PAMHD_OK) rc = reset_run_state(*b);
		if (rc == PAMHD_OK) rc = check(cudaEventRecord(e0, b->stream));
		if (rc == PAMHD_OK) rc = issue_run(*b, trial_steps + 1);  // the priming step and the trial steps
		if (rc == PAMHD_OK) rc = check(cudaEventRecord(e1, b->stream));
		if (rc == PAMHD_OK) rc = check(cudaEventSynchronize(e1));
		float ms = 0.0f;
		if (rc == PAMHD_OK) rc = check(cudaEventElapsedTime(&ms, e0, e1));
		if (rc == PAMHD_OK and ms < best) {
			best = ms;
			best_planes = planes;
			best_ty = ty;
		}
	}
	b->ty = best_ty;
	if (rc == PAMHD_OK) rc = build_work(*b, best_planes);
	if (rc == PAMHD_OK) {
		rc = check(cudaMemcpyAsync(b->state[0], backup, size_t(b->total) * sizeof(double), cudaMemcpyDeviceToDevice,
		                           b->stream));
	}
	b->cur = 0;
	if (rc == PAMHD_OK) rc = reset_run_state(*b);
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(backup);
	if (tile_rows_chosen != nullptr) *tile_rows_chosen = best_ty;
	if (planes_chosen != nullptr) *planes_chosen = best_planes;
	return rc;
}

int pamhd_gpu_batch_tiling(pamhd_batch* b, int32_t* tile_rows, int32_t* planes, int32_t* grid)
{
	if (b == nullptr) return PAMHD_ERR_ARGUMENT;
	if (tile_rows != nullptr) *tile_rows = b->ty;
	if (planes != nullptr) *planes = b->planes_per_item;
	if (grid != nullptr) *grid = b->grid;
	return PAMHD_OK;
}

int pamhd_gpu_batch_sync(pamhd_batch* b)
{
	if (b == nullptr) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(b->device)));
	std::vector<Status> s(b->nboxes);
	PAMHD_TRY(check(cudaMemcpyAsync(s.data(), b->status, s.size() * sizeof(Status), cudaMemcpyDeviceToHost,
	                                b->stream)));
	PAMHD_TRY(check(cudaStreamSynchronize(b->stream)));
	for (const auto& x: s) {
		if (x.flags & PAMHD_FLAG_TIMEOUT) return PAMHD_ERR_TIMEOUT;
	}
	for (const auto& x: s) {
		if (x.flags != 0) return PAMHD_ERR_PHYSICS;
	}
	return PAMHD_OK;
}

int pamhd_gpu_batch_get_stream(pamhd_batch* b, void** stream)
{
	if (b == nullptr or stream == nullptr) return PAMHD_ERR_ARGUMENT;
	*stream = static_cast<void*>(b->stream);
	return PAMHD_OK;
}

int pamhd_gpu_batch_time(pamhd_batch* b, const int32_t box, double* time, int64_t* steps, double* last_dt)
{
	PAMHD_TRY(box_ok(b, box));
	PAMHD_TRY(check(cudaSetDevice(b->device)));
	Clock c;
	PAMHD_TRY(check(cudaMemcpyAsync(&c, b->clock + 3 * box + b->steps % 3, sizeof c, cudaMemcpyDeviceToHost,
	                                b->stream)));
	PAMHD_TRY(check(cudaStreamSynchronize(b->stream)));
	if (time != nullptr) *time = c.t;
	if (steps != nullptr) *steps = c.steps;
	if (last_dt != nullptr) *last_dt = c.dt;
	return PAMHD_OK;
}

int pamhd_gpu_batch_dt_history(pamhd_batch* b, const int32_t box, double* dt, const int32_t count, int32_t* written)
{
	PAMHD_TRY(box_ok(b, box));
	if (dt == nullptr or count < 0) return PAMHD_ERR_ARGUMENT;
	PAMHD_TRY(check(cudaSetDevice(b->device)));
	std::vector<double> all(b->hist_len);
	PAMHD_TRY(check(cudaMemcpyAsync(all.data(), b->dt_hist + (long long)b->hist_len * box,
	                                b->hist_len * sizeof(double), cudaMemcpyDeviceToHost, b->stream)));
	// the steps the box took (a box that stopped at a failure holds its count)
	Clock c;
	PAMHD_TRY(check(cudaMemcpyAsync(&c, b->clock + 3 * box + b->steps % 3, sizeof c, cudaMemcpyDeviceToHost,
	                                b->stream)));
	PAMHD_TRY(check(cudaStreamSynchronize(b->stream)));
	const long long n = std::min<long long>(std::min<long long>(c.steps, b->hist_len), count);
	for (long long i = 0; i < n; i++) dt[i] = all[(c.steps - n + i) % b->hist_len];
	if (written != nullptr) *written = int32_t(n);
	return PAMHD_OK;
}

int pamhd_gpu_batch_status(pamhd_batch* b, const int32_t box, uint32_t* flags, int32_t cell[3], int32_t* dir)
{
	PAMHD_TRY(box_ok(b, box));
	PAMHD_TRY(check(cudaSetDevice(b->device)));
	Status s;
	PAMHD_TRY(check(cudaMemcpyAsync(&s, b->status + box, sizeof s, cudaMemcpyDeviceToHost, b->stream)));
	PAMHD_TRY(check(cudaStreamSynchronize(b->stream)));
	if (flags != nullptr) *flags = s.flags;
	int32_t c[3] = {0, 0, 0};
	int32_t d = 0;
	if (s.flags != 0 and s.first != ~0ull) {
		const Step_Params& P = b->params[0][box];
		const unsigned long long key = s.first >> 8;
		d = int32_t(key & 3ull);
		unsigned long long lin = key >> 2;
		const unsigned long long nx = P.L.n[0] + 2 * P.ext[0], ny = P.L.n[1] + 2 * P.ext[1];
		c[0] = int32_t(lin % nx) - P.ext[0];
		lin /= nx;
		c[1] = int32_t(lin % ny) - P.ext[1];
		c[2] = int32_t(lin / ny) - P.ext[2];
	}
	// in the caller's axes
	if (cell != nullptr) {
		for (int a = 0; a < 3; a++) cell[b->map.perm[a]] = c[a];
	}
	if (dir != nullptr) *dir = d > 0 ? b->map.perm[d - 1] + 1 : 0;
	return PAMHD_OK;
}

} // extern "C"
