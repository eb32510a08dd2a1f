/*
The single-grid context behind pamhd_ctx (include/pamhd_gpu.h), shared by
the entry points of context.cu and the adjoint driver of adjoint.cu.
*/
#ifndef PAMHD_B200_CONTEXT_CUH
#define PAMHD_B200_CONTEXT_CUH

#include <cuda_runtime.h>

#include <vector>

#include "grid_setup.cuh"
#include "step.cuh"

using namespace pamhd_b200;

struct Adjoint_Work;

struct pamhd_ctx {
	pamhd_cfg cfg;        // the internal configuration (axes relabelled, see Axis_Map)
	Axis_Map map{{0, 1, 2}};
	int device = 0;
	cudaStream_t stream = nullptr;
	Layout L;
	Step_Params base;
	double* state[2] = {nullptr, nullptr};
	int cur = 0;
	Speed_Max* red = nullptr;
	Clock* clock = nullptr;
	Status* status = nullptr;
	Control* control = nullptr;
	double* dt_hist = nullptr;
	int hist_len = 1 << 16;
	long long steps = 0;
	int half = 0;         // 1 between the two parts of a step split by pamhd_gpu_step_part
	double control_max_dt = -2.0, control_t_end = -2.0;  // the device Control last written
	double* staging = nullptr;
	double* partial = nullptr;
	int partial_blocks = 296;
	bool needs_boundary_speeds = false;
	cudaGraphExec_t graph = nullptr;
	bool loaded = false;
	Adjoint_Work* adjoint = nullptr;  // adjoint workspace, kept between pamhd_gpu_adjoint calls
	// time-stamped inflow of VALUE sides: host copies and the device tables (times, then states)
	std::vector<double> inflow_times[3][2], inflow_states[3][2];
	double* inflow_dev[3][2] = {{nullptr, nullptr}, {nullptr, nullptr}, {nullptr, nullptr}};
	Inflow_Table* inflow_tables = nullptr;  // [3][2] in device memory, pointed to by the step parameters
};

namespace pamhd_b200 {
// the next step of a context (launch only; advances the step counter and parity)
int context_issue_step(pamhd_ctx& x);
// frees the adjoint workspace of a context (adjoint.cu)
void release_adjoint(pamhd_ctx& x);
}

#endif
