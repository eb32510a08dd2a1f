/*
Device-side data structures of the fused MHD step, shared by the kernels
(step_kernels.cu) and the host context (context.cu).
*/
#ifndef PAMHD_B200_STEP_CUH
#define PAMHD_B200_STEP_CUH

#include <cstdint>

#include "mhd_device.cuh"

namespace pamhd_b200 {

/*
Layout of one state copy in HBM: eight FP64 arrays (rho, mom xyz, E,
B xyz), each a padded 3-D block with one ghost layer on every active
dimension.  Rows are padded so that the first interior cell of every row
sits on a 32-byte boundary (a full DRAM sector); periodic dimensions have
ghosts too, refreshed by the step kernel itself.
*/
struct Layout {
	int n[3];        // interior cells
	int g[3];        // ghost width (1 on active dimensions, else 0)
	int xoff;        // column of interior x = 0
	int pitch;       // doubles per row
	int rows;        // rows per plane: n[1] + 2 g[1]
	int planes;      // n[2] + 2 g[2]
	long long plane; // doubles per plane
	long long var;   // doubles per variable array

	__host__ __device__ long long offset(const int i, const int j, const int k) const
	{
		return (long long)(k + g[2]) * plane + (long long)(j + g[1]) * pitch + (i + xoff);
	}
};

// per-step reduction of face signal speeds (bit patterns of non-negative doubles)
struct Speed_Max {
	unsigned long long smax[3];
	unsigned int zero;   // some face had speed <= 0 (or no reduction yet)
	unsigned int pad;
};

// simulation clock, one slot per step phase
struct Clock {
	double t;
	double dt;
	long long steps;
	double pad;
};

// error state: OR of flags and the first failing face ((key << 8) | flag)
struct Status {
	unsigned int flags;
	unsigned int fail_step;        // the cell-centred steps: 1 + the clock's step count of the failing step (0: none)
	unsigned long long first;
};

// limits read by the step kernel from device memory (so graphs need no re-capture)
struct Control {
	double max_dt;   // >= 0: cap of dt; < 0: cap is t_end - t
	double t_end;
};

/*
Time-stamped inflow of a VALUE side (the solar-wind boundary of
mhd/solar_wind_box.hpp:227-268): states[i] (8 conservative values) holds
while i of the count timestamps are <= the simulation time.  Device
memory; states == nullptr: the side keeps its constant ghost values.
*/
struct Inflow_Table {
	const double* times;
	const double* states;   // (count + 1) x 8
	int count;
};

/*
Scheduler state of the persistent batched run: the next (step, work item)
to hand out, and an error word set by a block whose bounded wait ran out.
*/
struct Run_Sync {
	unsigned int next;
	unsigned int error;
	unsigned int pad[2];
};

struct Step_Params {
	const double* __restrict__ in;
	double* __restrict__ out;
	Layout L;
	Gas gas;
	double len[3];
	double inv_len[3];
	double cfl;
	int active[3];
	int periodic[3];
	int bc_lo[3];
	int bc_hi[3];
	int ext[3];          // ghost extent of the failure numbering (1 on non-periodic active dims)
	Speed_Max* red;      // [3], ring by step phase
	Clock* clock;        // [3]
	Status* status;
	const Control* control;
	double* dt_hist;
	int hist_len;
	int phase;           // step index mod 3
	int kchunk;          // z planes per block
	double forced_dt;    // >= 0: the step's dt (a prescribed schedule); < 0: the CFL rule
	int kpart;           // z planes a launch computes: 0 all, 1 the first and last only, 2 the others
	const Inflow_Table* inflow;  // [3][2] by dimension and side (lo, hi) in device memory, or nullptr
};

// launchers (step_kernels.cu)
int launch_step(const Step_Params& P, int solver, cudaStream_t stream);
int launch_boundary_speeds(const Step_Params& P, int solver, cudaStream_t stream);
int launch_scatter(const double* packed, double* var_base, const Layout& L, cudaStream_t stream);
int launch_gather(const double* var_base, double* packed, const Layout& L, cudaStream_t stream);
int launch_fill_ghosts_values(const Step_Params& P, double* state, const double lo[3][8], const double hi[3][8],
                              cudaStream_t stream);
int prepare_step_kernels(int solver, bool y_active);
int launch_face_flux(int solver, long long n, const double* neg, const double* pos, const double* bg,
                     const Gas& gas, double* flux, double* speed, uint32_t* flags, cudaStream_t stream);
int launch_totals(const double* state, const Layout& L, double volume, double* partial, int nblocks,
                  cudaStream_t stream);
int step_tile_rows(int solver);
int batch_tile_rows();
int prepare_batch_kernels(int solver, int tile_rows);
int batch_blocks_per_sm(int solver, int tile_rows, int* blocks);
int launch_batch_step(const Step_Params* boxes, const int4* items, int nitems, int phase, int grid, int solver,
                      int tile_rows, cudaStream_t stream);
int launch_batch_boundary_speeds(const Step_Params* boxes, int nboxes, int largest, int phase, int solver,
                                 cudaStream_t stream);
// the persistent batched run: nsteps steps of every box in one cooperative launch (see batch_run_kernel)
int prepare_batch_run_kernels(int solver, int tile_rows);
int batch_run_blocks_per_sm(int solver, int tile_rows, int* blocks);
int launch_batch_run(const Step_Params* boxes_even, const Step_Params* boxes_odd, const int4* items, int nitems,
                     const int* box_items, unsigned int* done, int nboxes, long long step0, int nsteps,
                     Run_Sync* sync, long long wait_limit, int grid, int solver, int tile_rows, cudaStream_t stream);
constexpr int BOUNDARY_CHUNK = 4096;  // ghost-ghost faces per boundary work item of the persistent run

} // namespace pamhd_b200

#endif
