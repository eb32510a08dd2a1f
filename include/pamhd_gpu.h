/*
pamhd_gpu.h - C ABI of the B200 (sm_100a) finite-volume MHD step.

This is the drop-in boundary for PAMHD's cell-centred ("Mode C") MHD step
on uniform Cartesian grids: the conservative state (mass density, momentum
density, total energy density, magnetic field), the Rusanov / HLL / HLLD /
Roe face fluxes, flux application and the lagged CFL timestep rule; and for
its staggered-field step (face magnetic field by constrained transport,
pamhd_gpu_staggered_*) on uniform grids, periodic or bounded.
Host code (C or C++) calls these entry points with plain pointers and
sizes; no C++ types, exceptions or torch types cross this boundary.

Conventions
  - Every function returns an int status: PAMHD_OK (0) or a PAMHD_ERR_*.
  - Arrays of cell data are structure-of-arrays: eight arrays, one per
    conservative variable in the order of the reference's detail::MHD
    (mhd/variables.hpp:240): rho, mom_x, mom_y, mom_z, E, B_x, B_y, B_z.
    Each holds n[0]*n[1]*n[2] doubles, x fastest (index i + n0*(j + n1*k)),
    the order of dccrg's level-0 cell ids on a uniform grid.
  - Host arrays passed in are caller-owned and copied; device arrays are
    owned by the context.
  - A context is bound to one CUDA device and one CUDA stream and is not
    thread-safe; different contexts may be used from different threads.
  - All arithmetic is IEEE FP64.
*/
#ifndef PAMHD_GPU_H
#define PAMHD_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PAMHD_GPU_ABI_VERSION 2

/* Return codes. */
enum {
	PAMHD_OK = 0,
	PAMHD_ERR_ARGUMENT = 1,  /* invalid argument or configuration */
	PAMHD_ERR_CUDA = 2,      /* a CUDA runtime call failed */
	PAMHD_ERR_PHYSICS = 3,   /* a solver met a state the reference throws on
	                            (see pamhd_gpu_status for which and where) */
	PAMHD_ERR_STATE = 4,     /* call made in the wrong order */
	PAMHD_ERR_TIMEOUT = 5,   /* a bounded device-side wait gave up */
	PAMHD_ERR_TOO_LARGE = 6, /* request larger than the fixed scratch of a
	                            no-alloc entry point (split it) */
	PAMHD_ERR_IO = 7         /* a file could not be opened, read or written */
};

/*
Riemann solver ids, in the numeric order of the reference's
enum class Solver (mhd/common.hpp:54-61).  rusanov_staggered is accepted by
the reference's option parser but aborts in its dispatcher
(mhd/solve.hpp:150-153); here it is rejected with PAMHD_ERR_ARGUMENT.
*/
enum {
	PAMHD_RUSANOV = 0,
	PAMHD_RUSANOV_STAGGERED = 1,
	PAMHD_HLL_ATHENA = 2,
	PAMHD_HLLD_ATHENA = 3,
	PAMHD_ROE_ATHENA = 4
};

/*
Boundary kinds per grid side.  PERIODIC must be given on both sides of a
dimension.  COPY fills a ghost from its inward face neighbour (density,
velocity, thermal pressure and magnetic field copied; mhd/boundaries.hpp:
818-1030).  VALUE holds a fixed conservative state (value boundaries,
mhd/boundaries.hpp:760-880, and the solar-wind inflow of
mhd/solar_wind_box.hpp:227).
*/
enum {
	PAMHD_BC_PERIODIC = 0,
	PAMHD_BC_COPY = 1,
	PAMHD_BC_VALUE = 2,
	PAMHD_BC_EXTERNAL = 3    /* z sides only: the ghost plane belongs to a neighbouring
	                            slab and is written by the caller (halo exchange, see
	                            pamhd_gpu_halo); the step never writes it */
};

/*
Status flag bits reported by pamhd_gpu_status() and by
pamhd_gpu_face_flux().  Each matches a std::domain_error the reference
throws (and then aborts on, mhd/solve.hpp:156-181).
*/
enum {
	PAMHD_FLAG_DENSITY = 1u << 0,        /* non-positive or non-normal mass density */
	PAMHD_FLAG_PRESSURE = 1u << 1,       /* non-positive or non-normal thermal pressure */
	PAMHD_FLAG_WAVE_SPEED = 1u << 2,     /* invalid fast magnetosonic / signal speed */
	PAMHD_FLAG_FLUX = 1u << 3,           /* non-finite flux or momentum */
	PAMHD_FLAG_ROE_DENSITY = 1u << 4,    /* roe_athena.hpp:505: intermediate density */
	PAMHD_FLAG_ROE_PRESSURE = 1u << 5,   /* roe_athena.hpp:523: intermediate pressure */
	PAMHD_FLAG_NEW_STATE = 1u << 6,      /* common.hpp:728-742: updated state invalid */
	PAMHD_FLAG_TIMEOUT = 1u << 7         /* a bounded device wait expired */
};

/*
Grid configuration.  Replaces the parts of the reference's JSON options
that the step reads: the solver (mhd/options.hpp:97-112), the timestep
factor (mhd/options.hpp:119-132, "mhd-time-step-factor"), the adiabatic
index and vacuum permeability (simulation_options.hpp:59-60), the uniform
cell size (grid/options.hpp) and the boundary kinds.
A dimension with n == 1 is inactive: it has no faces and does not enter
the timestep.  Any set of active dimensions is accepted (grids that are
not x, x-y or x-y-z run with their axes relabelled internally; every array,
side, state, status and gradient of this ABI stays in the caller's axes).
*/
typedef struct pamhd_cfg {
	int32_t n[3];                /* interior cells in x, y, z */
	int32_t solver;              /* PAMHD_RUSANOV ... PAMHD_ROE_ATHENA */
	double cell_length[3];       /* dx, dy, dz */
	double adiabatic_index;      /* gamma */
	double vacuum_permeability;  /* mu0 */
	double time_step_factor;     /* CFL number */
	int32_t bc_lo[3];            /* PAMHD_BC_* of the -x, -y, -z sides */
	int32_t bc_hi[3];            /* PAMHD_BC_* of the +x, +y, +z sides */
	double value_lo[3][8];       /* ghost state of VALUE sides (rho, mom, E, B) */
	double value_hi[3][8];
	int32_t device;              /* CUDA device ordinal */
	int32_t reserved;            /* must be 0 */
} pamhd_cfg;

typedef struct pamhd_ctx pamhd_ctx;

/* ABI version of the loaded library (PAMHD_GPU_ABI_VERSION). */
int pamhd_gpu_abi_version(void);

/* Text of a return code. */
const char* pamhd_gpu_errstr(int code);

/*
Creates a context: allocates the state (two copies, ping-pong) and the
reduction buffers on cfg->device.  Replaces the dccrg grid set-up and the
cell-data allocation of tests/mhd/test.cpp:330-444 for uniform grids.
Launch limits (PAMHD_ERR_ARGUMENT beyond them): at most 524,280 cells
along the second active dimension (262,140 with Roe) and 1,048,560 along
the third.
*/
int pamhd_gpu_create(const pamhd_cfg* cfg, pamhd_ctx** ctx);

/* Frees everything the context owns. */
int pamhd_gpu_destroy(pamhd_ctx* ctx);

/*
Copies the interior state in from eight host arrays and fills the ghost
cells (apply_boundaries, mhd/boundaries.hpp:1261).  Marks the context as
not primed: the next step is the dt = 0 priming step.
*/
int pamhd_gpu_set_state(pamhd_ctx* ctx, const double* const soa[8]);

/* Copies the interior state out to eight host arrays (synchronises). */
int pamhd_gpu_get_state(pamhd_ctx* ctx, double* const soa[8]);

/* As set/get_state but with device pointers, ordered on the context's stream. */
int pamhd_gpu_set_state_device(pamhd_ctx* ctx, const double* const soa[8]);
int pamhd_gpu_get_state_device(pamhd_ctx* ctx, double* const soa[8]);

/*
One step of the lagged-CFL rule; replaces pamhd::mhd::timestep()
(mhd/solve.hpp:1837-1924) in its Mode C, no-substepping form:
  dt = min over faces of CFL * dx_d / s_face from the previous step's face
  speeds (0 if any face speed <= 0), capped by max_dt
  (substepping.hpp:285-338, solve.hpp:1933-2007);
  fluxes for every face, scaled by dt (solve.hpp:217-392);
  U += (F- - F+)/dx, then y, then z (solve.hpp:1543-1587);
  ghost refresh.
The first step after create/set_state is the reference's dt = 0 priming
step whatever max_dt is (tests/mhd/test.cpp:462-470).
Synchronises; *dt_taken receives the step length.  max_signal (NULL, or
three doubles) receives the largest signal speed of this step's faces
normal to x, y and z (0 for a dimension of one cell): the maxima of the
per-face Max_v the reference's get_fluxes stores (mhd/solve.hpp:319-322)
and its minimize_timestep reads (mhd/solve.hpp:1933-2014), so that a host
caller can apply its own timestep rule: dt = min over dimensions d of
CFL * dx_d / max_signal[d].  Faces between two ghost cells of a
non-periodic side count, as in the reference.
Returns PAMHD_ERR_PHYSICS if any face met an invalid state.  The step in
which a face fails completes (its state is what the faces gave); the grid
then stops, as the reference aborts there (mhd/solve.hpp:156-181): every
later step (pamhd_gpu_step, _steps, _step_part) leaves the state, the time
and the step count as they are (dt 0, max_signal the failing step's) until
set_state.
*/
int pamhd_gpu_step(pamhd_ctx* ctx, double max_dt, double* dt_taken, double* max_signal);

/*
Runs nsteps steps without host synchronisation (captured in a CUDA graph
after the first call), each capped so that simulation time does not pass
t_end, as the loop of tests/mhd/test.cpp:514-530 does.  Primes first if
needed.  Does not wait for the GPU; use pamhd_gpu_sync() and
pamhd_gpu_time() to collect the result.
*/
int pamhd_gpu_steps(pamhd_ctx* ctx, int32_t nsteps, double t_end);

/*
One step in two launches, for a z slab that overlaps its halo exchange with
the step's interior: part 1 computes the new state of the first and last z
planes (and the speeds of ghost-ghost faces), part 2 the planes between them
and ends the step.  Between the two, pamhd_gpu_halo returns the planes of the
state being written, so the caller can send the new cut planes to its
neighbours (and receive theirs into the new ghost planes) while part 2 runs.
Both parts read the same state and fold into the same speed reduction: the
result equals pamhd_gpu_steps(ctx, 1, t_end) bit for bit.  Parts must
alternate, starting with 1; needs active z.  No host synchronisation (the
time cap t_end is written to the device only when it changes).  The
reference overlaps its remote-neighbour update with the inner cells the same
way (mhd/solve.hpp:1767-1802).
*/
int pamhd_gpu_step_part(pamhd_ctx* ctx, int32_t part, double t_end);

/*
The CUDA stream (a cudaStream_t) every kernel of the context runs on, so
that callers can order their own work with it or time it with CUDA events.
No reference counterpart (the reference has no device streams).
*/
int pamhd_gpu_get_stream(pamhd_ctx* ctx, void** stream);

/*
Time-stamped inflow of a VALUE side (dim 0..2, side 0 = low, 1 = high), as
the solar-wind boundary of mhd/solar_wind_box.hpp:227-268: with count
increasing timestamps times[0..count-1] and count + 1 conservative states
states[(count + 1) * 8], the side's ghosts hold states[i] while i of the
timestamps are <= the simulation time.  The step writes them for the time
its new state holds, on the device (no host round trip, graph replay
unchanged); the current state's ghosts take the value of the current time
at once.  Replaces the side's constant value; count = 0 with one state sets
a constant.  Not with pamhd_gpu_adjoint (rejected).
*/
int pamhd_gpu_set_inflow(pamhd_ctx* ctx, int32_t dim, int32_t side, int32_t count, const double* times,
                         const double* states);

/*
Halo planes of a z slab, for the exchange between slabs of one grid split
along z (one slab per GPU; the cut sides are PAMHD_BC_EXTERNAL).  The
dccrg halo update the reference does between steps (mhd/solve.hpp:
1767-1791) becomes: after each step, copy the interior boundary planes of
each slab into its neighbours' ghost planes.
side: 0 = low z, 1 = high z; ghost: 0 = the interior plane next to that
side (to send), 1 = the ghost plane of that side (to receive).
planes[v] receives the device address of variable v's plane in the
current state (between the parts of a step split by pamhd_gpu_step_part:
the state that step writes), *count the plane's length in doubles (padded
rows; a plane of one variable is contiguous).  The addresses alternate
between two buffers from step to step: ask again after every step.
*/
int pamhd_gpu_halo(pamhd_ctx* ctx, int32_t side, int32_t ghost, double* planes[8], int64_t* count);

/*
Device address of the speed reduction the next step takes its dt from:
four 64-bit words, the per-axis maxima of face speed / cell length as the
bits of non-negative doubles (so an integer max over slabs is the max of
the doubles) and a flag word (non-zero if any face speed was <= 0).  Slabs
of one grid combine it by an element-wise max over all slabs before the
next step, so that every slab takes the grid's dt
(mhd/solve.hpp:1933-2014 takes the minimum over all cells of all ranks).
*/
int pamhd_gpu_speed_slot(pamhd_ctx* ctx, void** slot);

/* Waits for the context's stream; returns PAMHD_ERR_PHYSICS if a face failed. */
int pamhd_gpu_sync(pamhd_ctx* ctx);

/* Simulation time, number of steps taken and the last dt (synchronises). */
int pamhd_gpu_time(pamhd_ctx* ctx, double* time, int64_t* steps, double* last_dt);

/*
Copies the dt of the last min(count, recorded) steps (oldest first) out
(synchronises); *written receives how many.
*/
int pamhd_gpu_dt_history(pamhd_ctx* ctx, double* dt, int32_t count, int32_t* written);

/*
Error state of the context: OR of PAMHD_FLAG_* seen since the last
set_state, and the first failing face in x-fastest cell order:
cell index (interior numbering, ghosts as -1/n) and face direction
(+1, +2, +3) — the face at which the reference would have aborted
(mhd/solve.hpp:156-181).
*/
int pamhd_gpu_status(pamhd_ctx* ctx, uint32_t* flags, int32_t cell[3], int32_t* dir);

/*
Conserved totals over interior cells: sum of rho, mom[3], E, B[3] times the
cell volume, summed in a fixed order (deterministic).
*/
int pamhd_gpu_totals(pamhd_ctx* ctx, double totals[8]);

/*
Solver-level entry point: the face flux and max signal speed of n
independent face problems, each given as the two states in the face frame
(x = face normal) and the face's background field.  Replaces the compile
time plugin get_flux_X<Mas, Mom, Nrj, Mag>(state_neg, state_pos, bg_face_B,
gamma, mu0) -> tuple<MHD, Scalar> of mhd/rusanov.hpp:67,
mhd/hll_athena.hpp:65, mhd/hlld_athena.hpp:62 and mhd/roe_athena.hpp:575.
Host arrays: neg, pos and flux hold n*8 doubles (cell-major), bg n*3 (NULL
means zero), speed n, flags n (0 or PAMHD_FLAG_* of the first check that
failed).  Runs on `device`; returns PAMHD_ERR_PHYSICS if any face failed.
*/
int pamhd_gpu_face_flux(
	int32_t device, int32_t solver, int64_t n,
	const double* neg, const double* pos, const double* bg,
	double adiabatic_index, double vacuum_permeability,
	double* flux, double* speed, uint32_t* flags);

/* Most faces one pamhd_gpu_face_flux_noalloc call takes. */
#define PAMHD_NOALLOC_MAX_FACES 16384

/*
pamhd_gpu_face_flux without device memory allocation.  No reference
counterpart: the reference evaluates its solvers on the host.  Same
arguments and results as pamhd_gpu_face_flux, for callers that cannot
allocate device memory once set up (device memory reserved by another
allocator, or a loop that cannot take the device-wide synchronisation of
cudaMalloc / cudaFree).  Faces are staged through a fixed 3.56 MiB scratch
area of this library's device code instead of per-call buffers, so:
  - n > PAMHD_NOALLOC_MAX_FACES is rejected with PAMHD_ERR_TOO_LARGE
    before any CUDA call: split the faces into calls of at most that many;
  - all calls on one device share the scratch, so calls that overlap in
    time (from several host threads) race: serialise them;
  - the first call on a device does the set-up (loads this scratch, which
    the CUDA driver places when it loads the library's device code, and
    looks up its address): make it before any stream capture;
  - the address is kept for the life of the process: a cudaDeviceReset
    between calls is not supported;
  - devices 0..63 only (PAMHD_ERR_ARGUMENT for a higher ordinal that
    exists; a device that does not exist gives PAMHD_ERR_CUDA, as
    pamhd_gpu_face_flux does); n = 0 returns PAMHD_OK before any CUDA call.
Runs on the legacy default stream of `device`, synchronously, and restores
the caller's current device before it returns.
*/
int pamhd_gpu_face_flux_noalloc(
	int32_t device, int32_t solver, int64_t n,
	const double* neg, const double* pos, const double* bg,
	double adiabatic_index, double vacuum_permeability,
	double* flux, double* speed, uint32_t* flags);

/*
nsteps steps with the given dt each (host array), instead of the CFL rule:
the forward map the adjoint linearises, for perturbed runs on a frozen dt
schedule.  No reference counterpart (the reference always takes the CFL
dt, mhd/solve.hpp:1870-1877).
*/
int pamhd_gpu_steps_dt(pamhd_ctx* ctx, int32_t nsteps, const double* dt);

/*
Discrete adjoint of nsteps steps from the context's current state U_0:
runs the forward steps (CFL rule, or the dt_in schedule when not NULL),
storing the state every `every` steps, leaves the context at U_N, then
computes grad = (dU_N/dU_0)^T seed by a reverse sweep that recomputes each
segment from its checkpoint, on the forward run's dt schedule held fixed.
seed and grad: eight host arrays each (the layout of set_state).
grad_value (NULL or 48 doubles): the gradient with respect to the state
of each VALUE side, [dimension][lo, hi][8].  dt_out (NULL or nsteps
doubles) receives the schedule.  Solvers: Rusanov, HLL, HLLD, Roe.  The
device memory (ceil(nsteps/every) checkpoints, two buffers of every - 1
recompute states, cotangents) stays with the context after the first call
and is reused by later calls; it grows when a call needs more and is freed
by pamhd_gpu_destroy.  No reference counterpart: the reference has no
derivatives.
*/
int pamhd_gpu_adjoint(pamhd_ctx* ctx, int32_t nsteps, int32_t every, const double* const seed[8],
                      double* const grad[8], double* grad_value, const double* dt_in, double* dt_out);

/*
Batched ensemble: independent uniform boxes of uneven sizes (each its own
pamhd_cfg: cells, cell size, boundary kinds and values) advanced together,
one kernel launch per step for the whole ensemble, each box with its own
CFL timestep and clock.  The reference advances one grid per program
(tests/mhd/test.cpp, tests/mhd/solar_wind_box.cpp); an ensemble there is
one run per box, which pamhd_gpu_create / pamhd_gpu_steps reproduce box
by box.  All boxes use the same solver and the same active dimensions.
*/
typedef struct pamhd_batch pamhd_batch;

int pamhd_gpu_batch_create(int32_t device, int32_t nboxes, const pamhd_cfg* cfgs, pamhd_batch** batch);
int pamhd_gpu_batch_destroy(pamhd_batch* batch);

/*
Copies the interior state of one box in from host arrays and fills its
ghosts.  Any set_state restarts the whole ensemble's step count: the next
step is a dt = 0 priming step for every box.
*/
int pamhd_gpu_batch_set_state(pamhd_batch* batch, int32_t box, const double* const soa[8]);
int pamhd_gpu_batch_get_state(pamhd_batch* batch, int32_t box, double* const soa[8]);

/*
nsteps steps of every box, each capped so that its time does not pass t_end;
no host sync.  A box in which a face failed stops after that step (its state,
time and step count stay as they are, as pamhd_gpu_step describes) while the
other boxes go on.
*/
int pamhd_gpu_batch_steps(pamhd_batch* batch, int32_t nsteps, double t_end);

/*
nsteps steps of every box in ONE persistent kernel launch (the time loop of
each box, tests/mhd/solar_wind_box.cpp:466-527, for the whole ensemble):
a cooperative launch of the SMs' resident capacity hands out the (step,
work item) pairs in order (a box's tiles, and chunks of the ghost-ghost
faces whose speeds enter its timestep); an item of step s of a box waits
until the box's items of step s - 1 are done, so each box advances at its
own pace with its own lagged CFL dt from its own reduction ring, capped so
that its time does not pass t_end.  The launch is captured in a CUDA graph
and replayed (captured again for another nsteps, state parity or step
phase).  Each wait is bounded (pamhd_gpu_batch_set_wait_limit polls, about
a second by default): when one runs out, the launch winds down, every box's
status gets PAMHD_FLAG_TIMEOUT and pamhd_gpu_batch_sync returns
PAMHD_ERR_TIMEOUT; the state is then mid-step (set it again).  Results
equal pamhd_gpu_batch_steps bit for bit.  Does not wait for the GPU.
*/
int pamhd_gpu_batch_run(pamhd_batch* batch, int32_t nsteps, double t_end);

/* Polls a wait of pamhd_gpu_batch_run makes before it gives up (>= 0; 0: no wait at all). */
int pamhd_gpu_batch_set_wait_limit(pamhd_batch* batch, int64_t polls);

/*
The persistent run's launch: blocks (the resident capacity for the current
tiling), work items per step, and whether the last run was replayed from a
CUDA graph (1) or launched directly (0).
*/
int pamhd_gpu_batch_run_info(pamhd_batch* batch, int32_t* grid, int32_t* items, int32_t* graphed);

/*
Autotuner of the persistent run: times trial_steps steps of the loaded
ensemble for each tile shape (32 x 4, 32 x 8) and z planes per work item
(8, 16, 32, 64), keeps the fastest and restores the state it started from.
*/
int pamhd_gpu_batch_tune_run(pamhd_batch* batch, int32_t trial_steps, int32_t* tile_rows, int32_t* planes);

/*
Autotuner: times trial_steps steps of the loaded ensemble for each
candidate tile shape (32 x 4 or 32 x 8 cells per block, 32 x 1 when y is
inactive), number of z planes per work item (8, 16, 32, 64) and resident
grid size (one wave, two waves, one block per item), keeps the fastest and
restores the state it started from.
*/
int pamhd_gpu_batch_tune(pamhd_batch* batch, int32_t trial_steps, int32_t* planes, int32_t* grid);

/* The work split in use: tile rows (cells per block = 32 x tile_rows), z planes per item, grid. */
int pamhd_gpu_batch_tiling(pamhd_batch* batch, int32_t* tile_rows, int32_t* planes, int32_t* grid);

/* Sets the work split directly (a tiling found by an earlier pamhd_gpu_batch_tune, say). */
int pamhd_gpu_batch_set_tiling(pamhd_batch* batch, int32_t tile_rows, int32_t planes, int32_t grid);

/* Time-stamped inflow of a VALUE side of one box (see pamhd_gpu_set_inflow). */
int pamhd_gpu_batch_set_inflow(pamhd_batch* batch, int32_t box, int32_t dim, int32_t side, int32_t count,
                               const double* times, const double* states);

int pamhd_gpu_batch_sync(pamhd_batch* batch);
int pamhd_gpu_batch_get_stream(pamhd_batch* batch, void** stream);
int pamhd_gpu_batch_time(pamhd_batch* batch, int32_t box, double* time, int64_t* steps, double* last_dt);
int pamhd_gpu_batch_dt_history(pamhd_batch* batch, int32_t box, double* dt, int32_t count, int32_t* written);
int pamhd_gpu_batch_status(pamhd_batch* batch, int32_t box, uint32_t* flags, int32_t cell[3], int32_t* dir);

/*
The reference's MHD output files (.dc, file version 4; written by
mhd/save.hpp:75-375, read by the reference's tests/common.py and its tools
such as tests/mhd/mhd_diff.py), for uniform grids: header, cell id list and
the variable "mhd     " (mass density, momentum density, total energy
density, magnetic field: 8 doubles per cell).  Host only: pair them with
pamhd_gpu_get_state / pamhd_gpu_set_state.
*/
typedef struct pamhd_dc_info {
	uint64_t step;               /* simulation step */
	double time;                 /* simulation time */
	double adiabatic_index;
	double proton_mass;
	double vacuum_permeability;
	int32_t n[3];                /* level-0 cells */
	int32_t periodic[3];
	double start[3];             /* grid start coordinate */
	double cell_length[3];
	uint64_t cells;              /* n[0] * n[1] * n[2] (read only) */
} pamhd_dc_info;

/* Writes a .dc file: soa in the layout of pamhd_gpu_set_state (x fastest). */
int pamhd_dc_write(const char* path, const pamhd_dc_info* info, const double* const soa[8]);

/*
Reads the header of a .dc file.  PAMHD_ERR_ARGUMENT for another file
version or byte order, a refined (non-uniform) grid or a missing cell;
PAMHD_ERR_IO when the file cannot be read.
*/
int pamhd_dc_read_info(const char* path, pamhd_dc_info* info);

/* Reads the "mhd     " variable of a .dc file into eight arrays of info.cells doubles. */
int pamhd_dc_read(const char* path, double* const soa[8]);

/*
Staggered-field step: the reference's timestep() with the normal magnetic
field of every face (Face_B) advanced by constrained transport
(mhd/solve.hpp:1837-1924: get_fluxes with assign_face_dBs_f{x,y,z},
update_mhd_state, update_vol_B with constant thermal pressure before and
after sync_magnetic_field), on a uniform grid.  A periodic dimension of
one cell is its own neighbour, as in the reference's emulated 1-D and 2-D
runs.  Solvers: Rusanov, HLL, HLLD, Roe.

A dimension of two cells or more may be bounded (PAMHD_BC_COPY or
PAMHD_BC_VALUE on both sides, at most one VALUE side in the grid), as the
reference's solar-wind box (tests/mhd/solar_wind_box.cpp:527-553), the
driver of its staggered runs with open sides: a layer of boundary cells
lies outside the walls (faces, edges and vertices of the box alike,
grid/solar_wind_box.hpp:268-376); its faces are solved and enter the
timestep; the step updates interior cells and faces only, a wall face's
two copies meeting about half way in sync_magnetic_field
(common_functions.hpp:216-251); after the step the layer is refilled from
the interior cell each layer cell touches, faces mirrored across the walls
(apply_boundaries_sw_box, mhd/solar_wind_box.hpp:386-537), and the VALUE
plane takes its state with the inner cells' shared faces
(apply_solar_wind_boundaries, :227-306).

  - create: cfg as pamhd_gpu_create, each dimension periodic on both sides
    or on neither (a dimension of one cell periodic), n[1] at most 262140
    (else PAMHD_ERR_ARGUMENT); replaces the state a PAMHD program keeps in
    Mas, Mom, Nrj, Vol_B and Face_B (tests/mhd/test.cpp:422-456).
  - set_state / get_state: cells as pamhd_gpu_set_state (eight arrays, x
    fastest; cells[5..7] is the volume field Vol_B) and faces[d] the normal
    field of every cell's -d face (Face_B(-d); a cell's +d face is the -d
    face of its +d neighbour), x fastest; along a bounded dimension d,
    faces[d] holds n[d] + 1 faces per row, the high wall last.  set_state
    resets the clock and fills the boundary layer; the first step after it
    is the reference's dt = 0 priming step when called with max_dt = 0.
    get_state may be given faces == NULL.
  - set_inflow: time-stamped states of the VALUE side (count timestamps,
    count + 1 states of 8 conservative values, as pamhd_gpu_set_inflow;
    the configured value until then); refills the plane at once.
  - step: one step with dt = min(lagged CFL dt, max_dt) as pamhd_gpu_step;
    PAMHD_ERR_PHYSICS when a face failed (the state is left as it was).
  - steps: nsteps steps launched on the context's stream, each capped by
    t_end - t; steps once t >= t_end leave the state unchanged.  Returns
    at once; sync waits and reports failures.
*/
typedef struct pamhd_stag pamhd_stag;

int pamhd_gpu_staggered_create(const pamhd_cfg* cfg, pamhd_stag** ctx);
int pamhd_gpu_staggered_destroy(pamhd_stag* ctx);
int pamhd_gpu_staggered_set_state(pamhd_stag* ctx, const double* const cells[8], const double* const faces[3]);
int pamhd_gpu_staggered_get_state(pamhd_stag* ctx, double* const cells[8], double* const faces[3]);
int pamhd_gpu_staggered_set_inflow(pamhd_stag* ctx, int32_t dim, int32_t side, int32_t count, const double* times,
                                   const double* states);
/*
Background magnetic field of every face (the reference's Bg_B, mhd/solve.hpp:120-121):
bg[3 d + c][cell] is component c at the cell's -d face; NULL removes it.  Rusanov and HLL
use it in the flux and the fast speeds, HLLD and Roe ignore it (as the reference's solvers,
mhd/hlld_athena.hpp:77).  The cell state and the faces hold the field without it.
Periodic grids only (PAMHD_ERR_ARGUMENT on a bounded one).
*/
int pamhd_gpu_staggered_set_background(pamhd_stag* ctx, const double* const bg[9]);
int pamhd_gpu_staggered_step(pamhd_stag* ctx, double max_dt, double* dt_taken);
int pamhd_gpu_staggered_steps(pamhd_stag* ctx, int32_t nsteps, double t_end);
int pamhd_gpu_staggered_sync(pamhd_stag* ctx);
int pamhd_gpu_staggered_time(pamhd_stag* ctx, double* time, int64_t* steps, double* last_dt);
int pamhd_gpu_staggered_status(pamhd_stag* ctx, uint32_t* flags, int32_t cell[3], int32_t* dir);
int pamhd_gpu_staggered_get_stream(pamhd_stag* ctx, void** stream);

/*
Two-population step: the reference's N_solve + apply_fluxes_N
(mhd/N_solve.hpp:79-587) on a uniform grid periodic in every dimension
(dimensions of one cell have no faces).  Two fluid populations share one
magnetic field; every face is solved for the two cells' total states with
the split solvers get_flux_N_rusanov (mhd/N_rusanov.hpp:61) or
get_flux_N_hll (mhd/N_hll_athena.hpp:47, as the reference computes it,
including its second scaling of the positive side's momentum flux and its
unscaled field flux), the populations taking their mass fractions' share.

  - create: n, cell_length as pamhd_cfg, solver PAMHD_RUSANOV or
    PAMHD_HLL_ATHENA, min_pressure the floor apply_fluxes_N raises the
    total thermal pressure to (mhd/N_solve.hpp:553-583).
  - set_state / get_state: 13 arrays of n0 n1 n2 doubles, x fastest:
    rho1, mom1 xyz, E1, rho2, mom2 xyz, E2, B xyz (each population's energy
    as the reference keeps it; the total state is their sum).
  - step: one N_solve + apply_fluxes_N with the caller's dt;
    *max_dt receives the next step's limit, min over faces of
    d_len / signal speed (what N_solve returns); PAMHD_ERR_PHYSICS when a
    face failed (the state is left as it was).
  - run: nsteps steps on the context's stream with the loop of
    tests/mhd/two_reference.cpp: dt = min(cfl * max_dt, t_end - t), max_dt
    the previous step's limit (0 before the first step); steps once
    t >= t_end leave the state unchanged.  Returns at once; sync waits.
*/
typedef struct pamhd_npop pamhd_npop;

int pamhd_gpu_npop_create(const int32_t n[3], const double cell_length[3], int32_t solver, double gamma, double mu0,
                          double min_pressure, int32_t device, pamhd_npop** ctx);
int pamhd_gpu_npop_destroy(pamhd_npop* ctx);
int pamhd_gpu_npop_set_state(pamhd_npop* ctx, const double* const state[13]);
int pamhd_gpu_npop_get_state(pamhd_npop* ctx, double* const state[13]);
int pamhd_gpu_npop_step(pamhd_npop* ctx, double dt, double* max_dt);
int pamhd_gpu_npop_run(pamhd_npop* ctx, int32_t nsteps, double cfl, double t_end);
int pamhd_gpu_npop_sync(pamhd_npop* ctx);
int pamhd_gpu_npop_time(pamhd_npop* ctx, double* time, int64_t* steps, double* last_dt);
int pamhd_gpu_npop_status(pamhd_npop* ctx, uint32_t* flags, int32_t cell[3], int32_t* dir);
int pamhd_gpu_npop_get_stream(pamhd_npop* ctx, void** stream);

/*
Cell-centred step with local time stepping: the reference's timestep() with
substeps (mhd/solve.hpp:1837-1924, substepping.hpp) on a uniform grid
periodic in every dimension.  Every cell advances with a period of 2^k
substeps of one common substep length; k is bounded by the caller's
per-cell exponents (the reference's "substep-min" and "substep-max"
options evaluated at the cell), by the cell's CFL limit against the
substep and by its neighbours' (at most one above any face or edge
neighbour).  With every exponent 0 this is pamhd_gpu_step's rule.

  - create: cfg as pamhd_gpu_create, every side PAMHD_BC_PERIODIC.
  - set_state / get_state: as pamhd_gpu_set_state; set_state clears the
    face speeds, so the next step is the dt = 0 priming step when called
    with max_dt = 0.
  - set_exponents: n0 n1 n2 int32 minima and maxima, 0 .. 30 (default 0).
  - step: one step capped by max_dt; *dt_taken its length (the substep
    added once per substep), *substeps their number; PAMHD_ERR_PHYSICS
    when a face failed (the step stops at that substep).  Synchronises.
  - periods: the last step's period of every cell.
*/
typedef struct pamhd_sub pamhd_sub;

int pamhd_gpu_substep_create(const pamhd_cfg* cfg, pamhd_sub** ctx);
int pamhd_gpu_substep_destroy(pamhd_sub* ctx);
int pamhd_gpu_substep_set_state(pamhd_sub* ctx, const double* const cells[8]);
int pamhd_gpu_substep_get_state(pamhd_sub* ctx, double* const cells[8]);
int pamhd_gpu_substep_set_exponents(pamhd_sub* ctx, const int32_t* mins, const int32_t* maxs);
int pamhd_gpu_substep_step(pamhd_sub* ctx, double max_dt, double* dt_taken, int32_t* substeps);
int pamhd_gpu_substep_periods(pamhd_sub* ctx, int32_t* periods);
int pamhd_gpu_substep_status(pamhd_sub* ctx, uint32_t* flags, int32_t cell[3], int32_t* dir);

#ifdef __cplusplus
}
#endif

#endif
