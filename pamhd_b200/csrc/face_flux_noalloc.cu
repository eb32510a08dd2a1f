/*
pamhd_gpu_face_flux_noalloc: the solver-level entry point
pamhd_gpu_face_flux without any device memory allocation.

pamhd_gpu_face_flux stages its host arrays through six device buffers that
it allocates and frees on every call.  This variant stages them through one
fixed scratch area, a file-scope __device__ array of
PAMHD_NOALLOC_MAX_FACES faces (3.56 MiB), whose address is looked up once
per device (and kept for the life of the process: a cudaDeviceReset between
calls is not supported, since the driver may place the array elsewhere when
it reloads the module).  The caller's current device is restored on every
return.  It is for callers that cannot allocate device memory between
set-up and tear-down: a process whose device memory is reserved by another
allocator, or a loop that cannot accept the device-wide synchronisation of
cudaMalloc / cudaFree.

Scratch layout (byte offsets, each a multiple of 256):
  neg   MAX * 8 doubles    pos   MAX * 8 doubles    flux  MAX * 8 doubles
  bg    MAX * 3 doubles    speed MAX doubles        flags MAX uint32
Nothing in it has to start at zero: the kernel writes every flux, speed and
flag slot of the n faces of a call, and only those slots are read back.
*/
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "step.cuh"

using namespace pamhd_b200;

namespace {

constexpr long long MAX_FACES = PAMHD_NOALLOC_MAX_FACES;
constexpr size_t NEG_AT = 0;
constexpr size_t POS_AT = NEG_AT + size_t(MAX_FACES) * 8 * sizeof(double);
constexpr size_t FLUX_AT = POS_AT + size_t(MAX_FACES) * 8 * sizeof(double);
constexpr size_t BG_AT = FLUX_AT + size_t(MAX_FACES) * 8 * sizeof(double);
constexpr size_t SPEED_AT = BG_AT + size_t(MAX_FACES) * 3 * sizeof(double);
constexpr size_t FLAGS_AT = SPEED_AT + size_t(MAX_FACES) * sizeof(double);
constexpr size_t SCRATCH_BYTES = FLAGS_AT + size_t(MAX_FACES) * sizeof(uint32_t);
static_assert(POS_AT % 256 == 0 and FLUX_AT % 256 == 0 and BG_AT % 256 == 0 and SPEED_AT % 256 == 0
              and FLAGS_AT % 256 == 0, "scratch sections must stay 256-byte aligned");

static __device__ __align__(256) unsigned char face_scratch[SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex scratch_lock;
unsigned char* scratch_of[MAX_DEVICES] = {};

int check(const cudaError_t e)
{
	return e == cudaSuccess ? PAMHD_OK : PAMHD_ERR_CUDA;
}

// makes `device` current for the life of the guard, then restores the caller's current device
struct Device_Guard {
	int previous = -1;
	int rc = PAMHD_OK;
	explicit Device_Guard(const int device)
	{
		rc = check(cudaGetDevice(&previous));
		if (rc == PAMHD_OK) rc = check(cudaSetDevice(device));
	}
	~Device_Guard()
	{
		if (previous >= 0) cudaSetDevice(previous);
	}
};

// address of this device's scratch; the device must be current
int scratch_address(const int device, unsigned char** out)
{
	const std::lock_guard<std::mutex> hold(scratch_lock);
	if (scratch_of[device] == nullptr) {
		void* p = nullptr;
		const int rc = check(cudaGetSymbolAddress(&p, face_scratch));
		if (rc != PAMHD_OK) return rc;
		scratch_of[device] = static_cast<unsigned char*>(p);
	}
	*out = scratch_of[device];
	return PAMHD_OK;
}

} // namespace

extern "C" {

int pamhd_gpu_face_flux_noalloc(const int32_t device, const int32_t solver, const int64_t n, const double* neg,
                                const double* pos, const double* bg, const double adiabatic_index,
                                const double vacuum_permeability, double* flux, double* speed, uint32_t* flags)
{
	if (n < 0 or neg == nullptr or pos == nullptr or flux == nullptr or speed == nullptr or flags == nullptr) {
		return PAMHD_ERR_ARGUMENT;
	}
	if (n > MAX_FACES) return PAMHD_ERR_TOO_LARGE;
	if (solver != PAMHD_RUSANOV and solver != PAMHD_HLL_ATHENA and solver != PAMHD_HLLD_ATHENA
		and solver != PAMHD_ROE_ATHENA) {
		return PAMHD_ERR_ARGUMENT;
	}
	if (not (adiabatic_index > 1.0) or not (vacuum_permeability > 0.0)) return PAMHD_ERR_ARGUMENT;
	if (n == 0) return PAMHD_OK;
	// the same code as pamhd_gpu_face_flux for a device that does not exist (the failed
	// cudaSetDevice), then the limit of the per-device address table
	const Device_Guard on(device);
	if (on.rc != PAMHD_OK) return on.rc;
	if (device >= MAX_DEVICES) return PAMHD_ERR_ARGUMENT;
	int rc = PAMHD_OK;
	unsigned char* s = nullptr;
	rc = scratch_address(device, &s);
	if (rc != PAMHD_OK) return rc;
	double* dn = reinterpret_cast<double*>(s + NEG_AT);
	double* dp = reinterpret_cast<double*>(s + POS_AT);
	double* df = reinterpret_cast<double*>(s + FLUX_AT);
	double* db = bg == nullptr ? nullptr : reinterpret_cast<double*>(s + BG_AT);
	double* ds = reinterpret_cast<double*>(s + SPEED_AT);
	uint32_t* dg = reinterpret_cast<uint32_t*>(s + FLAGS_AT);

	Gas g;
	g.gamma = adiabatic_index;
	g.mu0 = vacuum_permeability;
	g.inv_mu0 = 1.0 / vacuum_permeability;
	g.sqrt_mu0 = std::sqrt(vacuum_permeability);
	g.inv_sqrt_mu0 = 1.0 / g.sqrt_mu0;
	const size_t s8 = size_t(n) * 8 * sizeof(double);
	rc = check(cudaMemcpy(dn, neg, s8, cudaMemcpyHostToDevice));
	if (rc == PAMHD_OK) rc = check(cudaMemcpy(dp, pos, s8, cudaMemcpyHostToDevice));
	if (rc == PAMHD_OK and bg != nullptr) {
		rc = check(cudaMemcpy(db, bg, size_t(n) * 3 * sizeof(double), cudaMemcpyHostToDevice));
	}
	if (rc == PAMHD_OK) rc = launch_face_flux(solver, n, dn, dp, db, g, df, ds, dg, nullptr);
	if (rc == PAMHD_OK) rc = check(cudaMemcpy(flux, df, s8, cudaMemcpyDeviceToHost));
	if (rc == PAMHD_OK) rc = check(cudaMemcpy(speed, ds, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost));
	if (rc == PAMHD_OK) rc = check(cudaMemcpy(flags, dg, size_t(n) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
	if (rc != PAMHD_OK) return rc;
	for (int64_t i = 0; i < n; i++) {
		if (flags[i] != 0) return PAMHD_ERR_PHYSICS;
	}
	return PAMHD_OK;
}

} // extern "C"
