/*
Host-side set-up shared by the single-grid context (context.cu) and the
batch (batch.cu): configuration checks, the HBM layout of one grid and the
constant part of its step parameters.
*/
#ifndef PAMHD_B200_GRID_SETUP_CUH
#define PAMHD_B200_GRID_SETUP_CUH

#include <algorithm>
#include <cmath>
#include <cstring>

#include "step.cuh"

#ifndef PAMHD_CHUNK_BLOCKS
#define PAMHD_CHUNK_BLOCKS 4736   // blocks of a step the z chunking aims at: 32 per SM
#endif

namespace pamhd_b200 {

inline int validate(const pamhd_cfg& c)
{
	if (c.reserved != 0) return PAMHD_ERR_ARGUMENT;
	if (c.solver != PAMHD_RUSANOV and c.solver != PAMHD_HLL_ATHENA and c.solver != PAMHD_HLLD_ATHENA
		and c.solver != PAMHD_ROE_ATHENA) {
		return PAMHD_ERR_ARGUMENT;
	}
	for (int d = 0; d < 3; d++) {
		if (c.n[d] < 1) return PAMHD_ERR_ARGUMENT;
		if (not (c.cell_length[d] > 0.0) or not std::isfinite(c.cell_length[d])) return PAMHD_ERR_ARGUMENT;
		for (const int b: {c.bc_lo[d], c.bc_hi[d]}) {
			if (b != PAMHD_BC_PERIODIC and b != PAMHD_BC_COPY and b != PAMHD_BC_VALUE and b != PAMHD_BC_EXTERNAL) {
				return PAMHD_ERR_ARGUMENT;
			}
			// slab cuts: z only, and the slab needs z faces (two planes or more)
			if (b == PAMHD_BC_EXTERNAL and (d != 2 or c.n[2] < 2)) return PAMHD_ERR_ARGUMENT;
		}
		if (c.n[d] > 1 and ((c.bc_lo[d] == PAMHD_BC_PERIODIC) != (c.bc_hi[d] == PAMHD_BC_PERIODIC))) {
			return PAMHD_ERR_ARGUMENT;
		}
	}
	// active dimensions must be x, x-y or x-y-z (other sets are relabelled first, see axis_map)
	if (c.n[0] < 2) return PAMHD_ERR_ARGUMENT;
	if (c.n[1] < 2 and c.n[2] > 1) return PAMHD_ERR_ARGUMENT;
	if (not (c.adiabatic_index > 1.0) or not (c.vacuum_permeability > 0.0) or not (c.time_step_factor > 0.0)) {
		return PAMHD_ERR_ARGUMENT;
	}
	return PAMHD_OK;
}

/*
Axis relabelling.  The step kernels tile along x and march along z, so they
need the active dimensions to be x, x-y or x-y-z.  A grid whose active
dimensions are another set (y, z, y-z or x-z: the reference's 2-D tests
often use a y-z plane) runs with its axes relabelled: internal axis a is
the caller's axis perm[a], vector components (momentum, field) follow
their axes.  With the inactive axes one cell long, the x-fastest order of
the caller's cells is also the internal order, so state arrays only swap
which array holds which component.  y, z and y-z use a rotation of the
axes, whose face frames equal the caller's (the reference's
get_rotated_vector), so every face sees the same numbers; x-z swaps y and
z, a reflection, under which ideal MHD is invariant and the faces see
their two tangential components in the other order.
*/
struct Axis_Map {
	int perm[3];
	bool identity() const { return perm[0] == 0 and perm[1] == 1 and perm[2] == 2; }
	// the caller's variable held in internal variable v
	int user_var(const int v) const
	{
		if (v >= 1 and v <= 3) return 1 + perm[v - 1];
		if (v >= 5 and v <= 7) return 5 + perm[v - 5];
		return v;
	}
};

inline Axis_Map axis_map(const pamhd_cfg& c)
{
	const bool ax = c.n[0] > 1, ay = c.n[1] > 1, az = c.n[2] > 1;
	if (not ax and ay) return Axis_Map{{1, 2, 0}};             // y, y-z
	if (not ax and not ay and az) return Axis_Map{{2, 0, 1}};  // z
	if (ax and not ay and az) return Axis_Map{{0, 2, 1}};      // x-z
	return Axis_Map{{0, 1, 2}};
}

// the internal configuration of a caller's configuration
inline pamhd_cfg relabelled(const pamhd_cfg& c, const Axis_Map& m)
{
	pamhd_cfg r = c;
	for (int a = 0; a < 3; a++) {
		const int u = m.perm[a];
		r.n[a] = c.n[u];
		r.cell_length[a] = c.cell_length[u];
		r.bc_lo[a] = c.bc_lo[u];
		r.bc_hi[a] = c.bc_hi[u];
		for (int v = 0; v < 8; v++) {
			r.value_lo[a][v] = c.value_lo[u][m.user_var(v)];
			r.value_hi[a][v] = c.value_hi[u][m.user_var(v)];
		}
	}
	return r;
}

inline Layout make_layout(const pamhd_cfg& c)
{
	Layout L;
	for (int d = 0; d < 3; d++) {
		L.n[d] = c.n[d];
		L.g[d] = c.n[d] > 1 ? 1 : 0;
	}
	L.xoff = 4;  // ghost column at 3: interior rows start 32-byte aligned
	L.pitch = ((L.xoff + L.n[0] + 1) + 3) / 4 * 4;
	L.rows = L.n[1] + 2 * L.g[1];
	L.planes = L.n[2] + 2 * L.g[2];
	L.plane = (long long)L.pitch * L.rows;
	L.var = (L.plane * L.planes + 31) / 32 * 32;
	return L;
}

/*
Constant step parameters of one grid; the buffers (state, reduction ring,
clock, status, control, dt history) are filled in by the caller.  Returns
whether the grid needs the boundary-layer speed pass (a non-periodic
active dimension next to another active one).
*/
inline bool grid_params(const pamhd_cfg& c, const Layout& L, Step_Params& P, const int kchunk_cap = 0)
{
	std::memset(&P, 0, sizeof P);
	P.L = L;
	P.gas.gamma = c.adiabatic_index;
	P.gas.mu0 = c.vacuum_permeability;
	P.gas.inv_mu0 = 1.0 / c.vacuum_permeability;
	P.gas.sqrt_mu0 = std::sqrt(c.vacuum_permeability);
	P.gas.inv_sqrt_mu0 = 1.0 / std::sqrt(c.vacuum_permeability);
	P.cfl = c.time_step_factor;
	P.forced_dt = -1.0;
	bool needs_boundary_speeds = false;
	int active_count = 0;
	for (int d = 0; d < 3; d++) {
		P.len[d] = c.cell_length[d];
		P.inv_len[d] = 1.0 / c.cell_length[d];
		P.active[d] = c.n[d] > 1;
		P.periodic[d] = P.active[d] and c.bc_lo[d] == PAMHD_BC_PERIODIC;
		P.bc_lo[d] = c.bc_lo[d];
		P.bc_hi[d] = c.bc_hi[d];
		P.ext[d] = (P.active[d] and not P.periodic[d]) ? 1 : 0;
		active_count += P.active[d];
	}
	for (int d = 0; d < 3; d++) {
		const bool own_side = c.bc_lo[d] != PAMHD_BC_EXTERNAL or c.bc_hi[d] != PAMHD_BC_EXTERNAL;
		if (P.active[d] and not P.periodic[d] and own_side and active_count > 1) needs_boundary_speeds = true;
	}
	// z planes per block: enough blocks for several waves on 148 SMs, few redundant z faces
	const int ty = P.active[1] ? step_tile_rows(c.solver) : 1;
	const long long tiles = (long long)((c.n[0] + 31) / 32) * ((c.n[1] + ty - 1) / ty);
	long long chunks = (PAMHD_CHUNK_BLOCKS + tiles - 1) / tiles;
	chunks = std::max(1LL, std::min(chunks, (long long)std::max(1, c.n[2] / 16)));
	P.kchunk = int((c.n[2] + chunks - 1) / chunks);
	if (kchunk_cap > 0) P.kchunk = std::min(P.kchunk, kchunk_cap);
	return needs_boundary_speeds;
}

} // namespace pamhd_b200

#endif
