/*
Stand-in for the part of dccrg's grid interface that the reference's
staggered-field step (mhd/solve.hpp timestep, common_functions.hpp
sync_magnetic_field, mhd/solar_wind_box.hpp apply_boundaries_sw_box) uses,
for a uniform box on one rank, written for this project: cells with id
(from 1, x fastest), data, is_local and neighbors_of; each neighbour with
its id, data, face_neighbor (+-(d + 1) along dimension d, else 0),
edge_neighbor ({edge dimension, sign of the offset along the lower other
dimension, sign along the higher}, or {-1, 0, 0}), relative_size (0: every
cell the same size), x, y, z (offset in index units) and is_local.  A
cell's neighbourhood is the 26 cells around it (dccrg's neighbourhood of
length 1); periodic dimensions wrap, bounded ones end at the box (cells
past it do not exist).  local_cells() and inner_cells() are every cell in
id order; outer_cells() and remote_cells() are empty (one rank holds
everything, rank 0); the remote-copy calls do nothing.  Topology and geometry only,
no arithmetic of the step.  TEST INFRASTRUCTURE (oracle/ref_stag_bridge.cpp).
*/
#ifndef PAMHD_ORACLE_BOX_GRID_HPP
#define PAMHD_ORACLE_BOX_GRID_HPP

#include <array>
#include <cstdint>
#include <vector>

#include "single_rank_mpi.hpp"

namespace oracle_shim {

template <class Cell_Data> class Box_Grid {
public:
	using cell_data_type = Cell_Data;

	struct Neighbor {
		uint64_t id;
		Cell_Data* data;
		int face_neighbor;
		std::array<int, 3> edge_neighbor;
		int relative_size;
		int x, y, z;
		bool is_local;
	};
	struct Cell {
		uint64_t id;
		Cell_Data* data;
		bool is_local;
		std::vector<Neighbor> neighbors_of;
	};
	struct Geometry {
		std::array<int, 3> n;
		std::array<double, 3> len;
		std::array<double, 3> get_length(const uint64_t) const { return len; }
		std::array<double, 3> get_center(const uint64_t id) const
		{
			const uint64_t i = id - 1;
			const uint64_t c[3] = {i % n[0], (i / n[0]) % n[1], i / (uint64_t(n[0]) * n[1])};
			return {(c[0] + 0.5) * len[0], (c[1] + 0.5) * len[1], (c[2] + 0.5) * len[2]};
		}
	};
	struct Mapping {
		std::array<int, 3> n;
		uint64_t get_cell_length_in_indices(const uint64_t) const { return 1; }
		std::array<uint64_t, 3> get_indices(const uint64_t id) const
		{
			const uint64_t i = id - 1;
			return {i % n[0], (i / n[0]) % n[1], i / (uint64_t(n[0]) * n[1])};
		}
	};

	Geometry geometry;
	Mapping mapping;
	std::vector<Cell_Data> data;
	std::vector<Cell> cells;
	std::vector<Cell> none;

	Box_Grid(const std::array<int, 3>& n, const std::array<double, 3>& len, const std::array<bool, 3>& periodic)
	{
		geometry.n = n;
		geometry.len = len;
		mapping.n = n;
		const size_t count = size_t(n[0]) * n[1] * n[2];
		data.resize(count);
		cells.resize(count);
		for (size_t i = 0; i < count; i++) {
			const int c[3] = {int(i % n[0]), int((i / n[0]) % n[1]), int(i / (size_t(n[0]) * n[1]))};
			Cell& cell = cells[i];
			cell.id = i + 1;
			cell.data = &data[i];
			cell.is_local = true;
			for (int dz = -1; dz <= 1; dz++)
			for (int dy = -1; dy <= 1; dy++)
			for (int dx = -1; dx <= 1; dx++) {
				const int o[3] = {dx, dy, dz};
				int nonzero = 0, last = -1, zero_dim = -1;
				bool exists = true;
				int m[3];
				for (int d = 0; d < 3; d++) {
					if (o[d] != 0) {
						nonzero++;
						last = d;
					} else {
						zero_dim = d;
					}
					m[d] = c[d] + o[d];
					if (periodic[d]) {
						m[d] = (m[d] % n[d] + n[d]) % n[d];
					} else if (m[d] < 0 or m[d] >= n[d]) {
						exists = false;
					}
				}
				if (nonzero == 0 or not exists) continue;
				Neighbor nb;
				const size_t j = m[0] + size_t(n[0]) * (m[1] + size_t(n[1]) * m[2]);
				nb.id = j + 1;
				nb.data = &data[j];
				nb.face_neighbor = nonzero == 1 ? (o[last] > 0 ? last + 1 : -(last + 1)) : 0;
				if (nonzero == 2) {
					const int lo = (zero_dim + 1) % 3 < (zero_dim + 2) % 3 ? (zero_dim + 1) % 3 : (zero_dim + 2) % 3;
					const int hi = 3 - zero_dim - lo;
					nb.edge_neighbor = {zero_dim, o[lo], o[hi]};
				} else {
					nb.edge_neighbor = {-1, 0, 0};
				}
				nb.relative_size = 0;
				nb.x = o[0];
				nb.y = o[1];
				nb.z = o[2];
				nb.is_local = true;
				cell.neighbors_of.push_back(nb);
			}
		}
	}

	const std::vector<Cell>& local_cells() const { return cells; }
	const std::vector<Cell>& inner_cells() const { return cells; }
	const std::vector<Cell>& all_cells() const { return cells; }
	const std::vector<Cell>& outer_cells() const { return none; }
	const std::vector<Cell>& remote_cells() const { return none; }
	Cell_Data* operator[](const uint64_t id) { return id >= 1 and id <= data.size() ? &data[id - 1] : nullptr; }
	MPI_Comm get_communicator() const { return 0; }
	int get_rank() const { return 0; }
	void update_copies_of_remote_neighbors() {}
	void start_remote_neighbor_copy_updates() {}
	void wait_remote_neighbor_copy_update_receives() {}
	void wait_remote_neighbor_copy_update_sends() {}
};

} // namespace oracle_shim

#endif
