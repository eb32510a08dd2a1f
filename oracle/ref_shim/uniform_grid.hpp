/*
Stand-in for the part of dccrg's grid interface that the reference's
substepping.hpp uses, for a uniform grid on one rank: local_cells() with
each cell's id, data and neighbours_of (face_neighbor: +-(d + 1) for the
face neighbours along dimension d, else 0; edge_neighbor[0]: >= 0 for the
edge neighbours, else -1), geometry.get_center, get_communicator and
update_copies_of_remote_neighbors (a no-op: one rank holds every cell).
Dimensions are periodic and a cell's neighbourhood is the 26 cells around
it, wrapped (a dimension of one cell makes a cell its own neighbour, as
dccrg does).  Cell ids start at 1, x fastest.  Topology only, no arithmetic
of the step.  TEST INFRASTRUCTURE (oracle/ref_substep_bridge.cpp).
*/
#ifndef PAMHD_ORACLE_UNIFORM_GRID_HPP
#define PAMHD_ORACLE_UNIFORM_GRID_HPP

#include <array>
#include <cstdint>
#include <vector>

#include "single_rank_mpi.hpp"

namespace oracle_shim {

template <class Cell_Data> class Uniform_Grid {
public:
	using cell_data_type = Cell_Data;

	struct Neighbor {
		Cell_Data* data;
		int face_neighbor;
		int edge_neighbor[3];
	};
	struct Cell {
		uint64_t id;
		Cell_Data* data;
		std::vector<Neighbor> neighbors_of;
	};
	struct Geometry {
		std::array<int, 3> n;
		std::array<double, 3> len;
		std::array<double, 3> get_center(const uint64_t id) const
		{
			const uint64_t i = id - 1;
			const uint64_t c[3] = {i % n[0], (i / n[0]) % n[1], i / (uint64_t(n[0]) * n[1])};
			return {(c[0] + 0.5) * len[0], (c[1] + 0.5) * len[1], (c[2] + 0.5) * len[2]};
		}
	};

	Geometry geometry;
	std::vector<Cell_Data> data;
	std::vector<Cell> cells;

	Uniform_Grid(const std::array<int, 3>& n, const std::array<double, 3>& len)
	{
		geometry.n = n;
		geometry.len = len;
		const size_t count = size_t(n[0]) * n[1] * n[2];
		data.resize(count);
		cells.resize(count);
		for (size_t i = 0; i < count; i++) {
			const int c[3] = {int(i % n[0]), int((i / n[0]) % n[1]), int(i / (size_t(n[0]) * n[1]))};
			Cell& cell = cells[i];
			cell.id = i + 1;
			cell.data = &data[i];
			for (int dz = -1; dz <= 1; dz++)
			for (int dy = -1; dy <= 1; dy++)
			for (int dx = -1; dx <= 1; dx++) {
				const int o[3] = {dx, dy, dz};
				int nonzero = 0, last = -1, zero_dim = -1;
				for (int d = 0; d < 3; d++) {
					if (o[d] != 0) {
						nonzero++;
						last = d;
					} else {
						zero_dim = d;
					}
				}
				if (nonzero == 0) continue;
				int m[3];
				for (int d = 0; d < 3; d++) m[d] = ((c[d] + o[d]) % n[d] + n[d]) % n[d];
				Neighbor nb;
				nb.data = &data[m[0] + size_t(n[0]) * (m[1] + size_t(n[1]) * m[2])];
				nb.face_neighbor = nonzero == 1 ? (o[last] > 0 ? last + 1 : -(last + 1)) : 0;
				nb.edge_neighbor[0] = nonzero == 2 ? zero_dim : -1;  // the edge runs along the zero offset
				nb.edge_neighbor[1] = nb.edge_neighbor[2] = 0;
				cell.neighbors_of.push_back(nb);
			}
		}
	}

	const std::vector<Cell>& local_cells() const { return cells; }
	MPI_Comm get_communicator() const { return 0; }
	void update_copies_of_remote_neighbors() {}
};

} // namespace oracle_shim

#endif
