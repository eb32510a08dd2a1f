/*
The reference's MHD output files (.dc, file version 4) for uniform grids,
written and read on the host, so that states of this library can be
compared with the reference's own runs and read by its tools
(tests/mhd/mhd_diff.py, mhd2vtk.py, ...), and the reference's outputs can
be loaded as initial states.

Layout (mhd/save.hpp:75-375 writes it through dccrg's save_grid_data; the
reference's reader is tests/common.py:35-200), little endian:
  uint64 file version (4), uint64 simulation step,
  double simulation time, adiabatic index, proton mass, vacuum
    permeability, particle temperature / energy ratio (-1 when unused),
  uint8 number of variables, uint64 file offset of each variable,
  uint64 endianness mark 0x1234567890abcdef,
  uint64[3] level-0 cells, int32 maximum refinement level,
  uint32 neighbourhood length, uint8[3] periodicity, int32 geometry id (1),
  double[3] grid start, double[3] level-0 cell length,
  uint64 number of cells, uint64 cell ids (1 + i + nx (j + ny k) on level 0),
  then each variable: an 8-character name and its data, cell by cell in the
  order of the id list.
This file writes and reads the variable "mhd     ": per cell the mass
density, momentum density (3), total energy density and volume magnetic
field (3), 8 doubles.  Other variables of a file being read are skipped.
*/
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "pamhd_gpu.h"

namespace {

constexpr uint64_t FILE_VERSION = 4;
constexpr uint64_t ENDIANNESS = 0x1234567890abcdefull;
const char MHD_NAME[9] = "mhd     ";

struct File {
	std::FILE* f = nullptr;
	explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
	~File() { if (f != nullptr) std::fclose(f); }
	template <class T> bool put(const T& v) { return std::fwrite(&v, sizeof v, 1, f) == 1; }
	bool put_bytes(const void* p, const size_t n) { return std::fwrite(p, 1, n, f) == n; }
	template <class T> bool get(T& v) { return std::fread(&v, sizeof v, 1, f) == 1; }
	bool get_bytes(void* p, const size_t n) { return std::fread(p, 1, n, f) == n; }
	bool seek(const uint64_t at) { return std::fseek(f, long(at), SEEK_SET) == 0; }
};

// the fixed part of a file up to the cell list, and the offsets of its variables
struct Header {
	pamhd_dc_info info;
	std::vector<uint64_t> offsets;
	uint64_t cell_list = 0;
};

int read_header(File& in, Header& h)
{
	uint64_t version = 0, step = 0, endian = 0, cells[3], total = 0;
	double params[5];
	uint8_t nvar = 0, periodic[3];
	int32_t max_lvl = 0, geometry = 0;
	uint32_t neighbourhood = 0;
	double start[3], length[3];
	if (not in.get(version) or not in.get(step) or not in.get_bytes(params, sizeof params) or not in.get(nvar)) {
		return PAMHD_ERR_IO;
	}
	if (version != FILE_VERSION) return PAMHD_ERR_ARGUMENT;
	h.offsets.resize(nvar);
	if (nvar > 0 and not in.get_bytes(h.offsets.data(), nvar * sizeof(uint64_t))) return PAMHD_ERR_IO;
	if (not in.get(endian) or not in.get_bytes(cells, sizeof cells) or not in.get(max_lvl)
		or not in.get(neighbourhood) or not in.get_bytes(periodic, sizeof periodic) or not in.get(geometry)
		or not in.get_bytes(start, sizeof start) or not in.get_bytes(length, sizeof length) or not in.get(total)) {
		return PAMHD_ERR_IO;
	}
	if (endian != ENDIANNESS or geometry != 1) return PAMHD_ERR_ARGUMENT;
	// uniform grids only: no refinement, every level-0 cell present
	if (max_lvl != 0 or total != cells[0] * cells[1] * cells[2]) return PAMHD_ERR_ARGUMENT;
	std::memset(&h.info, 0, sizeof h.info);
	h.info.step = step;
	h.info.time = params[0];
	h.info.adiabatic_index = params[1];
	h.info.proton_mass = params[2];
	h.info.vacuum_permeability = params[3];
	for (int d = 0; d < 3; d++) {
		if (cells[d] < 1 or cells[d] > 0x7fffffffull) return PAMHD_ERR_ARGUMENT;
		h.info.n[d] = int32_t(cells[d]);
		h.info.periodic[d] = periodic[d] != 0;
		h.info.start[d] = start[d];
		h.info.cell_length[d] = length[d];
	}
	h.info.cells = total;
	h.cell_list = uint64_t(std::ftell(in.f));
	return PAMHD_OK;
}

} // namespace

extern "C" {

int pamhd_dc_write(const char* path, const pamhd_dc_info* info, const double* const soa[8])
{
	if (path == nullptr or info == nullptr or soa == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int v = 0; v < 8; v++) if (soa[v] == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int d = 0; d < 3; d++) if (info->n[d] < 1) return PAMHD_ERR_ARGUMENT;
	const uint64_t nx = uint64_t(info->n[0]), ny = uint64_t(info->n[1]), nz = uint64_t(info->n[2]);
	const uint64_t total = nx * ny * nz;
	File out(path, "wb");
	if (out.f == nullptr) return PAMHD_ERR_IO;
	const uint8_t nvar = 1;
	// the header: 65 bytes before the grid part with one variable, 103 in the grid part, then the ids
	const uint64_t cell_list = 8 + 8 + 5 * 8 + 1 + nvar * 8 + 8 + 24 + 4 + 4 + 3 + 4 + 24 + 24 + 8;
	const uint64_t mhd_offset = cell_list + total * 8;
	const double params[5] = {info->time, info->adiabatic_index, info->proton_mass, info->vacuum_permeability,
	                          -1.0};
	const uint64_t cells[3] = {nx, ny, nz};
	const uint8_t periodic[3] = {uint8_t(info->periodic[0] != 0), uint8_t(info->periodic[1] != 0),
	                             uint8_t(info->periodic[2] != 0)};
	const int32_t max_lvl = 0, geometry = 1;
	const uint32_t neighbourhood = 1;
	bool ok = out.put(FILE_VERSION) and out.put(info->step) and out.put_bytes(params, sizeof params)
		and out.put(nvar) and out.put(mhd_offset) and out.put(ENDIANNESS) and out.put_bytes(cells, sizeof cells)
		and out.put(max_lvl) and out.put(neighbourhood) and out.put_bytes(periodic, sizeof periodic)
		and out.put(geometry) and out.put_bytes(info->start, sizeof info->start)
		and out.put_bytes(info->cell_length, sizeof info->cell_length) and out.put(total);
	if (not ok or uint64_t(std::ftell(out.f)) != cell_list) return PAMHD_ERR_IO;
	std::vector<uint64_t> ids(total);
	for (uint64_t c = 0; c < total; c++) ids[c] = c + 1;
	ok = out.put_bytes(ids.data(), total * sizeof(uint64_t)) and out.put_bytes(MHD_NAME, 8);
	std::vector<double> rows(8 * std::min<uint64_t>(total, 1 << 16));
	for (uint64_t first = 0; ok and first < total; first += rows.size() / 8) {
		const uint64_t count = std::min<uint64_t>(total - first, rows.size() / 8);
		for (uint64_t c = 0; c < count; c++) {
			for (int v = 0; v < 8; v++) rows[8 * c + v] = soa[v][first + c];
		}
		ok = out.put_bytes(rows.data(), count * 8 * sizeof(double));
	}
	return ok ? PAMHD_OK : PAMHD_ERR_IO;
}

int pamhd_dc_read_info(const char* path, pamhd_dc_info* info)
{
	if (path == nullptr or info == nullptr) return PAMHD_ERR_ARGUMENT;
	File in(path, "rb");
	if (in.f == nullptr) return PAMHD_ERR_IO;
	Header h;
	const int rc = read_header(in, h);
	if (rc != PAMHD_OK) return rc;
	*info = h.info;
	return PAMHD_OK;
}

int pamhd_dc_read(const char* path, double* const soa[8])
{
	if (path == nullptr or soa == nullptr) return PAMHD_ERR_ARGUMENT;
	for (int v = 0; v < 8; v++) if (soa[v] == nullptr) return PAMHD_ERR_ARGUMENT;
	File in(path, "rb");
	if (in.f == nullptr) return PAMHD_ERR_IO;
	Header h;
	int rc = read_header(in, h);
	if (rc != PAMHD_OK) return rc;
	const uint64_t total = h.info.cells;
	std::vector<uint64_t> ids(total);
	if (not in.get_bytes(ids.data(), total * sizeof(uint64_t))) return PAMHD_ERR_IO;
	// the variable named "mhd     "
	uint64_t data = 0;
	for (const uint64_t offset: h.offsets) {
		char name[8];
		if (not in.seek(offset) or not in.get_bytes(name, 8)) return PAMHD_ERR_IO;
		if (std::memcmp(name, MHD_NAME, 8) == 0) data = offset + 8;
	}
	if (data == 0) return PAMHD_ERR_ARGUMENT;
	if (not in.seek(data)) return PAMHD_ERR_IO;
	std::vector<double> rows(8 * std::min<uint64_t>(total, 1 << 16));
	for (uint64_t first = 0; first < total; first += rows.size() / 8) {
		const uint64_t count = std::min<uint64_t>(total - first, rows.size() / 8);
		if (not in.get_bytes(rows.data(), count * 8 * sizeof(double))) return PAMHD_ERR_IO;
		for (uint64_t c = 0; c < count; c++) {
			const uint64_t id = ids[first + c];
			if (id < 1 or id > total) return PAMHD_ERR_ARGUMENT;
			for (int v = 0; v < 8; v++) soa[v][id - 1] = rows[8 * c + v];
		}
	}
	return PAMHD_OK;
}

} // extern "C"
