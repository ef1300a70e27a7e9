// Map files on either side of the statistics: NESTED `.npy` arrays and
// HEALPix FITS binary tables, as the reference's synthesis tools read and
// write them (crates/stl-mpi/src/io.rs:18-569): whole maps, the length of a
// map without reading it, a pixel range read at its offset, and files
// written in pieces (each piece at its own offset).  Host code only; errors
// are std::runtime_error naming the file.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace stl {
namespace mapio {

// nside of a full-sky map of npix pixels (a power of two); throws otherwise
int64_t nside_of(size_t npix);

// pixels of the map in the file (.fits / .fit: HEALPix FITS, else .npy)
size_t map_len(const std::string& path);
// the whole map as NESTED float64 (RING FITS maps are reordered)
std::vector<double> read_map(const std::string& path);
// the shape of a .npy array (C order) and its values as float64
std::vector<double> read_npy(const std::string& path, std::vector<size_t>* shape);
// the shape alone, from the header
std::vector<size_t> npy_shape(const std::string& path);
// pixels [start, end) of the NESTED map (a RING FITS map is read whole)
std::vector<double> read_map_range(const std::string& path, size_t start, size_t end);

// little-endian float64 .npy (format 1.0) of the given C-order shape
void write_npy(const std::string& path, const double* values, const std::vector<size_t>& shape);
// a full-sky NESTED map as a HEALPix binary table of one column: float32
// ('E') or float64 ('D'), big-endian
void write_healpix_fits(const std::string& path, const double* values, size_t n, const std::string& column,
                        bool dbl);

// Files written in pieces: create() writes the headers and sizes the file
// for n pixels (.npy float64, or FITS with an 'E' / 'D' column), then
// write_piece() puts pixels [start, start + count) at their offset.
void create_map(const std::string& path, size_t n, const std::string& column, bool dbl);
void write_piece(const std::string& path, size_t start, const double* values, size_t count, bool dbl);

}  // namespace mapio
}  // namespace stl
