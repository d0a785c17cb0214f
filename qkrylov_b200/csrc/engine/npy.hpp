// Minimal reader/writer of NumPy's .npy format (version 1.0: magic
// "\x93NUMPY", the version bytes, a little-endian u16 header length, a
// Python-dict header padded with spaces to a 64-byte boundary, then the raw
// little-endian data in C order), for the one-dimensional float64 and
// complex128 arrays and scalars of solver checkpoints.  numpy.load reads the
// files as they are.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace qkb {

// descr "<f8" (float64) or "<c16" (complex128); shape {} for a scalar.
void npy_write(const std::string& path, const void* data, const std::string& descr,
               const std::vector<uint64_t>& shape);
// The raw data of a file written as above; descr and shape are returned.
std::vector<char> npy_read(const std::string& path, std::string& descr, std::vector<uint64_t>& shape);

}  // namespace qkb
