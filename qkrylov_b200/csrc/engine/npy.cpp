#include "npy.hpp"

#include <cstring>
#include <fstream>
#include <stdexcept>

namespace qkb {

namespace {
size_t elem_size(const std::string& descr) {
  if (descr == "<f8") return 8;
  if (descr == "<c16") return 16;
  throw std::invalid_argument("npy: unsupported dtype " + descr);
}
}  // namespace

void npy_write(const std::string& path, const void* data, const std::string& descr,
               const std::vector<uint64_t>& shape) {
  const size_t es = elem_size(descr);
  uint64_t n = 1;
  std::string sh = "(";
  for (size_t i = 0; i < shape.size(); ++i) {
    n *= shape[i];
    sh += std::to_string(shape[i]) + (shape.size() == 1 ? "," : (i + 1 < shape.size() ? ", " : ""));
  }
  sh += ")";
  std::string hdr = "{'descr': '" + descr + "', 'fortran_order': False, 'shape': " + sh + ", }";
  const size_t pre = 10;  // magic (6) + version (2) + length (2)
  size_t total = pre + hdr.size() + 1;
  hdr += std::string((64 - total % 64) % 64, ' ');
  hdr += '\n';
  if (hdr.size() > 65535) throw std::invalid_argument("npy: header too long");
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) throw std::runtime_error("npy: cannot write " + path);
  const char magic[8] = {'\x93', 'N', 'U', 'M', 'P', 'Y', 1, 0};
  f.write(magic, 8);
  const uint16_t hl = uint16_t(hdr.size());
  const char lb[2] = {char(hl & 0xFF), char(hl >> 8)};
  f.write(lb, 2);
  f.write(hdr.data(), std::streamsize(hdr.size()));
  f.write(static_cast<const char*>(data), std::streamsize(n * es));
  if (!f) throw std::runtime_error("npy: write failed for " + path);
}

std::vector<char> npy_read(const std::string& path, std::string& descr, std::vector<uint64_t>& shape) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("npy: cannot read " + path);
  char magic[10];
  f.read(magic, 10);
  if (!f || std::memcmp(magic, "\x93NUMPY", 6) != 0 || magic[6] != 1)
    throw std::runtime_error("npy: not a version-1 .npy file: " + path);
  const uint16_t hl = uint16_t(uint8_t(magic[8])) | uint16_t(uint16_t(uint8_t(magic[9])) << 8);
  std::string hdr(hl, '\0');
  f.read(&hdr[0], hl);
  auto field = [&](const std::string& key) {
    const size_t k = hdr.find("'" + key + "':");
    if (k == std::string::npos) throw std::runtime_error("npy: header without " + key + ": " + path);
    return k + key.size() + 3;
  };
  size_t k = hdr.find('\'', field("descr"));
  const size_t e = hdr.find('\'', k + 1);
  descr = hdr.substr(k + 1, e - k - 1);
  if (hdr.find("True", field("fortran_order")) < hdr.find(',', field("fortran_order")))
    throw std::runtime_error("npy: Fortran order not supported: " + path);
  k = hdr.find('(', field("shape"));
  const size_t c = hdr.find(')', k);
  shape.clear();
  uint64_t n = 1;
  std::string dims = hdr.substr(k + 1, c - k - 1);
  size_t p = 0;
  while (p < dims.size()) {
    while (p < dims.size() && (dims[p] == ' ' || dims[p] == ',')) ++p;
    if (p >= dims.size()) break;
    size_t q = p;
    while (q < dims.size() && dims[q] >= '0' && dims[q] <= '9') ++q;
    if (q == p) throw std::runtime_error("npy: bad shape in " + path);
    shape.push_back(std::stoull(dims.substr(p, q - p)));
    n *= shape.back();
    p = q;
  }
  std::vector<char> out(n * elem_size(descr));
  f.read(out.data(), std::streamsize(out.size()));
  if (!f) throw std::runtime_error("npy: truncated data in " + path);
  return out;
}

}  // namespace qkb
