// Which die of the B200 each SM sits on.
//
// A B200 is two dies with 74 SMs each; each die has its own half of the L2.
// A line an SM reads is cached in its own die's L2, and an SM of the other
// die that reads the line later finds it there through the die-to-die link
// (measured on this GPU: ~280 cycles for a hit in the own die's L2, ~480 for
// one in the other die's, ~800 from DRAM).  Data that both dies read is
// therefore cached twice, and each die's L2 holds only its own SMs' working
// set.  Kernels with partner reuse (the row kernels of H.x) give each die
// its own share of the work so that the two L2 halves hold two disjoint
// working sets instead of two copies of one.
//
// The SM-to-die assignment is not a fixed function of %smid (it follows the
// chip's floorsweeping), so it is measured once per device: one CTA warms a
// 64 KB region per SM into its die's L2, then every SM chases pointers
// through its own region; SMs of the warming CTA's die see the short
// latency.  A GPU whose latencies are not bimodal is reported as one die.
#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace qkd {
namespace {

constexpr uint32_t kTopoLines = 512;               // 128-byte lines per region (64 KB)
constexpr uint32_t kTopoWords = kTopoLines * 32;   // u32 words per region
constexpr uint32_t kTopoStride = 173;              // odd: one cycle through all lines
constexpr uint32_t kTopoSteps = 256;
constexpr int kTopoMaxSm = 1024;

__device__ __forceinline__ uint32_t smid_reg() {
  uint32_t s;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(s));
  return s;
}

// chain: word 0 of line i of every region holds the next line, (i + stride) mod lines
__global__ void k_topo_init(uint32_t* buf, uint32_t nreg) {
  const size_t n = size_t(nreg) * kTopoLines;
  for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
    const uint32_t line = uint32_t(k % kTopoLines);
    buf[k * 32] = (line + kTopoStride) % kTopoLines;
  }
}

// one CTA: read every line of every region (into this SM's die's L2)
__global__ void k_topo_warm(const uint32_t* buf, uint32_t nreg, uint32_t* ref_sm, uint32_t* sink) {
  uint32_t acc = 0;
  const size_t n = size_t(nreg) * kTopoLines;
  for (size_t k = threadIdx.x; k < n; k += blockDim.x) acc += __ldcg(buf + k * 32);
  if (threadIdx.x == 0) *ref_sm = smid_reg();
  if (acc == 0xFFFFFFFFu) *sink = acc;
}

// the first CTA on each SM chases the SM's own region and records cycles/step
__global__ void k_topo_chase(const uint32_t* buf, uint32_t nreg, unsigned* claim, uint32_t* lat) {
  if (threadIdx.x != 0) return;
  const uint32_t s = smid_reg();
  if (s >= nreg || atomicCAS(claim + s, 0u, 1u) != 0u) return;
  const uint32_t* r = buf + size_t(s) * kTopoWords;
  uint32_t j = 0;
  const long long t0 = clock64();
  for (uint32_t k = 0; k < kTopoSteps; ++k) j = __ldcg(r + j * 32);
  const long long t1 = clock64();
  lat[s] = uint32_t((t1 - t0) / kTopoSteps) | (j >= kTopoLines ? 0x80000000u : 0u);
}

struct DieMap {
  bool done = false;
  uint8_t* dev = nullptr;  // die of each SM id (0: the warming CTA's die)
  int nsmid = 0, n0 = 0, n1 = 0;
};
std::mutex g_topo_mu;
DieMap g_topo[64];

void measure(int device, DieMap& m) {
  int nsmid = 0, nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  nsmid = nsm;
  // %smid can exceed the SM count on a floorswept chip: leave room
  const uint32_t nreg = uint32_t(std::min(kTopoMaxSm, std::max(nsm * 2, 1)));
  uint32_t *buf = nullptr, *small = nullptr;
  const size_t bytes = size_t(nreg) * kTopoWords * 4;
  // small: [0] ref SM, [1] sink, [2 .. 2 + nreg) latency, then nreg claims
  if (cudaMalloc(&buf, bytes) != cudaSuccess || cudaMalloc(&small, (2 + 2 * size_t(nreg)) * 4) != cudaSuccess) {
    (void)cudaGetLastError();
    cudaFree(buf);
    return;
  }
  std::vector<uint32_t> h(2 + 2 * size_t(nreg), 0);
  bool ok = cudaMemset(small, 0, h.size() * 4) == cudaSuccess;
  if (ok) {
    k_topo_init<<<256, 256>>>(buf, nreg);
    k_topo_warm<<<1, 1024>>>(buf, nreg, small, small + 1);
    k_topo_chase<<<nreg * 4, 32>>>(buf, nreg, small + 2 + nreg, small + 2);
    ok = cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess &&
         cudaMemcpy(h.data(), small, h.size() * 4, cudaMemcpyDeviceToHost) == cudaSuccess;
  }
  (void)cudaGetLastError();
  cudaFree(buf);
  cudaFree(small);
  if (!ok) return;
  uint32_t tmin = 0xFFFFFFFFu, tmax = 0, maxid = 0;
  for (uint32_t s = 0; s < nreg; ++s) {
    const uint32_t t = h[2 + s];
    if (t == 0 || (t & 0x80000000u)) continue;
    tmin = std::min(tmin, t);
    tmax = std::max(tmax, t);
    maxid = s + 1;
  }
  // two dies: near and far hits differ by well over a third of the near latency
  if (maxid == 0 || tmax < tmin + tmin / 3) return;
  nsmid = int(maxid);
  std::vector<uint8_t> die(nsmid, 0);
  const uint32_t mid = (tmin + tmax) / 2;
  for (int s = 0; s < nsmid; ++s) {
    const uint32_t t = h[2 + s];
    die[s] = (t != 0 && !(t & 0x80000000u) && t > mid) ? 1 : 0;
    (die[s] ? m.n1 : m.n0) += (t != 0) ? 1 : 0;
  }
  if (m.n0 == 0 || m.n1 == 0) { m.n0 = m.n1 = 0; return; }
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, nsmid) != cudaSuccess || cudaMemcpy(d, die.data(), nsmid, cudaMemcpyHostToDevice) != cudaSuccess) {
    (void)cudaGetLastError();
    cudaFree(d);
    m.n0 = m.n1 = 0;
    return;
  }
  m.dev = d;
  m.nsmid = nsmid;
}

}  // namespace

// Die of every SM of the current device, measured on the first call (a few
// launches, ~10 MB for a moment) and kept until exit.  Returns false when
// the device shows one die (or the measurement could not run); then
// *dev_map is null.
bool die_map(const uint8_t** dev_map, int* nsmid, int* n0, int* n1) {
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) {
    (void)cudaGetLastError();
    return false;
  }
  std::lock_guard<std::mutex> lk(g_topo_mu);
  DieMap& m = g_topo[device];
  if (!m.done) {
    measure(device, m);
    m.done = true;
  }
  *dev_map = m.dev;
  *nsmid = m.nsmid;
  *n0 = m.n0;
  *n1 = m.n1;
  return m.dev != nullptr;
}

}  // namespace qkd

extern "C" int qkd_die_count(int* sms_die0, int* sms_die1) {
  const uint8_t* d = nullptr;
  int ns = 0, a = 0, b = 0;
  const bool two = qkd::die_map(&d, &ns, &a, &b);
  if (sms_die0) *sms_die0 = a;
  if (sms_die1) *sms_die1 = b;
  return two ? 2 : 1;
}
