// Multi-vector dot that allocates nothing.
//
// Some callers cannot let a library call cudaMalloc: code whose device
// memory is owned by another allocator's pool (a framework caching
// allocator, a Julia or Python GPU array pool), where a raw cudaMalloc can
// fail even though the pool has room, and latency-critical loops where an
// allocation or a cudaFree would synchronise the device and stall other
// streams.  qkrylov_b200_multi_dot_noalloc serves them: it computes the same
// reorthogonalisation coefficients as qkrylov_b200_multi_dot,
// out[2j..2j+1] = <V_j, x> for j < k, with every byte of scratch (per-block
// partial sums, the completion ticket, the result staging and the device
// copy of the V pointers) in one file-scope device array of fixed size,
// kNoallocScratchBytes (about 129 KB), which every GPU that loads the
// library holds until the process exits.
//
// Limits: k <= kNoallocMaxK vectors per call (larger k is rejected with
// QKRYLOV_ERROR_INVALID_ARG); the reduction uses at most kNoallocBlocks
// blocks.  The array is shared by every call on a device and keeps the last
// call's contents; calls whose kernels overlap on the GPU (different host
// threads, different streams) race on it, so callers serialise them.  The
// completion ticket must start at zero: the first call on a device clears
// it, and every call leaves it at zero.
//
// Set-up: the first call on a device (with that device made current) asks
// CUDA for the array's device address with cudaGetSymbolAddress and clears
// the ticket; later calls reuse the cached address.  Make that first call
// before any stream capture.  In host code the array's name is only a
// host-side stand-in, never a device address, which is why the address is
// obtained this way.
#include <algorithm>
#include <mutex>
#include <string>

#include "reduce.cuh"

namespace qkd {
namespace {

constexpr int kNoallocMaxK = 16;
constexpr int kNoallocBlocks = 512;
constexpr size_t kPartialBytes = size_t(kNoallocMaxK) * kNoallocBlocks * 2 * sizeof(double);
constexpr size_t kTicketOff = kPartialBytes;               // 256 bytes reserved
constexpr size_t kResultOff = kTicketOff + 256;            // 2 * kNoallocMaxK doubles
constexpr size_t kPtrOff = kResultOff + 256;               // kNoallocMaxK pointers
constexpr size_t kNoallocScratchBytes = kPtrOff + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kThreadsNA = 256;
constexpr int kE = 8;

// The tiled multi-dot of the reorthogonalisation (vec.cu), with its
// partials, ticket, result and pointer array taken from g_noalloc_scratch.
template <int DT>
__global__ void __launch_bounds__(kThreadsNA) k_mdot_noalloc(size_t n, int k, const void* x) {
  using T = VT<DT>;
  using R = typename T::R;
  double* partials = reinterpret_cast<double*>(g_noalloc_scratch);
  unsigned* ticket = reinterpret_cast<unsigned*>(g_noalloc_scratch + kTicketOff);
  double* out = reinterpret_cast<double*>(g_noalloc_scratch + kResultOff);
  const void* const* V = reinterpret_cast<const void* const*>(g_noalloc_scratch + kPtrOff);
  __shared__ double sacc[kThreadsNA / 32][kNoallocMaxK][2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int j = lane; j < k; j += 32) { sacc[warp][j][0] = 0.0; sacc[warp][j][1] = 0.0; }
  __syncwarp();
  const size_t tile = size_t(32) * kE;
  const size_t nwarps = size_t(gridDim.x) * (kThreadsNA / 32);
  for (size_t base = (size_t(blockIdx.x) * (kThreadsNA / 32) + warp) * tile; base < n; base += nwarps * tile) {
    double xr[kE], xi[kE];
    #pragma unroll
    for (int e = 0; e < kE; ++e) {
      const size_t i = base + size_t(e) * 32 + lane;
      xr[e] = 0.0; xi[e] = 0.0;
      if (i < n) { R r, m; T::ld(x, i, r, m); xr[e] = r; xi[e] = m; }
    }
    for (int j = 0; j < k; ++j) {
      const void* vj = V[j];
      double pr = 0.0, pi = 0.0;
      #pragma unroll
      for (int e = 0; e < kE; ++e) {
        const size_t i = base + size_t(e) * 32 + lane;
        if (i < n) {
          R vr, vi; T::ld(vj, i, vr, vi);
          pr += double(vr) * xr[e] + double(vi) * xi[e];
          pi += double(vr) * xi[e] - double(vi) * xr[e];
        }
      }
      pr = warp_sum(pr);
      pi = warp_sum(pi);
      if (lane == 0) { sacc[warp][j][0] += pr; sacc[warp][j][1] += pi; }
    }
  }
  __syncthreads();
  const int G = gridDim.x;
  for (int j = threadIdx.x; j < k; j += kThreadsNA) {
    double re = 0.0, im = 0.0;
    for (int w = 0; w < kThreadsNA / 32; ++w) { re += sacc[w][j][0]; im += sacc[w][j][1]; }
    partials[(size_t(j) * G + blockIdx.x) * 2] = re;
    partials[(size_t(j) * G + blockIdx.x) * 2 + 1] = im;
  }
  grid_finish(partials, ticket, k, out);
}

std::mutex g_setup_mu;
unsigned char* g_scratch_addr[64] = {nullptr};

// Once per device, with the device current: the array's device address.
// Returns the CUDA error of a failed set-up step (cudaSuccess otherwise).
cudaError_t scratch_address(int device, cudaStream_t s, unsigned char** out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_addr[device]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e == cudaSuccess && !ptr) e = cudaErrorInvalidSymbol;
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      return e;
    }
    unsigned char* base = static_cast<unsigned char*>(ptr);
    e = cudaMemsetAsync(base + kTicketOff, 0, 256, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      return e;
    }
    g_scratch_addr[device] = base;
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

}  // namespace
}  // namespace qkd

namespace qkapi {
void set_error(const std::string& msg);
}

extern "C" int qkrylov_b200_multi_dot_noalloc(int device, int dtype, size_t n, int k, const void* const* V,
                                              const void* x, double* out, void* stream) {
  using namespace qkd;
  if (device < 0 || device >= 64 || dtype < QK_C128 || dtype > QK_F32 || k <= 0 || !V || !x || !out) {
    qkapi::set_error("multi_dot_noalloc: invalid argument");
    return -1;
  }
  if (k > kNoallocMaxK) {
    qkapi::set_error("multi_dot_noalloc: k = " + std::to_string(k) + " exceeds the static scratch maximum of " +
                     std::to_string(kNoallocMaxK) + " vectors per call");
    return -1;
  }
  for (int j = 0; j < k; ++j)
    if (!V[j]) { qkapi::set_error("multi_dot_noalloc: null vector"); return -1; }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device >= ndev) {
    (void)cudaGetLastError();
    qkapi::set_error("multi_dot_noalloc: invalid argument (device " + std::to_string(device) + " of " +
                     std::to_string(ndev) + ")");
    return -1;
  }
  int prev = 0;
  cudaError_t e = cudaGetDevice(&prev);
  if (e == cudaSuccess) e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    qkapi::set_error(std::string("multi_dot_noalloc: cannot select the device: ") + cudaGetErrorString(e));
    return -2;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned char* base = nullptr;
  e = scratch_address(device, s, &base);
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + kPtrOff, V, sizeof(void*) * k, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    const size_t need = (n + 2047) / 2048;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    const unsigned G = unsigned(std::max<size_t>(1, std::min<size_t>({need, size_t(nsm) * 4, size_t(kNoallocBlocks)})));
    switch (dtype) {
      case QK_C128: k_mdot_noalloc<QK_C128><<<G, kThreadsNA, 0, s>>>(n, k, x); break;
      case QK_C64: k_mdot_noalloc<QK_C64><<<G, kThreadsNA, 0, s>>>(n, k, x); break;
      case QK_F64: k_mdot_noalloc<QK_F64><<<G, kThreadsNA, 0, s>>>(n, k, x); break;
      default: k_mdot_noalloc<QK_F32><<<G, kThreadsNA, 0, s>>>(n, k, x); break;
    }
    count_launch();
    e = cudaPeekAtLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, base + kResultOff, sizeof(double) * 2 * k, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    qkapi::set_error(std::string("multi_dot_noalloc: ") + cudaGetErrorString(e));
  }
  cudaSetDevice(prev);
  return e == cudaSuccess ? 0 : -2;
}
