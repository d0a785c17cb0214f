#include "runtime.hpp"

#include <map>
#include <mutex>

namespace qkb {

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw DeviceError(std::string("qkrylov_b200: ") + what + ": " + cudaGetErrorString(e));
  }
}

void qkd_check(int rc, const char* what) {
  if (rc == QKD_OK) return;
  const char* why = rc == QKD_EINVAL ? "invalid argument"
                    : rc == QKD_ENOMEM ? "out of device memory"
                    : rc == QKD_ETIMEOUT ? "device wait timed out"
                                        : "CUDA launch failed";
  throw DeviceError(std::string("qkrylov_b200: ") + what + ": " + why);
}

Context::Context(int dev) : device(dev) {
  int n = 0;
  cuda_check(cudaGetDeviceCount(&n), "cudaGetDeviceCount");
  if (dev < 0 || dev >= n) throw DeviceError("qkrylov_b200: no CUDA device " + std::to_string(dev));
  cuda_check(cudaSetDevice(dev), "cudaSetDevice");
  cuda_check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
  qkd_check(qkd_workspace_create(dev, &ws), "workspace");
  cuda_check(cudaMallocHost(&host, sizeof(double) * kHost), "cudaMallocHost");
  // Solver vectors come from the device's stream-ordered pool, which keeps
  // freed memory for the next solve instead of returning it at every
  // synchronisation (a Lanczos run allocates and frees one vector per step).
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = ~0ull;
    (void)cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  (void)cudaGetLastError();
}

void* Context::alloc(size_t bytes) {
  void* p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, bytes, stream);
  if (e != cudaSuccess) {  // give the pool's cached memory back and retry once
    (void)cudaGetLastError();
    cudaStreamSynchronize(stream);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    e = cudaMallocAsync(&p, bytes, stream);
  }
  cuda_check(e, "device allocation");
  return p;
}

void Context::release(void* p) {
  if (p) cudaFreeAsync(p, stream);
}

Context& Context::get(int dev) {
  static std::mutex mu;
  static std::map<int, Context*> all;  // lives until exit, like the device itself
  std::lock_guard<std::mutex> lk(mu);
  auto it = all.find(dev);
  if (it == all.end()) it = all.emplace(dev, new Context(dev)).first;
  it->second->activate();
  return *it->second;
}

void Context::activate() const { cuda_check(cudaSetDevice(device), "cudaSetDevice"); }

const double* Context::fetch(const double* dev, int n) {
  if (n > kHost) throw std::invalid_argument("qkrylov_b200: fetch too large");
  cuda_check(cudaMemcpyAsync(host, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, stream), "fetch");
  cuda_check(cudaStreamSynchronize(stream), "fetch sync");
  return host;
}

void Context::sync() { cuda_check(cudaStreamSynchronize(stream), "stream sync"); }

DevVec::DevVec(size_t n, qk_dtype t, int device, bool zero) : n_(n), t_(t), dev_(device) {
  if (n == 0) return;
  Context& c = Context::get(device);
  p_ = c.alloc(bytes());
  if (zero) cuda_check(cudaMemsetAsync(p_, 0, bytes(), c.stream), "memset");
}

DevVec::~DevVec() {
  if (p_) Context::get(dev_).release(p_);
}

DevVec& DevVec::operator=(DevVec&& o) noexcept {
  if (this != &o) {
    if (p_) Context::get(dev_).release(p_);
    p_ = o.p_; n_ = o.n_; t_ = o.t_; dev_ = o.dev_;
    o.p_ = nullptr; o.n_ = 0;
  }
  return *this;
}

PtrArray::PtrArray(size_t cap, int device) : h_(cap, nullptr), cap_(cap) {
  Context::get(device);
  cuda_check(cudaMalloc(reinterpret_cast<void**>(&d_), sizeof(void*) * cap), "pointer array");
}

PtrArray::~PtrArray() { cudaFree(d_); }

void PtrArray::set(size_t i, const void* p, cudaStream_t s) {
  if (i >= cap_) throw std::out_of_range("qkrylov_b200: pointer array");
  h_[i] = p;
  // h_ outlives the copy: the element stays valid until overwritten.
  cuda_check(cudaMemcpyAsync(d_ + i, &h_[i], sizeof(void*), cudaMemcpyHostToDevice, s), "pointer upload");
}

}  // namespace qkb
