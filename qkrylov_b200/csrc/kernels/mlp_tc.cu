// Tensor-core forward pass of the warm-start MLP (inference over a basis):
// tcgen05.mma on the 5th-generation tensor cores with BF16 operands in
// shared memory and FP32 accumulators in tensor memory (TMEM).
//
// A persistent CTA (one per SM) holds the weights in shared memory once and
// runs four independent warpgroups of 128 threads.  Each warpgroup owns an
// activation tile, an mbarrier, 128 of the SM's 512 TMEM columns and its
// own named barrier, and works through tiles of 128 states (one thread per
// tile row):
//   X (128 x K1, BF16: spins as +-1, J2, zero padding) -> smem
//   D1 = X W1^T          (TMEM, FP32)                    tcgen05.mma, K1/16 steps
//   H1 = GELU(D1 + b1)   -> BF16 -> smem (overwrites X)  tcgen05.ld by row
//   D2 = H1 W2^T         (same TMEM columns)             tcgen05.mma, 8 steps
//   o  = W3 GELU(D2 + b2) + b3                           FP32 on the CUDA cores
// D1 has been read out of TMEM before the second product is issued, so one
// 128-column range serves both.  While one warpgroup waits on its MMAs the
// others run their GELU epilogues: the activation of 256 values per state
// (tanh form, two special-function ops each), not the 20 K multiply-adds per
// state, is the bulk of the work.
// Operands use the canonical K-major layout without swizzle: 8-row x
// 16-byte core matrices, core matrices along K 128 bytes apart (leading
// byte offset), 8-row groups K/8 * 128 bytes apart (stride byte offset).
// Each thread writes its row eight columns (one 16-byte core-matrix row)
// at a time.  One thread per warpgroup issues its MMAs and commits them to
// the warpgroup's mbarrier (a commit tracks the MMAs of the issuing
// thread); every wait on it is bounded (on expiry the warpgroup records an
// error and stops).  Activations are rounded to BF16 before each product,
// weights are BF16, accumulation is FP32.
#include <cuda_bf16.h>

#include <algorithm>

#include "reduce.cuh"

namespace qkd {
namespace {

constexpr int kTcRows = 128, kHid = 128, kGroups = 4, kTcThreads = kGroups * kTcRows, kTmemCols = 512;
constexpr uint32_t kWaitLimit = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (row, k) in a canonical K-major tile with K columns
__device__ __forceinline__ uint32_t kmaj_off(uint32_t row, uint32_t k, uint32_t K) {
  return (row >> 3) * (K / 8) * 128 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// shared-memory matrix descriptor: start, LBO, SBO in 16-byte units,
// descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= uint64_t((addr >> 4) & 0x3FFFu);
  d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46;
  return d;
}

// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(dtmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
  for (uint32_t it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
  #pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// eight BF16 values as one 16-byte core-matrix row
__device__ __forceinline__ uint4 pack8(const float* v) {
  uint4 q;
  uint32_t* w = reinterpret_cast<uint32_t*>(&q);
  #pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    w[i] = *reinterpret_cast<const uint32_t*>(&h);
  }
  return q;
}

// barrier over the 128 threads of warpgroup g (named barrier 1 + g); true
// when any of them passes true
__device__ __forceinline__ bool group_sync_or(int g, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.b32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, %3, p;\n\t"
      "selp.b32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"(uint32_t(v)), "r"(1 + g), "r"(kTcRows)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void group_sync(int g) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(kTcRows) : "memory");
}

// The network's activation (tanh form of GELU, as in training), with
// tanh(u) = 1 - 2 / (1 + e^(2u)): two special-function operations (the
// exponential and the reciprocal, each within a few ulps) and five FMAs per
// value instead of an erf evaluation.  |error| stays around 1e-7 for all u
// (e^(2u) overflows to infinity, giving 1, and underflows to 0, giving -1),
// so the BF16 rounding of the activations that follows sees the value the
// FP64 oracle computes.
__device__ __forceinline__ float gelu(float z) {
  const float u = 0.79788456080286536f * z * fmaf(0.044715f * z, z, 1.f);
  const float e = exp2f(2.8853900817779268f * u);  // e^(2u), 2 log2(e) u
  const float t = 1.f - __fdividef(2.f, 1.f + e);
  const float hz = 0.5f * z;
  return fmaf(hz, t, hz);
}

struct TcArgs {
  int n, nsites, k1;          // states, sites, padded input width (32 or 64)
  const uint64_t* states;
  float j2;
  const __nv_bfloat16* w1;    // [128][nsites+1]
  const __nv_bfloat16* w2;    // [128][128]
  const __nv_bfloat16* w3;    // [2][128]
  const float *b1, *b2, *b3;
  float* out;                 // [n][2]
  int* err;                   // set when an mbarrier wait expires
};

__global__ void __launch_bounds__(kTcThreads, 1) k_mlp_fwd_tc(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* sW2 = smem;                              // 128 x 128 BF16, 32 KB
  unsigned char* sW1 = sW2 + kHid * kHid * 2;             // 128 x k1 BF16, 8 or 16 KB
  __shared__ float s_b1[kHid], s_b2[kHid], s_w3[2 * kHid];
  __shared__ __align__(8) uint64_t s_mbar[kGroups];
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int g = tid / kTcRows, t = tid % kTcRows;         // warpgroup, tile row
  const int k1 = a.k1, ki = a.nsites + 1;
  unsigned char* sA = sW1 + kHid * k1 * 2 + g * (kTcRows * kHid * 2);  // this group's 128 x 128 BF16 tile
  // weights into shared memory, canonical K-major layouts
  for (int i = tid; i < kHid * k1; i += kTcThreads) {
    const int r = i / k1, k = i % k1;
    const __nv_bfloat16 v = k < ki ? a.w1[r * ki + k] : __float2bfloat16(0.f);
    *reinterpret_cast<__nv_bfloat16*>(sW1 + kmaj_off(r, k, k1)) = v;
  }
  for (int i = tid; i < kHid * kHid; i += kTcThreads) {
    const int r = i / kHid, k = i % kHid;
    *reinterpret_cast<__nv_bfloat16*>(sW2 + kmaj_off(r, k, kHid)) = a.w2[i];
  }
  for (int i = tid; i < kHid; i += kTcThreads) { s_b1[i] = a.b1[i]; s_b2[i] = a.b2[i]; }
  for (int i = tid; i < 2 * kHid; i += kTcThreads) s_w3[i] = __bfloat162float(a.w3[i]);
  if (tid < kGroups) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_mbar[tid])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {  // all 512 columns: 128 per warpgroup, D1 then D2
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem + uint32_t(g * kHid);     // this group's columns
  const uint32_t mbar = smem_u32(&s_mbar[g]);
  const uint32_t id = idesc_bf16(kTcRows, kHid);
  const uint32_t lane_base = uint32_t((warp % 4) * 32) << 16;  // a warp reaches TMEM lanes 32 (warp % 4) ..
  uint32_t phase = 0;
  bool ok = true;
  const int ntiles = (a.n + kTcRows - 1) / kTcRows;
  for (int tile = blockIdx.x * kGroups + g; tile < ntiles; tile += gridDim.x * kGroups) {
    const int row = tile * kTcRows + t;
    // X row of this thread, eight columns per store
    {
      const bool in = row < a.n;
      const uint64_t s = in ? a.states[row] : 0ull;
      for (int k0 = 0; k0 < k1; k0 += 8) {
        float v[8];
        #pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int k = k0 + i;
          v[i] = !in ? 0.f : k < a.nsites ? (((s >> k) & 1ull) ? 1.f : -1.f) : (k == a.nsites ? a.j2 : 0.f);
        }
        *reinterpret_cast<uint4*>(sA + kmaj_off(t, k0, k1)) = pack8(v);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // smem writes -> tensor core
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    group_sync(g);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (t == 0) {
      for (int kk = 0; kk < k1; kk += 16) {
        const uint64_t ad = sdesc(smem_u32(sA) + (kk / 8) * 128, 128, (k1 / 8) * 128);
        const uint64_t bd = sdesc(smem_u32(sW1) + (kk / 8) * 128, 128, (k1 / 8) * 128);
        mma_bf16(tmem, ad, bd, id, kk > 0);
      }
      mma_commit(mbar);
    }
    // every thread of the group waits on the commit; the group agrees on the
    // outcome before any thread leaves the loop, so its barriers stay matched
    if (group_sync_or(g, !mbar_wait(mbar, phase))) { ok = false; break; }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // H1 = GELU(D1 + b1) as BF16, row t, into the activation tile (K = 128)
    for (int c0 = 0; c0 < kHid; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + lane_base + uint32_t(c0), v);
      #pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = gelu(v[i] + s_b1[c0 + i]);
      *reinterpret_cast<uint4*>(sA + kmaj_off(t, c0, kHid)) = pack8(v);
      *reinterpret_cast<uint4*>(sA + kmaj_off(t, c0 + 8, kHid)) = pack8(v + 8);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    group_sync(g);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (t == 0) {
      for (int kk = 0; kk < kHid; kk += 16) {
        const uint64_t ad = sdesc(smem_u32(sA) + (kk / 8) * 128, 128, (kHid / 8) * 128);
        const uint64_t bd = sdesc(smem_u32(sW2) + (kk / 8) * 128, 128, (kHid / 8) * 128);
        mma_bf16(tmem, ad, bd, id, kk > 0);
      }
      mma_commit(mbar);
    }
    if (group_sync_or(g, !mbar_wait(mbar, phase))) { ok = false; break; }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    float o0 = 0.f, o1 = 0.f;
    for (int c0 = 0; c0 < kHid; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + lane_base + uint32_t(c0), v);
      #pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float h = gelu(v[i] + s_b2[c0 + i]);
        o0 = fmaf(s_w3[c0 + i], h, o0);
        o1 = fmaf(s_w3[kHid + c0 + i], h, o1);
      }
    }
    if (row < a.n) reinterpret_cast<float2*>(a.out)[row] = make_float2(o0 + a.b3[0], o1 + a.b3[1]);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    group_sync(g);  // the next tile overwrites the activation tile and the accumulator
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (!ok) {
    if (t == 0) atomicExch(a.err, 1);
    // the MMAs behind the expired wait may still be writing this group's
    // columns: one more bounded wait on their commit before the columns are
    // released (the host discards the results and reports the error either way)
    (void)mbar_wait(mbar, phase);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s_tmem), "r"(kTmemCols));
}

}  // namespace
}  // namespace qkd

using namespace qkd;

extern "C" int qkd_mlp_forward_tc(int n, int nsites, const uint64_t* states, float j2, const void* w1, const void* w2,
                                  const void* w3, const float* b1, const float* b2, const float* b3, float* out,
                                  int* err, cudaStream_t s) {
  if (n <= 0) return QKD_OK;
  if (!states || !w1 || !w2 || !w3 || !b1 || !b2 || !b3 || !out || !err || nsites < 1 || nsites > 62)
    return QKD_EINVAL;
  TcArgs a{n, nsites, nsites + 1 <= 32 ? 32 : 64, states, j2, static_cast<const __nv_bfloat16*>(w1),
           static_cast<const __nv_bfloat16*>(w2), static_cast<const __nv_bfloat16*>(w3), b1, b2, b3, out, err};
  const size_t smem = size_t(kHid) * kHid * 2 + size_t(kHid) * a.k1 * 2 + size_t(kGroups) * kTcRows * kHid * 2;
  if (cudaFuncSetAttribute(k_mlp_fwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) {
    (void)cudaGetLastError();
    return QKD_EINVAL;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  const int tiles = (n + kTcRows - 1) / kTcRows;
  // one CTA per SM: 168-176 KB of shared memory leave room for no second
  // one, so the 512-column TMEM allocation never waits
  const int grid = std::max(1, std::min((tiles + kGroups - 1) / kGroups, sm_count(dev)));
  k_mlp_fwd_tc<<<grid, kTcThreads, smem, s>>>(a);
  QKD_LAUNCH_CHECK();
  return QKD_OK;
}
