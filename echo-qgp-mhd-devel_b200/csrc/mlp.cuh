// mlp.cuh -- the learned con2prim seed for ideal RMHD.
//
// A 4x64 tanh MLP maps five normalised invariants of the conserved state
//   f0 = log U, f1 = D/U, f2 = S^2/U^2, f3 = B^2/U, f4 = (S.B)^2/U^3
// (U = energy, D = density, S = momentum, B = field, all already divided by
// sqrt(-g); the same quantities BRENTM's system sist3 is written in) to the
// two unknowns x = v^2 and q = p/U.  The third unknown y = (e+p)gamma^2
// follows from the EoS (sist3's third equation).  The seed is finished by
// the FP64 Newton solve on sist3; it is never used on its own.
//
// Inference runs per CTA of 128 threads, one cell per thread, on the
// fifth-generation tensor cores: every layer is one M=128 tcgen05.mma chain
// (BF16 operands from shared memory in the canonical no-swizzle K-major
// layout, FP32 accumulators in tensor memory).  Thread t of the CTA owns row
// t of the tile and of the accumulator (TMEM lane t), so bias, tanh and the
// BF16 repacking of the next layer's input happen in the thread's registers
// after one tcgen05.ld of its row.
#pragma once

#include <cuda_bf16.h>

#include "physics.cuh"

namespace echo {

enum { MLP_NIN = 5, MLP_H = 64, MLP_NOUT = 2, MLP_NHID = 4 };

// Weights: one BF16 image per layer in the canonical K-major layout of a
// tcgen05 B operand (core matrices of 8 rows x 16 bytes; rows n of W^T, K
// contiguous): element (n, k) at byte (k/8)*LBO + (n/8)*128 + (n%8)*16 +
// (k%8)*2 with LBO = (N/8)*128.  Layer 0 is K=16 (5 inputs, zero padded) x
// N=64, layers 1..3 64 x 64, the output layer 64 x N=16 (2 outputs).  Offsets
// and sizes in bytes; MLP_FRAG_N in u32.
enum {
  MLP_IMG_L0 = 0,
  MLP_IMG_L1 = MLP_IMG_L0 + 16 * 64 * 2,
  MLP_IMG_L2 = MLP_IMG_L1 + 64 * 64 * 2,
  MLP_IMG_L3 = MLP_IMG_L2 + 64 * 64 * 2,
  MLP_IMG_L4 = MLP_IMG_L3 + 64 * 64 * 2,
  MLP_IMG_BYTES = MLP_IMG_L4 + 64 * 16 * 2,
  MLP_FRAG_N = MLP_IMG_BYTES / 4
};
// biases and normalisation, FP32: b0..b3 (64 each), b4 (8, two used),
// feature mean/std (5+5), target mean/std (2+2)
enum {
  MLP_B0 = 0,
  MLP_B4 = 4 * 64,
  MLP_FMEAN = MLP_B4 + 8,
  MLP_FSTD = MLP_FMEAN + 5,
  MLP_TMEAN = MLP_FSTD + 5,
  MLP_TSTD = MLP_TMEAN + 2,
  MLP_PARAMS_N = MLP_TSTD + 2
};

struct MlpDev {
  const unsigned* __restrict__ frag;  // MLP_FRAG_N u32
  const float* __restrict__ par;      // MLP_PARAMS_N floats
};

// raw invariants of the cell (before standardisation)
__device__ __forceinline__ void mlp_invariants(double D, double SS2, double U, double B2, double SB2, float f[5]) {
  double iu = 1.0 / U;
  f[0] = (float)log(U);
  f[1] = (float)(D * iu);
  f[2] = (float)(SS2 * iu * iu);
  f[3] = (float)(B2 * iu);
  f[4] = (float)(SB2 * iu * iu * iu);
}

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<unsigned*>(&h);
}

// tanh of two FP32 accumulators, packed as the BF16 pair the next layer's A
// fragment takes: one conversion and one packed tanh
__device__ __forceinline__ unsigned tanh_pack_bf16(float lo, float hi) {
  unsigned p = pack_bf16(lo, hi), y;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(y) : "r"(p));
  return y;
}

// ---------------------------------------------------------------------------
// tcgen05 plumbing (PTX ISA: tcgen05.alloc/mma/commit/ld, mbarrier)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle, K-major: start address,
// leading byte offset (between the two 8-element K halves of a K=16 step)
// and stride byte offset (between 8-row core-matrix groups), version 1
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}
// instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N
__host__ __device__ constexpr uint32_t umma_idesc(int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// bounded wait for the phase of the given parity: false if it never came
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int i = 0; i < (1 << 20); i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// one thread: the bulk copy (TMA engine) of `bytes` from global memory into
// shared memory, completing on mbarrier `bar` (which expects the bytes)
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// the calling thread's TMEM lane, columns [col, col + 16)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}

// ---------------------------------------------------------------------------
// Seed of the calling thread's cell.  Called by all 128 threads of the CTA
// together (blockDim.x == 128; threads without a cell pass any finite
// features).  f: raw invariants; out: (x, q) de-standardised.  A tensor-core
// wait that never completes (bounded) leaves out = NaN, which the seeded
// Newton treats as a failed seed (the plain Newton then runs).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mlp_cta(const MlpDev& M, const float f[5], float out[2]) {
  __shared__ __align__(1024) uint4 s_act[128 * 64 * 2 / 16];   // 16 KB: the 128 x K activation tile
  __shared__ __align__(1024) uint4 s_w[2][64 * 64 * 2 / 16];   // 2 x 8 KB: weight images, double-buffered
  __shared__ __align__(8) unsigned long long s_bar[3];         // [0]: MMA done, [1], [2]: weights landed
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;  // a weight copy that never landed
  const int tid = threadIdx.x, warp = tid >> 5;
  unsigned char* act = reinterpret_cast<unsigned char*>(s_act);
  const unsigned char* img = reinterpret_cast<const unsigned char*>(M.frag);
  const uint32_t bar = smem_addr(&s_bar[0]);
  auto layer_img = [](int layer) {
    return layer == 0 ? (int)MLP_IMG_L0 : layer == 4 ? (int)MLP_IMG_L4 : (int)MLP_IMG_L1 + (layer - 1) * (64 * 64 * 2);
  };
  auto layer_bytes = [](int layer) { return layer == 0 || layer == 4 ? 2048u : 8192u; };
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                 "r"(64u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    s_fail = 0;
    for (int i = 0; i < 3; i++) asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(&s_bar[i])), "r"(1u));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    // the first two layers' weights, while the features are computed
    for (int l = 0; l < 2; l++)
      bulk_load(smem_addr(&s_w[l][0]), img + layer_img(l), layer_bytes(l), smem_addr(&s_bar[1 + l]));
  }
  // layer-0 input: the standardised invariants in columns 0..4 of 16
  {
    float fs[8];
#pragma unroll
    for (int j = 0; j < 5; j++) fs[j] = (f[j] - __ldg(M.par + MLP_FMEAN + j)) / __ldg(M.par + MLP_FSTD + j);
    fs[5] = fs[6] = fs[7] = 0.f;
    uint4 lo = make_uint4(pack_bf16(fs[0], fs[1]), pack_bf16(fs[2], fs[3]), pack_bf16(fs[4], fs[5]),
                          pack_bf16(fs[6], fs[7]));
    const int row_off = (tid >> 3) * 128 + (tid & 7) * 16;
    *reinterpret_cast<uint4*>(act + row_off) = lo;                                    // k 0..7
    *reinterpret_cast<uint4*>(act + 2048 + row_off) = make_uint4(0u, 0u, 0u, 0u);     // k 8..15
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t my_lane = tmem + ((uint32_t)(warp * 32) << 16);
  bool ok = true;
  float y0 = 0.f, y1 = 0.f;
#pragma unroll 1
  for (int layer = 0; layer < 5; layer++) {
    const int K = layer == 0 ? 16 : 64, N = layer == 4 ? 16 : 64, buf = layer & 1;
    // generic-proxy smem writes (this layer's input) -> visible to the
    // tensor core; TMEM reads of the previous layer done before overwrite
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      bool w_ok = mbar_wait(smem_addr(&s_bar[1 + buf]), (uint32_t)((layer >> 1) & 1));
      const uint32_t lbo_b = (uint32_t)(N / 8) * 128;
      const uint32_t wbase = smem_addr(&s_w[buf][0]);
      if (w_ok)
        for (int j = 0; j < K / 16; j++)
          umma_bf16(tmem, umma_desc(smem_addr(act + j * 2 * 2048), 2048, 128), umma_desc(wbase + j * 2 * lbo_b, lbo_b, 128),
                    umma_idesc(N), j > 0 ? 1u : 0u);
      umma_commit(bar);  // arrives when the MMAs above are done (at once if none was issued)
      if (!w_ok) s_fail = 1;
    }
    ok = mbar_wait(bar, (uint32_t)(layer & 1)) && ok;
    tc_fence_after();
    // the weights of layer + 2 into the buffer this layer's MMAs have released
    if (tid == 0 && layer + 2 < 5)
      bulk_load(smem_addr(&s_w[buf][0]), img + layer_img(layer + 2), layer_bytes(layer + 2), smem_addr(&s_bar[1 + buf]));
    if (layer < 4) {
      const float* b = M.par + MLP_B0 + layer * 64;
      const int row_off = (tid >> 3) * 128 + (tid & 7) * 16;
#pragma unroll
      for (int q = 0; q < 4; q++) {  // columns 16q .. 16q+15 -> K chunks 2q, 2q+1 of the next input
        float v[16];
        tmem_ld16(my_lane + 16 * q, v);
        uint32_t p[8];
#pragma unroll
        for (int j = 0; j < 8; j++)
          p[j] = tanh_pack_bf16(v[2 * j] + __ldg(b + 16 * q + 2 * j), v[2 * j + 1] + __ldg(b + 16 * q + 2 * j + 1));
        *reinterpret_cast<uint4*>(act + (2 * q) * 2048 + row_off) = make_uint4(p[0], p[1], p[2], p[3]);
        *reinterpret_cast<uint4*>(act + (2 * q + 1) * 2048 + row_off) = make_uint4(p[4], p[5], p[6], p[7]);
      }
    } else {
      float v[16];
      tmem_ld16(my_lane, v);
      y0 = v[0] + __ldg(M.par + MLP_B4 + 0);
      y1 = v[1] + __ldg(M.par + MLP_B4 + 1);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64u));
  }
  if (ok && !s_fail) {
    out[0] = y0 * __ldg(M.par + MLP_TSTD + 0) + __ldg(M.par + MLP_TMEAN + 0);
    out[1] = y1 * __ldg(M.par + MLP_TSTD + 1) + __ldg(M.par + MLP_TMEAN + 1);
  } else {
    out[0] = out[1] = __int_as_float(0x7fc00000);
  }
}

}  // namespace echo
