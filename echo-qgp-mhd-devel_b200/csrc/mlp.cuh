// mlp.cuh -- the learned con2prim seed for ideal and resistive RMHD.
//
// A 4x64 tanh MLP maps six normalised invariants of the conserved state
//   f0 = log U, f1 = D/U, f2 = S^2/U^2, f3 = B^2/U, f4 = (S.B)^2/U^3,
//   f5 = E^2/U (zero for ideal RMHD, where E is not a conserved variable)
// (U = energy, D = density, S = momentum, B = field, E = electric field,
// all already divided by sqrt(-g); the quantities BRENTM's system sist3 is
// written in) to the two unknowns x = v^2 and q = p/U.  For ideal RMHD the
// third unknown y = (e+p)gamma^2 follows from the EoS (sist3's third
// equation) and the seed is finished by the FP64 Newton solve on sist3; for
// resistive RMHD p starts the fixed point's inner Newton (cons2prim_res).
// The seed is never used on its own.
//
// Inference runs per warp (32 cells) on the tensor cores: BF16 operands,
// FP32 accumulation, mma.sync.m16n8k16.  The accumulator fragment of an
// m16n8 tile holds, per thread, rows (g, g+8) and columns (2t, 2t+1) -- the
// same elements the A fragment of an m16n8k16 operand holds for the k-tile
// that covers those columns -- so one layer's output becomes the next
// layer's input in registers, with no shuffles or shared memory.
#pragma once

#include <cuda_bf16.h>

#include "physics.cuh"

namespace echo {

enum { MLP_NIN = 6, MLP_H = 64, MLP_NOUT = 2, MLP_NHID = 4 };

// Weight fragments (u32 = two bf16) in the order the mma B operand needs:
// layer 0: [k-tile 0][n-tile 0..7][lane][2]; layers 1..3: [kt 0..3][nt 0..7]
// [lane][2]; layer 4: [kt 0..3][nt 0][lane][2].
enum {
  MLP_FRAG_L0 = 0,
  MLP_FRAG_L1 = MLP_FRAG_L0 + 1 * 8 * 64,
  MLP_FRAG_L2 = MLP_FRAG_L1 + 4 * 8 * 64,
  MLP_FRAG_L3 = MLP_FRAG_L2 + 4 * 8 * 64,
  MLP_FRAG_L4 = MLP_FRAG_L3 + 4 * 8 * 64,
  MLP_FRAG_N = MLP_FRAG_L4 + 4 * 1 * 64
};
// biases and normalisation, FP32: b0..b3 (64 each), b4 (8, two used),
// feature mean/std (6+6), target mean/std (2+2)
enum {
  MLP_B0 = 0,
  MLP_B4 = 4 * 64,
  MLP_FMEAN = MLP_B4 + 8,
  MLP_FSTD = MLP_FMEAN + MLP_NIN,
  MLP_TMEAN = MLP_FSTD + MLP_NIN,
  MLP_TSTD = MLP_TMEAN + 2,
  MLP_PARAMS_N = MLP_TSTD + 2
};

struct MlpDev {
  const unsigned* __restrict__ frag;  // MLP_FRAG_N u32
  const float* __restrict__ par;      // MLP_PARAMS_N floats
};

// raw invariants of the cell (before standardisation)
__device__ __forceinline__ void mlp_invariants(double D, double SS2, double U, double B2, double SB2, double E2,
                                               float f[MLP_NIN]) {
  double iu = 1.0 / U;
  f[0] = (float)log(U);
  f[1] = (float)(D * iu);
  f[2] = (float)(SS2 * iu * iu);
  f[3] = (float)(B2 * iu);
  f[4] = (float)(SB2 * iu * iu * iu);
  f[5] = (float)(E2 * iu);
}

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<unsigned*>(&h);
}

__device__ __forceinline__ void mma_bf16(float c[4], const unsigned a[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// tanh of two FP32 accumulators, packed as the BF16 pair the next layer's A
// fragment takes: one conversion and one packed tanh
__device__ __forceinline__ unsigned tanh_pack_bf16(float lo, float hi) {
  unsigned p = pack_bf16(lo, hi), y;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(y) : "r"(p));
  return y;
}

// Seed for the calling lane's cell.  Must be called by all 32 lanes of the
// warp together (inactive lanes pass any finite features).  f: raw
// invariants; out: (x, q) de-standardised.  The warp's 32 cells are two
// m-tiles of 16 rows, run one after the other so that only one tile's
// accumulators (32 registers) and A fragments (16) are live.
__device__ __forceinline__ void mlp_warp(const MlpDev& M, const float f[MLP_NIN], float out[2]) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float fs[MLP_NIN];
#pragma unroll
  for (int j = 0; j < MLP_NIN; j++) fs[j] = (f[j] - __ldg(M.par + MLP_FMEAN + j)) / __ldg(M.par + MLP_FSTD + j);
  // row r = mt*16 + h*8 + g' of the output sits in lane g'*4 (t = 0), element 2h / 2h+1
  const int mt_me = lane >> 4, h_me = (lane >> 3) & 1, src = (lane & 7) * 4;
  float y0 = 0.f, y1 = 0.f;
#pragma unroll 1
  for (int mt = 0; mt < 2; mt++) {
    // layer-0 A fragment (16 input columns, 6 used): rows g and g + 8 of this tile
    unsigned A[4][4];  // [k-tile][reg]
    {
      float lo[MLP_NIN], hi[MLP_NIN];
#pragma unroll
      for (int j = 0; j < MLP_NIN; j++) {
        lo[j] = __shfl_sync(full, fs[j], mt * 16 + g);
        hi[j] = __shfl_sync(full, fs[j], mt * 16 + g + 8);
      }
      // columns 2t and 2t+1
      float l0 = t == 0 ? lo[0] : t == 1 ? lo[2] : t == 2 ? lo[4] : 0.f;
      float l1 = t == 0 ? lo[1] : t == 1 ? lo[3] : t == 2 ? lo[5] : 0.f;
      float h0 = t == 0 ? hi[0] : t == 1 ? hi[2] : t == 2 ? hi[4] : 0.f;
      float h1 = t == 0 ? hi[1] : t == 1 ? hi[3] : t == 2 ? hi[5] : 0.f;
      A[0][0] = pack_bf16(l0, l1);
      A[0][1] = pack_bf16(h0, h1);
      A[0][2] = 0u;
      A[0][3] = 0u;
    }
    // hidden layers 0..3
#pragma unroll
    for (int layer = 0; layer < 4; layer++) {
      const int nk = layer == 0 ? 1 : 4;
      const unsigned* W = M.frag + (layer == 0 ? MLP_FRAG_L0 : MLP_FRAG_L1 + (layer - 1) * (4 * 8 * 64));
      const float* b = M.par + MLP_B0 + layer * 64;
      float C[8][4];
#pragma unroll
      for (int nt = 0; nt < 8; nt++) {
        float b0 = __ldg(b + nt * 8 + 2 * t), b1 = __ldg(b + nt * 8 + 2 * t + 1);
        C[nt][0] = b0;
        C[nt][1] = b1;
        C[nt][2] = b0;
        C[nt][3] = b1;
      }
#pragma unroll
      for (int kt = 0; kt < 4; kt++) {
        if (kt >= nk) break;
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
          const uint2 w = __ldg(reinterpret_cast<const uint2*>(W) + (kt * 8 + nt) * 32 + lane);
          mma_bf16(C[nt], A[kt], w.x, w.y);
        }
      }
      // tanh; the accumulators become the next layer's A fragments
#pragma unroll
      for (int kt = 0; kt < 4; kt++) {
        A[kt][0] = tanh_pack_bf16(C[2 * kt][0], C[2 * kt][1]);
        A[kt][1] = tanh_pack_bf16(C[2 * kt][2], C[2 * kt][3]);
        A[kt][2] = tanh_pack_bf16(C[2 * kt + 1][0], C[2 * kt + 1][1]);
        A[kt][3] = tanh_pack_bf16(C[2 * kt + 1][2], C[2 * kt + 1][3]);
      }
    }
    // output layer: 64 -> 8 (two used), linear
    float O[4];
    {
      float b0 = __ldg(M.par + MLP_B4 + 2 * t), b1 = __ldg(M.par + MLP_B4 + 2 * t + 1);
      O[0] = b0;
      O[1] = b1;
      O[2] = b0;
      O[3] = b1;
#pragma unroll
      for (int kt = 0; kt < 4; kt++) {
        const uint2 w = __ldg(reinterpret_cast<const uint2*>(M.frag + MLP_FRAG_L4) + kt * 32 + lane);
        mma_bf16(O, A[kt], w.x, w.y);
      }
    }
    float a0 = __shfl_sync(full, O[0], src), a1 = __shfl_sync(full, O[1], src);
    float a2 = __shfl_sync(full, O[2], src), a3 = __shfl_sync(full, O[3], src);
    if (mt == mt_me) {
      y0 = h_me ? a2 : a0;
      y1 = h_me ? a3 : a1;
    }
  }
  out[0] = y0 * __ldg(M.par + MLP_TSTD + 0) + __ldg(M.par + MLP_TMEAN + 0);
  out[1] = y1 * __ldg(M.par + MLP_TSTD + 1) + __ldg(M.par + MLP_TMEAN + 1);
}

}  // namespace echo
