// Image-domain U-Net preconditioner on sm_100a: BF16 tensor-core convolution kernels (tcgen05
// with TMEM accumulators by default, mma.sync m16n8k16 as the checked alternative; FP32
// accumulate) for inference and training, with the host orchestration of the network, its Adam
// optimiser and its C ABI (include/ds2d.h, ds2d_unet_*).
//
// The reference has no learned component; the network approximates the inverse Hessian of the
// Born operator (maps an RTM image to reflectivity) and preconditions CG-LSRTM.  Architecture
// (identical to the FP64 oracle that checks it): 4-level encoder-decoder, base 32 channels,
// conv3x3 + ReLU pairs, 2x2 average pooling, nearest 2x upsampling, skip concatenation, 1x1 output
// convolution.  Activations and gradients are BF16 NHWC (channels last); weights keep an FP32
// master copy (Adam) and BF16 copies laid out [tap][cout][cin] for the forward product and
// [tap][cin][cout] (spatially flipped) for the backward-data product.
//
// Every 3x3 convolution, forward and both backward products, is an implicit GEMM on the tensor
// cores:
//   forward      out[p][co]  = sum_{tap,ci} in[p + tap][ci] * W[tap][co][ci]
//   backward     dx[p][ci]   = sum_{tap,co} dz[p - tap][co] * W[tap][co][ci]  (= forward with the
//                              flipped, transposed weights)
//   weight grad  dW[tap][co][ci] = sum_p dz[p][co] * x[p + tap][ci]   (K = pixels, split over CTAs)
#include <cuda.h>  // CUtensorMap and its enums (the encoder is fetched through the runtime)
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ds2d.h"

namespace {

using bf16 = __nv_bfloat16;

// ---------------------------------------------------------------------------------------------
// Tensor-core primitive: D = A(16x16, row) * B(16x8, col) + C, BF16 in, FP32 accumulate.
// Fragment ownership (lane = 4 g + t): A regs {(g,2t..), (g+8,2t..), (g,2t+8..), (g+8,2t+8..)};
// B regs {(k 2t.., n g), (k 2t+8.., n g)}; C {(g, 2t), (g, 2t+1), (g+8, 2t), (g+8, 2t+1)}.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void mma16816(float (&c)[4], const unsigned (&a)[4], unsigned b0,
                                         unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned ld32(const bf16 *p) {
  return *reinterpret_cast<const unsigned *>(p);
}

// ---------------------------------------------------------------------------------------------
// 3x3 'same' convolution as an implicit GEMM.  CTA tile: 32 pixels of one image row x kCo output
// channels; warps 2 (pixels) x kCo/32 (channels), each warp 16 pixels x 32 channels (4 MMA n-tiles).
// K loop: input channels in chunks of 16, 9 taps per chunk.  Staging through shared memory with a
// 24-half row stride (conflict-free 32-bit fragment loads).
// ---------------------------------------------------------------------------------------------
constexpr int kPx = 32;  // pixels per CTA tile
constexpr int kSS = 24;  // shared row stride in halves (16 channels + 8 pad)

struct ConvArgs {
  const bf16 *in;   // [N][H][W][cin]
  const bf16 *wt;   // [9][cout][cin]
  const float *bias;  // [cout] or null
  bf16 *out;        // [N][H][W][ocs], channels [oco, oco + cout)
  float *out_f32;   // optional FP32 copy, same indexing as out
  const bf16 *mask; // optional: out *= (mask > 0), mask [N][H][W][ocs] at the same channels
  int n, h, w, cin, cout, ocs, oco, relu;
};

template <int kCo>
__global__ void __launch_bounds__(64 * (kCo / 32)) k_conv3x3(ConvArgs a) {
  __shared__ __align__(16) bf16 s_in[3][kPx + 2][kSS];
  __shared__ __align__(16) bf16 s_w[9][kCo][kSS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wp = warp & 1, wc = warp >> 1;
  const int w0 = blockIdx.x * kPx, row = blockIdx.y;
  const int ngrp = a.cout / kCo;
  const int img = blockIdx.z / ngrp, co0 = (blockIdx.z % ngrp) * kCo;
  constexpr int kThreads = 64 * (kCo / 32);
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0.f;

  for (int ci0 = 0; ci0 < a.cin; ci0 += 16) {
    // input halo tile: 3 rows x 34 pixels x 16 channels (two 16-byte vectors per pixel)
    for (int i = tid; i < 3 * (kPx + 2) * 2; i += kThreads) {
      const int half = i & 1, px = (i >> 1) % (kPx + 2), r = (i >> 1) / (kPx + 2);
      const int hh = row + r - 1, ww = w0 + px - 1;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (hh >= 0 && hh < a.h && ww >= 0 && ww < a.w)
        v = *reinterpret_cast<const uint4 *>(
            a.in + (((long long)img * a.h + hh) * a.w + ww) * a.cin + ci0 + half * 8);
      *reinterpret_cast<uint4 *>(&s_in[r][px][half * 8]) = v;
    }
    // weights: 9 taps x kCo couts x 16 channels
    for (int i = tid; i < 9 * kCo * 2; i += kThreads) {
      const int half = i & 1, co = (i >> 1) % kCo, tap = (i >> 1) / kCo;
      const uint4 v = *reinterpret_cast<const uint4 *>(
          a.wt + ((long long)tap * a.cout + co0 + co) * a.cin + ci0 + half * 8);
      *reinterpret_cast<uint4 *>(&s_w[tap][co][half * 8]) = v;
    }
    __syncthreads();
#pragma unroll
    for (int tap = 0; tap < 9; tap++) {
      const int ky = tap / 3, kx = tap % 3;
      const int p = wp * 16 + g + kx;
      unsigned fa[4];
      fa[0] = ld32(&s_in[ky][p][2 * t]);
      fa[1] = ld32(&s_in[ky][p + 8][2 * t]);
      fa[2] = ld32(&s_in[ky][p][2 * t + 8]);
      fa[3] = ld32(&s_in[ky][p + 8][2 * t + 8]);
#pragma unroll
      for (int nt = 0; nt < 4; nt++) {
        const int co = wc * 32 + nt * 8 + g;
        mma16816(acc[nt], fa, ld32(&s_w[tap][co][2 * t]), ld32(&s_w[tap][co][2 * t + 8]));
      }
    }
    __syncthreads();
  }
  // epilogue: bias, ReLU, mask, BF16 (and optional FP32) store
#pragma unroll
  for (int nt = 0; nt < 4; nt++) {
    const int co = co0 + wc * 32 + nt * 8 + 2 * t;
    const float b0 = a.bias ? a.bias[co] : 0.f, b1 = a.bias ? a.bias[co + 1] : 0.f;
#pragma unroll
    for (int hlf = 0; hlf < 2; hlf++) {
      const int ww = w0 + wp * 16 + g + 8 * hlf;
      if (ww >= a.w) continue;
      float v0 = acc[nt][2 * hlf] + b0, v1 = acc[nt][2 * hlf + 1] + b1;
      if (a.relu) {
        v0 = fmaxf(v0, 0.f);
        v1 = fmaxf(v1, 0.f);
      }
      const long long o = (((long long)img * a.h + row) * a.w + ww) * a.ocs + a.oco + co;
      if (a.mask) {
        const __nv_bfloat162 m = *reinterpret_cast<const __nv_bfloat162 *>(a.mask + o);
        if (!(__bfloat162float(m.x) > 0.f)) v0 = 0.f;
        if (!(__bfloat162float(m.y) > 0.f)) v1 = 0.f;
      }
      *reinterpret_cast<__nv_bfloat162 *>(a.out + o) = __floats2bfloat162_rn(v0, v1);
      if (a.out_f32) {
        a.out_f32[o] = v0;
        a.out_f32[o + 1] = v1;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------
// The same 3x3 convolution on the 5th-generation tensor cores (tcgen05, accumulators in TMEM).
// CTA: 128 threads, tile M = 128 consecutive output pixels of one image row x N output channels;
// K loop: input-channel chunks of 16, 9 taps per chunk, one UMMA (M 128, N, K 16) per tap issued by
// one thread.  Operands sit in shared memory in the canonical K-major no-swizzle layout: 8-row core
// matrices of 16 bytes per row, rows 16 bytes apart (SBO = 128 B between 8-row groups), the two
// 8-channel halves of a 16-channel chunk in separate planes (LBO = plane stride).  With rows
// uniformly 16 bytes apart, the tap shift kx is a 16-byte offset of the descriptor's start
// address, so one staged halo row serves all three kx taps.  The accumulator tile (128 lanes x N
// FP32 columns) is read back with tcgen05.ld by the warp owning each 32-lane quarter.
// ---------------------------------------------------------------------------------------------
constexpr int kTcM = 128;              // pixels per CTA (UMMA M)
constexpr int kTcHalo = kTcM + 2;      // halo pixels per staged row
constexpr int kTcPlaneA = kTcHalo * 16;  // bytes of one (row, channel-half) plane
constexpr int kTcSpin = 1 << 24;       // bound on every mbarrier wait

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major, no swizzle (SM100 descriptor version 1).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// Instruction descriptor: BF16 x BF16 -> FP32, both K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// kR output rows per CTA (1, 2 or 4): the staged weights of a chunk serve kR rows of pixels
// (kR + 2 halo rows staged, one accumulator tile of kN TMEM columns per row), so the weight
// staging per output pixel falls as 1 / kR and the halo rows' as (kR + 2) / (3 kR).
template <int kN, int kR = 1>
__global__ void __launch_bounds__(128) k_conv3x3_tc(ConvArgs a, int *err) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  // layout: A planes [kR + 2 rows][2 halves][130 px][16 B], B planes [9 taps][2 halves][kN][16 B]
  unsigned char *sA = tc_smem;
  unsigned char *sB = tc_smem + (kR + 2) * 2 * kTcPlaneA;
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int w0 = blockIdx.x * kTcM, row0 = blockIdx.y * kR;
  const int ngrp = a.cout / kN;
  const int img = blockIdx.z / ngrp, co0 = (blockIdx.z % ngrp) * kN;
  // TMEM columns: a power of two >= 32 holding kR accumulator tiles of kN columns
  constexpr uint32_t kCols = kR * kN <= 32 ? 32 : kR * kN <= 64 ? 64 : kR * kN <= 128 ? 128
                           : kR * kN <= 256 ? 256 : 512;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_base)), "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar)));
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = tmem_base;
  constexpr uint32_t idesc = umma_idesc(kTcM, kN);
  const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB);
  bool ok = true;
  int phase = 0;
  for (int ci0 = 0; ci0 < a.cin && ok; ci0 += 16) {
    // stage the kR + 2 halo rows: pixel px of row ky, channel half kh -> plane (ky, kh)
    for (int i = tid; i < (kR + 2) * 2 * kTcHalo; i += 128) {
      const int px = i % kTcHalo, kh = (i / kTcHalo) & 1, ky = i / (2 * kTcHalo);
      const int hh = row0 + ky - 1, ww = w0 + px - 1;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (hh >= 0 && hh < a.h && ww >= 0 && ww < a.w)
        v = *reinterpret_cast<const uint4 *>(
            a.in + (((long long)img * a.h + hh) * a.w + ww) * a.cin + ci0 + kh * 8);
      *reinterpret_cast<uint4 *>(sA + (ky * 2 + kh) * kTcPlaneA + px * 16) = v;
    }
    // stage the weights: tap, half, cout row
    for (int i = tid; i < 9 * 2 * kN; i += 128) {
      const int co = i % kN, kh = (i / kN) & 1, tap = i / (2 * kN);
      const uint4 v = *reinterpret_cast<const uint4 *>(
          a.wt + ((long long)tap * a.cout + co0 + co) * a.cin + ci0 + kh * 8);
      *reinterpret_cast<uint4 *>(sB + (tap * 2 + kh) * (kN * 16) + co * 16) = v;
    }
    // generic-proxy writes -> visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
#pragma unroll
      for (int j = 0; j < kR; j++)
#pragma unroll
        for (int tap = 0; tap < 9; tap++) {
          const int ky = tap / 3, kx = tap % 3;
          const uint64_t ad =
              umma_desc(a_base + ((j + ky) * 2) * kTcPlaneA + kx * 16, kTcPlaneA, 128);
          const uint64_t bd = umma_desc(b_base + (tap * 2) * (kN * 16), kN * 16, 128);
          const uint32_t acc = (ci0 > 0 || tap > 0) ? 1u : 0u;
          asm volatile(
              "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
                  tmem + (uint32_t)(j * kN)),
              "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
        }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          smem_u32(&mbar)));
    }
    // every thread waits until the MMAs of this chunk have read shared memory and finished
    uint32_t done = 0;
    for (int spin = 0; spin < kTcSpin && !done; spin++) {
      asm volatile(
          "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
          "selp.u32 %0, 1, 0, p;\n}\n"
          : "=r"(done)
          : "r"(smem_u32(&mbar)), "r"(phase)
          : "memory");
    }
    if (!done) {
      ok = false;
      if (tid == 0) atomicExch(err, 1);
    }
    phase ^= 1;
    __syncthreads();
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  for (int j = 0; j < kR && ok; j++) {
    // epilogue of output row row0 + j: thread (warp w, lane l) owns output pixel 32 w + l, reads
    // 8 columns of the row's accumulator tile at a time
    const int row = row0 + j;
    const int m = warp * 32 + lane;
    const int ww = w0 + m;
    const long long obase = (((long long)img * a.h + row) * a.w + ww) * a.ocs + a.oco + co0;
#pragma unroll 1
    for (int c0 = 0; c0 < kN; c0 += 8) {
      uint32_t r[8];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(j * kN + c0);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      if (ww < a.w && row < a.h) {
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
          v[j] = __uint_as_float(r[j]) + (a.bias ? a.bias[co0 + c0 + j] : 0.f);
          if (a.relu) v[j] = fmaxf(v[j], 0.f);
        }
        const long long o = obase + c0;
        if (a.mask) {
#pragma unroll
          for (int j = 0; j < 8; j++)
            if (!(__bfloat162float(a.mask[o + j]) > 0.f)) v[j] = 0.f;
        }
        __nv_bfloat162 p[4];
#pragma unroll
        for (int j = 0; j < 4; j++) p[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
        *reinterpret_cast<uint4 *>(a.out + o) = *reinterpret_cast<uint4 *>(p);
        if (a.out_f32) {
#pragma unroll
          for (int j = 0; j < 8; j++) a.out_f32[o + j] = v[j];
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kCols));
  }
}

// Dynamic shared memory of k_conv3x3_tc: the staged operands, raised where needed so that no more
// CTAs fit on an SM than its 512 TMEM columns hold (a CTA beyond that would wait in tcgen05.alloc
// holding an SM slot).
template <int kN, int kR = 1>
constexpr int tc_smem_bytes() {
  constexpr int kCols = kR * kN <= 32 ? 32 : kR * kN <= 64 ? 64 : kR * kN <= 128 ? 128
                      : kR * kN <= 256 ? 256 : 512;
  constexpr int operands = (kR + 2) * 2 * kTcPlaneA + 9 * 2 * kN * 16;
  constexpr int fit = 228 * 1024 / (512 / kCols + 1) + 2048;  // over (512 / kCols) CTAs per SM
  return operands > fit ? operands : fit;
}

// ---------------------------------------------------------------------------------------------
// The same convolution fed by the tensor-memory accelerator through a kS-stage ring (option
// "tcgen05_tma").  Per 16-channel chunk, one thread issues the tiled bulk-tensor loads of the
// kR + 2 halo rows (box: 8 channels x 130 pixels per channel half, out-of-image pixels and rows
// filled with zeros by the copy engine) and of the 9 x 2 weight planes (one box of the blocked
// weights: 8 input channels x kN output channels x 18 planes) into a free stage, counted on the
// stage's "full" mbarrier; a second thread
// waits for the stage, issues the stage's 9 kR UMMAs and commits them to its "empty" mbarrier,
// which frees the stage for the loads kS chunks later.  The boxes land in the K-major no-swizzle
// layout the descriptors of k_conv3x3_tc read (16-byte rows, one plane per channel half), so the
// MMAs and the epilogue are that kernel's.  Every wait is bounded.
// ---------------------------------------------------------------------------------------------
// A plane of a halo row in the ring: the 130 x 16-byte box rows, padded to a multiple of 128 bytes
// so every bulk-tensor destination starts on a 128-byte boundary (the descriptors' LBO).
constexpr int kTmaPlaneA = (kTcPlaneA + 127) / 128 * 128;
// Bytes the loads of one stage deliver (the mbarrier's transaction count) and the stage's size.
template <int kN, int kR>
__host__ __device__ constexpr int tma_tx_bytes() {
  return (kR + 2) * 2 * kTcPlaneA + 9 * 2 * kN * 16;
}
template <int kN, int kR>
__host__ __device__ constexpr int tma_stage_bytes() {
  return (kR + 2) * 2 * kTmaPlaneA + 9 * 2 * kN * 16;
}
template <int kN, int kR, int kS>
__host__ __device__ constexpr int tma_smem_bytes() {
  // stages, 1024-aligned, then the barriers (2 per stage + 1)
  return kS * ((tma_stage_bytes<kN, kR>() + 1023) / 1024 * 1024) + 8 * (2 * kS + 1);
}

__device__ __forceinline__ bool tc_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done = 0;
  for (int spin = 0; spin < kTcSpin && !done; spin++) {
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
  }
  return done != 0;
}

template <int kN, int kR, int kS>
__global__ void __launch_bounds__(128) k_conv3x3_tma(ConvArgs a, const __grid_constant__ CUtensorMap tmA,
                                                     const __grid_constant__ CUtensorMap tmB,
                                                     int *err) {
  extern __shared__ __align__(1024) unsigned char tm_smem[];
  constexpr int kStage = (tma_stage_bytes<kN, kR>() + 1023) / 1024 * 1024;
  uint64_t *full = reinterpret_cast<uint64_t *>(tm_smem + kS * kStage);
  uint64_t *empty = full + kS;
  uint64_t *done = empty + kS;
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int w0 = blockIdx.x * kTcM, row0 = blockIdx.y * kR;
  const int ngrp = a.cout / kN;
  const int img = blockIdx.z / ngrp, co0 = (blockIdx.z % ngrp) * kN;
  constexpr uint32_t kCols = kR * kN <= 32 ? 32 : kR * kN <= 64 ? 64 : kR * kN <= 128 ? 128
                           : kR * kN <= 256 ? 256 : 512;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_base)), "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    for (int k = 0; k < 2 * kS + 1; k++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(full + k)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = tmem_base;
  constexpr uint32_t idesc = umma_idesc(kTcM, kN);
  const int nch = a.cin / 16;
  if (tid == 0) {
    // producer: tiled bulk-tensor loads of chunk c into stage c mod kS
    const uint64_t ta = reinterpret_cast<uint64_t>(&tmA), tb = reinterpret_cast<uint64_t>(&tmB);
    for (int c = 0; c < nch; c++) {
      const int st = c % kS, k = c / kS;
      if (c >= kS && !tc_wait(empty + st, (k - 1) & 1)) {
        s_fail = 1;
        break;
      }
      unsigned char *sA = tm_smem + st * kStage, *sB = sA + (kR + 2) * 2 * kTmaPlaneA;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(
                       smem_u32(full + st)),
                   "r"((uint32_t)tma_tx_bytes<kN, kR>())
                   : "memory");
      const int ci0 = c * 16;
      for (int r = 0; r < kR + 2; r++)
        for (int kh = 0; kh < 2; kh++)
          asm volatile(
              "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
              " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(
                  smem_u32(sA + (r * 2 + kh) * kTmaPlaneA)),
              "l"(ta), "r"(ci0 + 8 * kh), "r"(w0 - 1), "r"(row0 + r - 1), "r"(img),
              "r"(smem_u32(full + st))
              : "memory");
      // the chunk's 9 x 2 weight planes of this output tile: one box of the blocked weights
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_u32(sB)),
          "l"(tb), "r"(0), "r"(co0), "r"(18 * c), "r"(smem_u32(full + st))
          : "memory");
    }
  } else if (tid == 32) {
    // MMA issuer: the stage's 9 kR UMMAs, then a commit that frees the stage
    for (int c = 0; c < nch; c++) {
      const int st = c % kS, k = c / kS;
      if (!tc_wait(full + st, k & 1)) {
        s_fail = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      const uint32_t a_base = smem_u32(tm_smem + st * kStage);
      const uint32_t b_base = a_base + (kR + 2) * 2 * kTmaPlaneA;
#pragma unroll
      for (int j = 0; j < kR; j++)
#pragma unroll
        for (int tap = 0; tap < 9; tap++) {
          const int ky = tap / 3, kx = tap % 3;
          const uint64_t ad =
              umma_desc(a_base + ((j + ky) * 2) * kTmaPlaneA + kx * 16, kTmaPlaneA, 128);
          const uint64_t bd = umma_desc(b_base + (tap * 2) * (kN * 16), kN * 16, 128);
          const uint32_t acc = (c > 0 || tap > 0) ? 1u : 0u;
          asm volatile(
              "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
                  tmem + (uint32_t)(j * kN)),
              "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
        }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
              smem_u32(empty + st)));
    }
    // completion of every MMA issued
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
            smem_u32(done)));
  }
  bool ok = tc_wait(done, 0);
  __syncwarp();
  ok = __syncthreads_and(ok && !s_fail);
  if (!ok && tid == 0) atomicExch(err, 1);
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  for (int j = 0; j < kR && ok; j++) {
    const int row = row0 + j;
    const int m = warp * 32 + lane;
    const int ww = w0 + m;
    const long long obase = (((long long)img * a.h + row) * a.w + ww) * a.ocs + a.oco + co0;
#pragma unroll 1
    for (int c0 = 0; c0 < kN; c0 += 8) {
      uint32_t r[8];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(j * kN + c0);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      if (ww < a.w && row < a.h) {
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
          v[q] = __uint_as_float(r[q]) + (a.bias ? a.bias[co0 + c0 + q] : 0.f);
          if (a.relu) v[q] = fmaxf(v[q], 0.f);
        }
        const long long o = obase + c0;
        if (a.mask) {
#pragma unroll
          for (int q = 0; q < 8; q++)
            if (!(__bfloat162float(a.mask[o + q]) > 0.f)) v[q] = 0.f;
        }
        __nv_bfloat162 pk[4];
#pragma unroll
        for (int q = 0; q < 4; q++) pk[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
        *reinterpret_cast<uint4 *>(a.out + o) = *reinterpret_cast<uint4 *>(pk);
        if (a.out_f32) {
#pragma unroll
          for (int q = 0; q < 8; q++) a.out_f32[o + q] = v[q];
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kCols));
  }
}

// ---------------------------------------------------------------------------------------------
// Weight gradient dW[tap][co][ci] += sum_p dz[p][co] x[p + tap][ci] and bias gradient.  CTA:
// 32 couts x 16*kCiT input channels, all 9 taps, over a contiguous range of 32-pixel row chunks
// (split-K over CTAs, FP32 atomics at the end).  Operands are staged transposed (channel-major,
// pixels contiguous) so both MMA fragments are 32-bit shared loads; x is staged once per
// horizontal tap shift so every fragment load is aligned.
// ---------------------------------------------------------------------------------------------
constexpr int kWS = kPx + 8;  // transposed pixel stride (halves)

struct WgradArgs {
  const bf16 *dz;  // [N][H][W][zcs] at channel offset 0, cout channels
  const bf16 *x;   // [N][H][W][cin]
  float *dw;       // [9][cout][cin] FP32 (accumulated)
  float *db;       // [cout] FP32 (accumulated) or null
  int n, h, w, cin, cout, zcs;
  int chunks_per_cta;
};

template <int kCiT>
__global__ void __launch_bounds__(128) k_conv3x3_wgrad(WgradArgs a) {
  constexpr int kCi = 16 * kCiT;
  __shared__ __align__(16) bf16 s_dz[32][kWS];            // [co][px]
  __shared__ __align__(16) bf16 s_x[3][kCi][3][kWS];      // [kx shift][ci][row][px]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int co0 = blockIdx.x * 32, ci0 = blockIdx.y * kCi;
  const int mt = warp & 1;                 // co block of 16
  constexpr int kNT = kCi / 8;             // n-tiles of 8 channels
  constexpr int kNTw = kNT / 2;            // n-tiles per warp (warps 0/1 vs 2/3 split them)
  const int nt0 = (warp >> 1) * kNTw;
  float acc[9][kNTw][4];
#pragma unroll
  for (int i = 0; i < 9; i++)
#pragma unroll
    for (int j = 0; j < kNTw; j++)
#pragma unroll
      for (int k = 0; k < 4; k++) acc[i][j][k] = 0.f;
  float bsum = 0.f;
  const int wchunks = (a.w + kPx - 1) / kPx;
  const long long total = (long long)a.n * a.h * wchunks;
  const long long c_begin = (long long)blockIdx.z * a.chunks_per_cta;
  const long long c_end = c_begin + a.chunks_per_cta < total ? c_begin + a.chunks_per_cta : total;
  for (long long cidx = c_begin; cidx < c_end; cidx++) {
    const int wc = (int)(cidx % wchunks);
    const long long rr = cidx / wchunks;
    const int row = (int)(rr % a.h), img = (int)(rr / a.h);
    const int w0 = wc * kPx;
    // dz chunk, transposed: 32 pixels x 32 couts
    for (int i = tid; i < kPx * 32; i += 128) {
      const int co = i & 31, px = i >> 5;
      const int ww = w0 + px;
      bf16 v = __float2bfloat16(0.f);
      if (ww < a.w) v = a.dz[(((long long)img * a.h + row) * a.w + ww) * a.zcs + co0 + co];
      s_dz[co][px] = v;
    }
    // x rows row-1..row+1, pixels w0-1 .. w0+kPx, staged for each kx shift
    for (int i = tid; i < 3 * (kPx + 2) * kCi; i += 128) {
      const int ci = i % kCi, px = (i / kCi) % (kPx + 2), r = i / (kCi * (kPx + 2));
      const int hh = row + r - 1, ww = w0 + px - 1;
      bf16 v = __float2bfloat16(0.f);
      if (hh >= 0 && hh < a.h && ww >= 0 && ww < a.w)
        v = a.x[(((long long)img * a.h + hh) * a.w + ww) * a.cin + ci0 + ci];
      // pixel px of the halo row serves output pixel px - kx for shift kx
#pragma unroll
      for (int kx = 0; kx < 3; kx++) {
        const int q = px - kx;
        if (q >= 0 && q < kPx) s_x[kx][ci][r][q] = v;
      }
    }
    __syncthreads();
    if (a.db && tid < 32) {
      float s = 0.f;
      for (int px = 0; px < kPx; px++) s += __bfloat162float(s_dz[tid][px]);
      bsum += s;
    }
#pragma unroll
    for (int ks = 0; ks < 2; ks++) {
      unsigned fa[4];
      const int m = mt * 16 + g, k = ks * 16 + 2 * t;
      fa[0] = ld32(&s_dz[m][k]);
      fa[1] = ld32(&s_dz[m + 8][k]);
      fa[2] = ld32(&s_dz[m][k + 8]);
      fa[3] = ld32(&s_dz[m + 8][k + 8]);
#pragma unroll
      for (int tap = 0; tap < 9; tap++) {
        const int ky = tap / 3, kx = tap % 3;
#pragma unroll
        for (int j = 0; j < kNTw; j++) {
          const int ci = (nt0 + j) * 8 + g;
          mma16816(acc[tap][j], fa, ld32(&s_x[kx][ci][ky][k]), ld32(&s_x[kx][ci][ky][k + 8]));
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int tap = 0; tap < 9; tap++)
#pragma unroll
    for (int j = 0; j < kNTw; j++) {
      const int ci = ci0 + (nt0 + j) * 8 + 2 * t;
#pragma unroll
      for (int hlf = 0; hlf < 2; hlf++) {
        const int co = co0 + mt * 16 + g + 8 * hlf;
        float *p = a.dw + ((long long)tap * a.cout + co) * a.cin + ci;
        atomicAdd(p, acc[tap][j][2 * hlf]);
        atomicAdd(p + 1, acc[tap][j][2 * hlf + 1]);
      }
    }
  if (a.db && tid < 32 && blockIdx.y == 0) atomicAdd(a.db + co0 + tid, bsum);
}

// ---------------------------------------------------------------------------------------------
// The weight gradient on the tensor cores (tcgen05, accumulators in TMEM).  The product is
// dW[tap][co][ci] = sum_p dz[p][co] x[p + tap][ci]: D = A B^T with A = dz^T (M = 128 output
// channels, K = pixels) and B = x shifted by the tap (N = kN input channels, K = pixels).  A CTA
// owns 128 output channels x kN input channels x the three taps of one kernel row ky (3 kN TMEM
// columns), and a contiguous range of 64-pixel row chunks (split-K over CTAs, FP32 atomics at the
// end).  Per chunk it copies the raw rows (dz: 64 pixels x 128 channels; x: row r + ky - 1, 66
// pixels x kN channels) into shared memory, rebuilds them transposed (pixels contiguous) in the
// canonical K-major no-swizzle layout -- one 8-pixel core-matrix row per 16-byte store, a copy of
// x per horizontal shift kx because a one-pixel shift along K is not a descriptor offset -- and
// one thread issues the 3 x 4 UMMAs (M 128, N kN, K 16).  The raw copy of the next chunk overlaps
// the MMAs of this one; the rebuild waits for them (bounded mbarrier wait).
// ---------------------------------------------------------------------------------------------
constexpr int kWgP = 64;                 // pixels per chunk (4 UMMA K-steps)
constexpr int kWgM = 128;                // output channels per CTA (UMMA M)
constexpr int kWgPlaneA = kWgM * 16;     // bytes of one 8-pixel plane of A

template <int kN>
constexpr int wg_tc_smem_bytes() {
  // raw dz [P][128] + raw x [P + 2][kN] + A [P/8][128][16 B] + B [3][P/8][kN][16 B]
  return kWgP * kWgM * 2 + (kWgP + 2) * kN * 2 + (kWgP / 8) * kWgPlaneA + 3 * (kWgP / 8) * kN * 16;
}

template <int kN>
__global__ void __launch_bounds__(128) k_conv3x3_wgrad_tc(WgradArgs a, int *err) {
  extern __shared__ __align__(1024) unsigned char wg_smem[];
  unsigned char *sA = wg_smem;                                   // transposed dz (1024-aligned)
  unsigned char *sB = sA + (kWgP / 8) * kWgPlaneA;                // transposed x, per kx
  bf16 *raw_dz = reinterpret_cast<bf16 *>(sB + 3 * (kWgP / 8) * kN * 16);  // [P][128]
  bf16 *raw_x = raw_dz + kWgP * kWgM;                             // [P + 2][kN]
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int co0 = blockIdx.x * kWgM;
  const int ci0 = (blockIdx.y / 3) * kN, ky = blockIdx.y % 3;
  constexpr uint32_t kCols = 3 * kN <= 64 ? 64 : 128;  // TMEM columns: a power of two >= 3 kN
  constexpr int kBPlane = kN * 16;                     // bytes of one 8-pixel plane of B
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_base)), "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar)));
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = tmem_base;
  constexpr uint32_t idesc = umma_idesc(kWgM, kN);
  const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB);
  const int wchunks = (a.w + kWgP - 1) / kWgP;
  const long long total = (long long)a.n * a.h * wchunks;
  const long long c_begin = (long long)blockIdx.z * a.chunks_per_cta;
  const long long c_end = c_begin + a.chunks_per_cta < total ? c_begin + a.chunks_per_cta : total;
  const bool do_bias = a.db && blockIdx.y == 0;
  float bsum = 0.f;
  bool ok = true, pending = false;
  int phase = 0;
  auto wait_mma = [&]() {
    uint32_t done = 0;
    for (int spin = 0; spin < kTcSpin && !done; spin++) {
      asm volatile(
          "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
          "selp.u32 %0, 1, 0, p;\n}\n"
          : "=r"(done)
          : "r"(smem_u32(&mbar)), "r"(phase)
          : "memory");
    }
    if (!done) {
      ok = false;
      if (tid == 0) atomicExch(err, 1);
    }
    phase ^= 1;
  };
  for (long long cidx = c_begin; cidx < c_end && ok; cidx++) {
    const int wc = (int)(cidx % wchunks);
    const long long rr = cidx / wchunks;
    const int row = (int)(rr % a.h), img = (int)(rr / a.h);
    const int w0 = wc * kWgP;
    // ---- raw copies (overlap the previous chunk's MMAs, which read only sA / sB) ----------
    for (int i = tid; i < kWgP * (kWgM / 8); i += 128) {  // dz: 16-byte pieces of 8 channels
      const int px = i / (kWgM / 8), cg = i % (kWgM / 8);
      const int ww = w0 + px, co = co0 + cg * 8;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (ww < a.w && co < a.cout)
        v = *reinterpret_cast<const uint4 *>(
            a.dz + (((long long)img * a.h + row) * a.w + ww) * a.zcs + co);
      *reinterpret_cast<uint4 *>(raw_dz + px * kWgM + cg * 8) = v;
    }
    const int hh = row + ky - 1;
    for (int i = tid; i < (kWgP + 2) * (kN / 8); i += 128) {  // x: row hh, pixels w0-1 .. w0+P
      const int px = i / (kN / 8), cg = i % (kN / 8);
      const int ww = w0 + px - 1;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (hh >= 0 && hh < a.h && ww >= 0 && ww < a.w)
        v = *reinterpret_cast<const uint4 *>(
            a.x + (((long long)img * a.h + hh) * a.w + ww) * a.cin + ci0 + cg * 8);
      *reinterpret_cast<uint4 *>(raw_x + px * kN + cg * 8) = v;
    }
    if (pending) wait_mma();  // the previous chunk's MMAs are done with sA / sB
    pending = false;
    if (!__syncthreads_and(ok)) {  // every thread leaves together if any wait gave up
      ok = false;
      break;
    }
    // ---- transposed rebuild: core-matrix row (channel, 8 pixels) per 16-byte store -------
    {
      const int m = tid;  // output channel co0 + m; plane g = pixels 8g .. 8g+7
#pragma unroll
      for (int g = 0; g < kWgP / 8; g++) {
        __align__(16) bf16 v[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
          v[j] = raw_dz[(8 * g + j) * kWgM + m];
          if (do_bias) bsum += __bfloat162float(v[j]);
        }
        *reinterpret_cast<uint4 *>(sA + g * kWgPlaneA + (m >> 3) * 128 + (m & 7) * 16) =
            *reinterpret_cast<const uint4 *>(v);
      }
    }
    for (int i = tid; i < 3 * (kWgP / 8) * kN; i += 128) {
      const int ci = i % kN, g = (i / kN) % (kWgP / 8), kx = i / (kN * (kWgP / 8));
      __align__(16) bf16 v[8];
#pragma unroll
      for (int j = 0; j < 8; j++) v[j] = raw_x[(8 * g + j + kx) * kN + ci];
      *reinterpret_cast<uint4 *>(sB + (kx * (kWgP / 8) + g) * kBPlane + (ci >> 3) * 128 +
                                 (ci & 7) * 16) = *reinterpret_cast<const uint4 *>(v);
    }
    // generic-proxy writes -> visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
#pragma unroll
      for (int kx = 0; kx < 3; kx++)
#pragma unroll
        for (int s = 0; s < kWgP / 16; s++) {
          const uint64_t ad = umma_desc(a_base + (2 * s) * kWgPlaneA, kWgPlaneA, 128);
          const uint64_t bd =
              umma_desc(b_base + (kx * (kWgP / 8) + 2 * s) * kBPlane, kBPlane, 128);
          const uint32_t acc = (cidx > c_begin || s > 0) ? 1u : 0u;
          asm volatile(
              "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
                  tmem + (uint32_t)(kx * kN)),
              "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
        }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
              smem_u32(&mbar)));
    }
    pending = true;
  }
  if (pending && ok) wait_mma();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  if (ok && c_end > c_begin) {
    // epilogue: thread (warp w, lane l) owns output channel co0 + 32 w + l
    const int co = co0 + warp * 32 + lane;
#pragma unroll 1
    for (int kx = 0; kx < 3; kx++) {
      float *dst = a.dw + ((long long)(ky * 3 + kx) * a.cout + co) * a.cin + ci0;
#pragma unroll 1
      for (int c0 = 0; c0 < kN; c0 += 8) {
        uint32_t r[8];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(kx * kN + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
              "=r"(r[7])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (co < a.cout) {
#pragma unroll
          for (int j = 0; j < 8; j++) atomicAdd(dst + c0 + j, __uint_as_float(r[j]));
        }
      }
    }
    if (do_bias && tid < kWgM && co0 + tid < a.cout) atomicAdd(a.db + co0 + tid, bsum);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kCols));
  }
}

// ---------------------------------------------------------------------------------------------
// The weight gradient with both operands MN-major (option "tcgen05_wgrad_tma"): in the product
// dW[tap][co][ci] = sum_p dz[p][co] x[p + tap][ci] the reduction runs over pixels, and the NHWC
// activations hold the M (co) and N (ci) indices contiguous, so a tiled bulk-tensor box of
// 8 channels x P pixels lands as one 8-channel column of the canonical MN-major no-swizzle layout
// (16-byte rows of 8 channels, one per pixel; 8-pixel core matrices 128 bytes apart along K,
// channel groups one box (x: one 128-byte-padded box) apart along M / N).  No transposition passes through the threads: one
// thread issues the boxes of a 64-pixel row chunk into a kS-stage ring (dz: up to 16 channel
// groups; x: the kN / 8 groups of 66 pixels, w0 - 1 .. w0 + 64, of row r + ky - 1, the copy engine
// filling pixels and rows outside the image with zeros), a second thread issues the chunk's
// 3 x 4 UMMAs (M 128 output channels, N kN input channels, K 16 pixels; the shift kx is a
// 16-byte offset of the B descriptor along K) and commits them to the stage's "empty" barrier.
// A CTA owns 128 output channels x kN input channels x the three taps of one kernel row and a
// contiguous range of chunks (split-K, FP32 atomics at the end).  The bias gradient is
// k_bias_grad's.  Every wait is bounded.
// ---------------------------------------------------------------------------------------------
constexpr int kWtStages = 4;
constexpr int kWtHalo = kWgP + 2;                // x pixels per chunk
// ring space of one x box (66 pixels x 16 B), padded so every box lands on a 128-byte boundary
constexpr int kWtXPlane = (kWtHalo * 16 + 127) / 128 * 128;
template <int kN>
__host__ __device__ constexpr int wt_stage_bytes() {
  return ((16 * kWgP * 16 + (kN / 8) * kWtXPlane) + 1023) / 1024 * 1024;
}
template <int kN>
__host__ __device__ constexpr int wt_smem_bytes() {
  return kWtStages * wt_stage_bytes<kN>() + 8 * (2 * kWtStages + 1);
}

template <int kN>
__global__ void __launch_bounds__(128) k_conv3x3_wgrad_tma(WgradArgs a,
                                                           const __grid_constant__ CUtensorMap tmZ,
                                                           const __grid_constant__ CUtensorMap tmX,
                                                           int *err) {
  extern __shared__ __align__(1024) unsigned char wt_smem[];
  constexpr int kStage = wt_stage_bytes<kN>();
  constexpr int kZBytes = 16 * kWgP * 16;   // dz: 16 channel groups x 64 pixels x 16 B
  uint64_t *full = reinterpret_cast<uint64_t *>(wt_smem + kWtStages * kStage);
  uint64_t *empty = full + kWtStages;
  uint64_t *done = empty + kWtStages;
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int co0 = blockIdx.x * kWgM;
  const int ci0 = (blockIdx.y / 3) * kN, ky = blockIdx.y % 3;
  const int gz = (a.cout - co0) / 8 < 16 ? (a.cout - co0) / 8 : 16;  // dz channel groups loaded
  constexpr uint32_t kCols = 3 * kN <= 32 ? 32 : 3 * kN <= 64 ? 64 : 3 * kN <= 128 ? 128
                           : 3 * kN <= 256 ? 256 : 512;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_base)), "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    for (int k = 0; k < 2 * kWtStages + 1; k++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(full + k)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = tmem_base;
  // both operands MN-major (instruction descriptor bits 15 and 16)
  constexpr uint32_t idesc = umma_idesc(kWgM, kN) | (1u << 15) | (1u << 16);
  const int wchunks = (a.w + kWgP - 1) / kWgP;
  const long long total = (long long)a.n * a.h * wchunks;
  const long long c_begin = (long long)blockIdx.z * a.chunks_per_cta;
  const long long c_end = c_begin + a.chunks_per_cta < total ? c_begin + a.chunks_per_cta : total;
  const int nck = c_end > c_begin ? (int)(c_end - c_begin) : 0;
  if (tid == 0) {
    // producer
    const uint64_t tz = reinterpret_cast<uint64_t>(&tmZ), tx = reinterpret_cast<uint64_t>(&tmX);
    const uint32_t tx_bytes = (uint32_t)(gz * kWgP * 16 + (kN / 8) * kWtHalo * 16);
    for (int i = 0; i < nck; i++) {
      const int st = i % kWtStages, k = i / kWtStages;
      if (i >= kWtStages && !tc_wait(empty + st, (k - 1) & 1)) {
        s_fail = 1;
        break;
      }
      const long long cidx = c_begin + i;
      const int wc = (int)(cidx % wchunks);
      const long long rr = cidx / wchunks;
      const int row = (int)(rr % a.h), img = (int)(rr / a.h);
      const int w0 = wc * kWgP;
      unsigned char *sZ = wt_smem + st * kStage, *sX = sZ + kZBytes;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(
                       smem_u32(full + st)),
                   "r"(tx_bytes)
                   : "memory");
      for (int g = 0; g < gz; g++)
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(smem_u32(sZ + g * (kWgP * 16))),
            "l"(tz), "r"(co0 + 8 * g), "r"(w0), "r"(row), "r"(img), "r"(smem_u32(full + st))
            : "memory");
      for (int g = 0; g < kN / 8; g++)
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(smem_u32(sX + g * kWtXPlane)),
            "l"(tx), "r"(ci0 + 8 * g), "r"(w0 - 1), "r"(row + ky - 1), "r"(img),
            "r"(smem_u32(full + st))
            : "memory");
    }
  } else if (tid == 32) {
    // MMA issuer
    for (int i = 0; i < nck; i++) {
      const int st = i % kWtStages, k = i / kWtStages;
      if (!tc_wait(full + st, k & 1)) {
        s_fail = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      const uint32_t z_base = smem_u32(wt_smem + st * kStage);
      const uint32_t x_base = z_base + kZBytes;
#pragma unroll
      for (int kx = 0; kx < 3; kx++)
#pragma unroll
        for (int s = 0; s < kWgP / 16; s++) {
          const uint64_t ad = umma_desc(z_base + s * 256, 128, kWgP * 16);
          const uint64_t bd = umma_desc(x_base + kx * 16 + s * 256, 128, kWtXPlane);
          const uint32_t acc = (i > 0 || s > 0) ? 1u : 0u;
          asm volatile(
              "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
                  tmem + (uint32_t)(kx * kN)),
              "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
        }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
              smem_u32(empty + st)));
    }
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
            smem_u32(done)));
  }
  bool ok = tc_wait(done, 0);
  __syncwarp();
  ok = __syncthreads_and(ok && !s_fail);
  if (!ok && tid == 0) atomicExch(err, 1);
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  if (ok && nck > 0) {
    // epilogue: thread (warp w, lane l) owns output channel co0 + 32 w + l
    const int co = co0 + warp * 32 + lane;
#pragma unroll 1
    for (int kx = 0; kx < 3; kx++) {
      float *dst = a.dw + ((long long)(ky * 3 + kx) * a.cout + co) * a.cin + ci0;
#pragma unroll 1
      for (int c0 = 0; c0 < kN; c0 += 8) {
        uint32_t r[8];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(kx * kN + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
              "=r"(r[7])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (co < a.cout) {
#pragma unroll
          for (int j = 0; j < 8; j++) atomicAdd(dst + c0 + j, __uint_as_float(r[j]));
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kCols));
  }
}

// Bias gradient db[co] += sum_p dz[p][co] (dz [P][zcs], cout channels): each thread sums one
// 8-channel group over a strided set of pixels, then shared and global atomics.
__global__ void __launch_bounds__(256) k_bias_grad(const bf16 *dz, int zcs, int cout, long long npx,
                                                   float *db) {
  __shared__ float s_db[512];  // cout <= 512 (base channels <= 64)
  for (int i = threadIdx.x; i < cout; i += blockDim.x) s_db[i] = 0.f;
  __syncthreads();
  const int g = cout / 8, per = blockDim.x / g;  // threads per channel group
  const int cg = threadIdx.x % g, lp = threadIdx.x / g;
  float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (lp < per) {
    for (long long p = (long long)blockIdx.x * per + lp; p < npx; p += (long long)gridDim.x * per) {
      const uint4 v = *reinterpret_cast<const uint4 *>(dz + p * zcs + cg * 8);
      const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int q = 0; q < 8; q++)
        acc[q] += __uint_as_float((q & 1) ? (wv[q >> 1] & 0xffff0000u) : (wv[q >> 1] << 16));
    }
#pragma unroll
    for (int q = 0; q < 8; q++) atomicAdd(&s_db[cg * 8 + q], acc[q]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < cout; i += blockDim.x) atomicAdd(db + i, s_db[i]);
}

// ---------------------------------------------------------------------------------------------
// Element-wise and small kernels
// ---------------------------------------------------------------------------------------------
// The layout kernels below move 8 channels (16 bytes) per thread: a CTA row of threads covers
// one image row (pixel x channel group), blockIdx.y strides over the rows of all images, so every
// index is one 64-bit division per row and one 32-bit division per thread.  Channel counts are
// multiples of 8 (base 32 or 64).  The arithmetic per element is the one of the scalar
// definitions in the comments, in the same order.
__device__ __forceinline__ uint4 ld16(const bf16 *p) { return *reinterpret_cast<const uint4 *>(p); }
__device__ __forceinline__ void st16(bf16 *p, uint4 v) { *reinterpret_cast<uint4 *>(p) = v; }
__device__ __forceinline__ float bfe(const uint4 &v, int q) {
  const uint32_t w = (&v.x)[q >> 1];
  return __uint_as_float((q & 1) ? (w & 0xffff0000u) : (w << 16));
}
__device__ __forceinline__ uint4 pack8(const float *f) {
  uint4 v;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const __nv_bfloat162 b = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
    (&v.x)[q] = *reinterpret_cast<const uint32_t *>(&b);
  }
  return v;
}

// FP32 image [N][H][W] -> BF16 [N][H][W][16] (channel 0 = value, 1..15 = 0)
__global__ void k_pack_input(const float *x, bf16 *out, long long npx) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npx) return;
  float f[8] = {x[p], 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  st16(out + p * 16, pack8(f));
  st16(out + p * 16 + 8, make_uint4(0, 0, 0, 0));
}

// 2x2 average pooling, [N][H][W][C] -> [N][H/2][W/2][C]:
// y = 0.25 (x[2y][2x] + x[2y][2x+1] + x[2y+1][2x] + x[2y+1][2x+1])
__global__ void k_pool(const bf16 *x, bf16 *y, int n, int h, int w, int c) {
  const int h2 = h / 2, w2 = w / 2, g = c / 8;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= w2 * g) return;
  const int xx = t / g, cg = t - xx * g;
  for (long long r = blockIdx.y; r < (long long)n * h2; r += gridDim.y) {
    const long long im = r / h2;
    const int yy = (int)(r - im * h2);
    const long long b = ((im * h + 2 * yy) * w + 2 * xx) * c + cg * 8;
    const uint4 v0 = ld16(x + b), v1 = ld16(x + b + c), v2 = ld16(x + b + (long long)w * c),
                v3 = ld16(x + b + (long long)w * c + c);
    float f[8];
#pragma unroll
    for (int q = 0; q < 8; q++) f[q] = 0.25f * (bfe(v0, q) + bfe(v1, q) + bfe(v2, q) + bfe(v3, q));
    st16(y + (r * w2 + xx) * c + cg * 8, pack8(f));
  }
}

// d(skip) = pool_grad(dy) * (s > 0) + extra, where extra (the skip's gradient through the
// decoder concatenation, already masked) is read at channel offset `eco` of stride `ecs`.
__global__ void k_pool_grad(const bf16 *dy, const bf16 *s, const bf16 *extra, int ecs, int eco,
                            bf16 *dx, int n, int h, int w, int c) {
  const int g = c / 8;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= w * g) return;
  const int xx = t / g, cg = t - xx * g;
  for (long long r = blockIdx.y; r < (long long)n * h; r += gridDim.y) {
    const long long im = r / h;
    const int yy = (int)(r - im * h);
    const long long px = r * w + xx;
    const long long j = ((im * (h / 2) + yy / 2) * (w / 2) + xx / 2) * c + cg * 8;
    const uint4 vs = ld16(s + px * c + cg * 8), vd = ld16(dy + j);
    uint4 ve = make_uint4(0, 0, 0, 0);
    if (extra) ve = ld16(extra + px * ecs + eco + cg * 8);
    float f[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      f[q] = bfe(vs, q) > 0.f ? 0.25f * bfe(vd, q) : 0.f;
      if (extra) f[q] += bfe(ve, q);
    }
    st16(dx + px * c + cg * 8, pack8(f));
  }
}

// Decoder input: out[.., 0:cu] = up2(u) (nearest), out[.., cu:cu+cs] = s; out [N][H][W][cu+cs]
__global__ void k_up_concat(const bf16 *u, int cu, const bf16 *s, int cs, bf16 *out, int n, int h,
                            int w) {
  const int gu = cu / 8, g = (cu + cs) / 8;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= w * g) return;
  const int xx = t / g, cg = t - xx * g;
  for (long long r = blockIdx.y; r < (long long)n * h; r += gridDim.y) {
    const long long im = r / h;
    const int yy = (int)(r - im * h);
    const long long px = r * w + xx;
    const uint4 v = cg < gu ? ld16(u + ((im * (h / 2) + yy / 2) * (w / 2) + xx / 2) * cu + cg * 8)
                            : ld16(s + px * cs + (cg - gu) * 8);
    st16(out + px * (cu + cs) + cg * 8, v);
  }
}

// d(u) = up2_grad(d(cat)[.., 0:cu]): sum of the 4 children
__global__ void k_up_grad(const bf16 *dcat, int c, bf16 *du, int cu, int n, int h, int w) {
  const int h2 = h / 2, w2 = w / 2, g = cu / 8;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= w2 * g) return;
  const int xx = t / g, cg = t - xx * g;
  for (long long r = blockIdx.y; r < (long long)n * h2; r += gridDim.y) {
    const long long im = r / h2;
    const int yy = (int)(r - im * h2);
    const long long b = ((im * h + 2 * yy) * w + 2 * xx) * c + cg * 8;
    const uint4 v0 = ld16(dcat + b), v1 = ld16(dcat + b + c), v2 = ld16(dcat + b + (long long)w * c),
                v3 = ld16(dcat + b + (long long)w * c + c);
    float f[8];
#pragma unroll
    for (int q = 0; q < 8; q++) f[q] = bfe(v0, q) + bfe(v1, q) + bfe(v2, q) + bfe(v3, q);
    st16(du + (r * w2 + xx) * cu + cg * 8, pack8(f));
  }
}

// 1x1 output convolution (c -> 1): y[p] = b + sum_c x[p][c] w[c], channels in ascending order
template <int kC>
__global__ void k_out_fwd(const bf16 *x, const float *w, const float *b, float *y, long long npx) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npx) return;
  float s = b[0];
#pragma unroll
  for (int cg = 0; cg < kC / 8; cg++) {
    const uint4 v = ld16(x + p * kC + cg * 8);
#pragma unroll
    for (int q = 0; q < 8; q++) s = fmaf(bfe(v, q), __ldg(w + cg * 8 + q), s);
  }
  y[p] = s;
}

// MSE loss gradient dy = 2 (y - t) / count, and per-block partial loss sums (FP64)
__global__ void k_mse(const float *y, const float *t, float *dy, long long npx, double *part) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < npx;
       p += (long long)gridDim.x * blockDim.x) {
    const float d = y[p] - t[p];
    dy[p] = 2.0f * d / (float)npx;
    acc += (double)d * d;
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// Backward of the 1x1 output convolution: dx[p][c] = dy[p] w[c] (x > 0), dw[c] += dy x, db += dy.
// Grid-stride over pixels with the kC + 1 sums in registers, reduced over the warp by shuffles,
// over the CTA in shared memory, and once per CTA into the global gradients.
template <int kC>
__global__ void __launch_bounds__(256) k_out_bwd(const bf16 *x, const float *dy, const float *w,
                                                 bf16 *dx, float *dw, float *db, long long npx) {
  __shared__ float s_dw[kC + 1];
  for (int i = threadIdx.x; i <= kC; i += blockDim.x) s_dw[i] = 0.f;
  __syncthreads();
  float acc[kC], accb = 0.f, wr[kC];
#pragma unroll
  for (int ch = 0; ch < kC; ch++) {
    acc[ch] = 0.f;
    wr[ch] = __ldg(w + ch);
  }
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < npx;
       p += (long long)gridDim.x * blockDim.x) {
    const float d = dy[p];
    accb += d;
#pragma unroll
    for (int cg = 0; cg < kC / 8; cg++) {
      const uint4 v = ld16(x + p * kC + cg * 8);
      float f[8];
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const float xv = bfe(v, q);
        f[q] = xv > 0.f ? d * wr[cg * 8 + q] : 0.f;
        acc[cg * 8 + q] += d * xv;
      }
      st16(dx + p * kC + cg * 8, pack8(f));
    }
  }
#pragma unroll
  for (int ch = 0; ch < kC; ch++) {
    float v = acc[ch];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_dw[ch], v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) accb += __shfl_xor_sync(0xffffffffu, accb, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(&s_dw[kC], accb);
  __syncthreads();
  if (threadIdx.x < kC) atomicAdd(dw + threadIdx.x, s_dw[threadIdx.x]);
  if (threadIdx.x == kC) atomicAdd(db, s_dw[kC]);
}

// Adam step on the FP32 master parameters (bias-corrected, as Kingma & Ba 2015).
__global__ void k_adam(float *p, const float *g, float *m, float *v, long long n, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// BF16 weight copies from the FP32 master [tap][co][ci_real]: forward [tap][co][cin_pad] and
// backward-data [tap'][ci][co] with tap' = 8 - tap (spatial flip), and both blocked for the
// bulk-tensor-fed convolution as [16-channel input chunk][tap][8-channel half][output ch][8], so
// the B operand of one chunk and output tile (18 planes of kN x 16 bytes) is one box.
__global__ void k_weights_bf16(const float *w, int k2, int co_n, int ci_real, int cin_pad,
                               bf16 *wf, bf16 *wb, bf16 *wfb, bf16 *wbb) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)k2 * co_n * cin_pad) return;
  const int ci = (int)(i % cin_pad);
  const int co = (int)((i / cin_pad) % co_n);
  const int tap = (int)(i / ((long long)cin_pad * co_n));
  const float v = ci < ci_real ? w[((long long)tap * co_n + co) * ci_real + ci] : 0.f;
  const bf16 b = __float2bfloat16(v);
  wf[i] = b;
  // blocked [ci / 16][tap][(ci / 8) & 1][co][ci & 7] (cin_pad a multiple of 16)
  if (wfb && cin_pad % 16 == 0)
    wfb[(((long long)(ci / 16) * k2 + tap) * 2 + ((ci >> 3) & 1)) * co_n * 8 + co * 8 + (ci & 7)] = b;
  if (ci < ci_real) {
    const int tb = k2 - 1 - tap;
    if (wb) wb[((long long)tb * ci_real + ci) * co_n + co] = b;
    // backward-data weights blocked the same way, input channels = co, output channels = ci
    if (wbb && co_n % 16 == 0)
      wbb[(((long long)(co / 16) * k2 + tb) * 2 + ((co >> 3) & 1)) * ci_real * 8 + ci * 8 + (co & 7)] = b;
  }
}

constexpr int kRedBlocks = 296;

// Channel 0 of the padded first-layer weight gradient [9*cout][cin_pad] -> [9*cout][1].
__global__ void k_fold_first(const float *g0, float *g, int rows, int cin_pad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < rows) g[i] = g0[(long long)i * cin_pad];
}

inline unsigned nblk(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// Grid of the row-wise layout kernels: x covers one row's (pixel, channel group) pairs, y the rows.
inline dim3 row_grid(long long rows, int per_row) {
  return dim3(nblk(per_row), (unsigned)(rows < 65535 ? rows : 65535));
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------------
struct ds2d_unet {
  struct Layer {
    std::string name;
    int cin, cout, k, cin_pad;
    long long w_off, b_off, nw;  // offsets into the flat FP32 parameter vector
    bf16 *wf = nullptr, *wb = nullptr;  // BF16 forward / backward-data weights
    // the same, blocked for the bulk-tensor-fed convolution: [cin/16][9][2][cout][8]
    bf16 *wfb = nullptr, *wbb = nullptr;
  };
  struct Act {
    bf16 *p = nullptr;
    int h = 0, w = 0, c = 0;
  };
  int base = 32, max_n = 0, max_h = 0, max_w = 0, device = 0;
  cudaStream_t stream = nullptr;
  std::vector<Layer> layers;
  long long nparam = 0;
  float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;
  long long adam_t = 0;
  // activations (forward) and their gradients (backward), per named slot
  enum {
    IN, E1A, E1B, P1, E2A, E2B, P2, E3A, E3B, P3, E4A, E4B, C3, D3A, D3B, C2, D2A, D2B, C1, D1A,
    D1B, NACT
  };
  Act act[NACT], grad[NACT];
  float *y = nullptr, *dy = nullptr;
  float *g0 = nullptr;  // padded [9][cout][16] weight gradient of the first layer (cin 1 -> 16)
  double *part = nullptr, *h_part = nullptr;
  std::string err;
  bool weights_dirty = true;
  int use_tc = 1;          // 3x3 convolutions on tcgen05 (1, default) or mma.sync (0)
  int tc_wgrad = 1;        // with use_tc: weight gradients on tcgen05 too (0: on mma.sync)
  int tc_wgrad_tma = 1;    // the weight gradient with MN-major bulk-tensor operands
  int tc_rows = 4;         // output rows per CTA of the tcgen05 convolution (1, 2 or 4)
  int tc_tma = 1;          // the tcgen05 convolution fed by tiled bulk-tensor loads (k_conv3x3_tma)
  int tc_stages = 2;       // ring stages of k_conv3x3_tma (2 or 3)
  int *d_err = nullptr;    // device flag raised by a bounded wait that gave up
  std::vector<void *> allocs;
};

namespace {

thread_local std::string g_unet_err;

int unet_fail(ds2d_unet *u, int code, const std::string &msg) {
  if (u) u->err = msg;
  else g_unet_err = msg;
  return code;
}

#define UCK(call)                                                                        \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return unet_fail(u, DS2D_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int ualloc(ds2d_unet *u, void **p, size_t bytes) {
  UCK(cudaMalloc(p, bytes));
  UCK(cudaMemsetAsync(*p, 0, bytes, u->stream));
  u->allocs.push_back(*p);
  return DS2D_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
using TmEncodeFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
TmEncodeFn tm_encode_fn() {
  static TmEncodeFn fn = []() -> TmEncodeFn {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<TmEncodeFn>(p);
  }();
  return fn;
}

// Tensor maps of one convolution: the input [n][h][w][cin] (box 8 channels x 130 pixels, zero
// fill outside the image) and the blocked weights [cin/16][9][2][cout][8] viewed as
// {8, cout, 18 cin/16} (box 8 x kn x 18: the whole B operand of a chunk and output tile).
bool conv_tensor_maps(const ConvArgs &a, const bf16 *wblk, int kn, CUtensorMap *ta,
                      CUtensorMap *tb) {
  TmEncodeFn enc = tm_encode_fn();
  if (!enc) return false;
  const cuuint64_t dA[4] = {(cuuint64_t)a.cin, (cuuint64_t)a.w, (cuuint64_t)a.h, (cuuint64_t)a.n};
  const cuuint64_t sA[3] = {(cuuint64_t)a.cin * 2, (cuuint64_t)a.w * a.cin * 2,
                            (cuuint64_t)a.h * a.w * a.cin * 2};
  const cuuint32_t bA[4] = {8, (cuuint32_t)kTcHalo, 1, 1}, e4[4] = {1, 1, 1, 1};
  if (enc(ta, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void *)a.in, dA, sA, bA, e4,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  const cuuint64_t dB[3] = {8, (cuuint64_t)a.cout, (cuuint64_t)18 * (a.cin / 16)};
  const cuuint64_t sB[2] = {16, (cuuint64_t)a.cout * 16};
  const cuuint32_t bB[3] = {8, (cuuint32_t)kn, 18}, e3[3] = {1, 1, 1};
  return enc(tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, (void *)wblk, dB, sB, bB, e3,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor maps of one weight gradient: dz [n][h][w][zcs] (cout channels; box 8 channels x 64
// pixels) and x [n][h][w][cin] (box 8 channels x 66 pixels), zero fill outside the image.
bool wgrad_tensor_maps(const WgradArgs &a, CUtensorMap *tz, CUtensorMap *tx) {
  TmEncodeFn enc = tm_encode_fn();
  if (!enc) return false;
  const cuuint32_t e4[4] = {1, 1, 1, 1};
  const cuuint64_t dZ[4] = {(cuuint64_t)a.cout, (cuuint64_t)a.w, (cuuint64_t)a.h, (cuuint64_t)a.n};
  const cuuint64_t sZ[3] = {(cuuint64_t)a.zcs * 2, (cuuint64_t)a.w * a.zcs * 2,
                            (cuuint64_t)a.h * a.w * a.zcs * 2};
  const cuuint32_t bZ[4] = {8, (cuuint32_t)kWgP, 1, 1};
  if (enc(tz, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void *)a.dz, dZ, sZ, bZ, e4,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  const cuuint64_t dX[4] = {(cuuint64_t)a.cin, (cuuint64_t)a.w, (cuuint64_t)a.h, (cuuint64_t)a.n};
  const cuuint64_t sX[3] = {(cuuint64_t)a.cin * 2, (cuuint64_t)a.w * a.cin * 2,
                            (cuuint64_t)a.h * a.w * a.cin * 2};
  const cuuint32_t bX[4] = {8, (cuuint32_t)kWtHalo, 1, 1};
  return enc(tx, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void *)a.x, dX, sX, bX, e4,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int kN, int kR, int kS>
void launch_tma(dim3 grid, const ConvArgs &a, const CUtensorMap &ta, const CUtensorMap &tb,
                ds2d_unet *u) {
  k_conv3x3_tma<kN, kR, kS><<<grid, 128, tma_smem_bytes<kN, kR, kS>(), u->stream>>>(a, ta, tb,
                                                                                    u->d_err);
}

template <int kN, int kR, int kS>
cudaError_t tma_attr() {
  return cudaFuncSetAttribute(k_conv3x3_tma<kN, kR, kS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              tma_smem_bytes<kN, kR, kS>());
}

int conv(ds2d_unet *u, const ds2d_unet::Layer &L, const bf16 *in, const bf16 *w, int cin, int cout,
         const float *bias, bf16 *out, int ocs, int oco, float *out_f32, const bf16 *mask, int relu,
         int n, int h, int wd) {
  ConvArgs a{in, w, bias, out, out_f32, mask, n, h, wd, cin, cout, ocs, oco, relu};
  if (u->use_tc && u->tc_tma && cout % 32 == 0 && cin % 16 == 0) {
    // tcgen05, operands by tiled bulk-tensor loads through a ring; output tiles of 128, 64, 96
    // (one tile for a 96-channel output, so its input is read once) or 32 channels
    const int kn = cout % 128 == 0 ? 128 : cout % 64 == 0 ? 64 : cout % 96 == 0 ? 96 : 32;
    const bf16 *wblk = w == L.wf ? L.wfb : (w == L.wb ? L.wbb : nullptr);
    CUtensorMap ta, tb;
    if (!wblk || !conv_tensor_maps(a, wblk, kn, &ta, &tb))
      return unet_fail(u, DS2D_E_CUDA, "conv: cuTensorMapEncodeTiled failed");
    // rows per CTA: 4 with option "tcgen05_rows" 4, else 2; ring stages: option "tcgen05_stages"
    const int kr = u->tc_rows == 4 ? 4 : 2, ks = u->tc_stages;
    dim3 grid((wd + kTcM - 1) / kTcM, (h + kr - 1) / kr, n * (cout / kn));
    const int v = kn == 96 ? (ks == 2 ? 12 : 13)  // 96 channels: two rows per CTA (TMEM)
                           : (kn == 128 ? 0 : kn == 64 ? 4 : 8) + (kr == 4 ? 2 : 0) + (ks == 2 ? 1 : 0);
    if (kn == 96) grid.y = (h + 1) / 2;
    switch (v) {
      case 0: launch_tma<128, 2, 3>(grid, a, ta, tb, u); break;
      case 1: launch_tma<128, 2, 2>(grid, a, ta, tb, u); break;
      case 2: launch_tma<128, 4, 3>(grid, a, ta, tb, u); break;
      case 3: launch_tma<128, 4, 2>(grid, a, ta, tb, u); break;
      case 4: launch_tma<64, 2, 3>(grid, a, ta, tb, u); break;
      case 5: launch_tma<64, 2, 2>(grid, a, ta, tb, u); break;
      case 6: launch_tma<64, 4, 3>(grid, a, ta, tb, u); break;
      case 7: launch_tma<64, 4, 2>(grid, a, ta, tb, u); break;
      case 8: launch_tma<32, 2, 3>(grid, a, ta, tb, u); break;
      case 9: launch_tma<32, 2, 2>(grid, a, ta, tb, u); break;
      case 10: launch_tma<32, 4, 3>(grid, a, ta, tb, u); break;
      case 11: launch_tma<32, 4, 2>(grid, a, ta, tb, u); break;
      case 12: launch_tma<96, 2, 2>(grid, a, ta, tb, u); break;
      default: launch_tma<96, 2, 3>(grid, a, ta, tb, u); break;
    }
    UCK(cudaGetLastError());
    return DS2D_OK;
  }
  if (u->use_tc && cout % 32 == 0) {
    const int kn = cout % 128 == 0 ? 128 : (cout % 64 == 0 ? 64 : 32);
    // rows per CTA: option "tcgen05_rows" (4 applies to tiles of up to 64 output channels; 128
    // channels take 2, keeping two CTAs per SM within the TMEM columns)
    const int kr = u->tc_rows == 4 && kn == 128 ? 2 : u->tc_rows;
    dim3 grid((wd + kTcM - 1) / kTcM, (h + kr - 1) / kr, n * (cout / kn));
    if (kr == 4) {
      if (kn == 64)
        k_conv3x3_tc<64, 4><<<grid, 128, tc_smem_bytes<64, 4>(), u->stream>>>(a, u->d_err);
      else
        k_conv3x3_tc<32, 4><<<grid, 128, tc_smem_bytes<32, 4>(), u->stream>>>(a, u->d_err);
    } else if (kr == 2) {
      if (kn == 128)
        k_conv3x3_tc<128, 2><<<grid, 128, tc_smem_bytes<128, 2>(), u->stream>>>(a, u->d_err);
      else if (kn == 64)
        k_conv3x3_tc<64, 2><<<grid, 128, tc_smem_bytes<64, 2>(), u->stream>>>(a, u->d_err);
      else
        k_conv3x3_tc<32, 2><<<grid, 128, tc_smem_bytes<32, 2>(), u->stream>>>(a, u->d_err);
    } else if (kn == 128) {
      k_conv3x3_tc<128><<<grid, 128, tc_smem_bytes<128>(), u->stream>>>(a, u->d_err);
    } else if (kn == 64) {
      k_conv3x3_tc<64><<<grid, 128, tc_smem_bytes<64>(), u->stream>>>(a, u->d_err);
    } else {
      k_conv3x3_tc<32><<<grid, 128, tc_smem_bytes<32>(), u->stream>>>(a, u->d_err);
    }
  } else if (cout % 64 == 0) {
    dim3 grid((wd + kPx - 1) / kPx, h, n * (cout / 64));
    k_conv3x3<64><<<grid, 128, 0, u->stream>>>(a);
  } else if (cout % 32 == 0) {
    dim3 grid((wd + kPx - 1) / kPx, h, n * (cout / 32));
    k_conv3x3<32><<<grid, 64, 0, u->stream>>>(a);
  } else {
    return unet_fail(u, DS2D_E_ARG, "conv: output channels must be a multiple of 32");
  }
  UCK(cudaGetLastError());
  return DS2D_OK;
}

int wgrad(ds2d_unet *u, const ds2d_unet::Layer &L, const bf16 *dz, int zcs, const bf16 *x, int n,
          int h, int wd, float *dw_padded = nullptr) {
  WgradArgs a{};
  a.dz = dz; a.x = x; a.dw = dw_padded ? dw_padded : u->grads + L.w_off; a.db = u->grads + L.b_off;
  a.n = n; a.h = h; a.w = wd; a.cin = L.cin_pad; a.cout = L.cout; a.zcs = zcs;
  const long long chunks = (long long)n * h * ((wd + kPx - 1) / kPx);
  const int kci = L.cin_pad >= 32 ? 32 : 16;
  const long long tiles = (long long)(L.cout / 32) * (L.cin_pad / kci);
  long long splits = (4 * 148 + tiles - 1) / tiles;
  if (splits > chunks) splits = chunks;
  if (splits < 1) splits = 1;
  a.chunks_per_cta = (int)((chunks + splits - 1) / splits);
  splits = (chunks + a.chunks_per_cta - 1) / a.chunks_per_cta;
  // the FP32 gradient is [tap][cout][cin]; a channel-padded layer (the first) accumulates into a
  // padded scratch that the caller folds
  if (L.cin_pad != L.cin && !dw_padded)
    return unet_fail(u, DS2D_E_STATE, "wgrad of a channel-padded layer needs a padded scratch");
  if (u->use_tc && u->tc_wgrad && u->tc_wgrad_tma && L.cin_pad % 16 == 0 && L.cout % 32 == 0 &&
      zcs % 8 == 0) {
    // tcgen05, MN-major operands by tiled bulk-tensor loads: CTAs of 128 output channels x kN
    // input channels x one kernel row over a range of 64-pixel chunks; bias by k_bias_grad
    const int kn = L.cin_pad % 128 == 0 ? 128 : L.cin_pad % 64 == 0 ? 64
                 : L.cin_pad % 96 == 0 ? 96 : L.cin_pad % 32 == 0 ? 32 : 16;
    CUtensorMap tz, tx;
    if (!wgrad_tensor_maps(a, &tz, &tx))
      return unet_fail(u, DS2D_E_CUDA, "wgrad: cuTensorMapEncodeTiled failed");
    const long long tchunks = (long long)n * h * ((wd + kWgP - 1) / kWgP);
    const long long ttiles = (long long)((L.cout + kWgM - 1) / kWgM) * (L.cin_pad / kn) * 3;
    long long ts = (4 * 148 + ttiles - 1) / ttiles;
    ts = ts > tchunks ? tchunks : (ts < 1 ? 1 : ts);
    a.chunks_per_cta = (int)((tchunks + ts - 1) / ts);
    ts = (tchunks + a.chunks_per_cta - 1) / a.chunks_per_cta;
    dim3 tgrid((L.cout + kWgM - 1) / kWgM, (L.cin_pad / kn) * 3, (unsigned)ts);
    if (kn == 128)
      k_conv3x3_wgrad_tma<128><<<tgrid, 128, wt_smem_bytes<128>(), u->stream>>>(a, tz, tx, u->d_err);
    else if (kn == 64)
      k_conv3x3_wgrad_tma<64><<<tgrid, 128, wt_smem_bytes<64>(), u->stream>>>(a, tz, tx, u->d_err);
    else if (kn == 96)
      k_conv3x3_wgrad_tma<96><<<tgrid, 128, wt_smem_bytes<96>(), u->stream>>>(a, tz, tx, u->d_err);
    else if (kn == 32)
      k_conv3x3_wgrad_tma<32><<<tgrid, 128, wt_smem_bytes<32>(), u->stream>>>(a, tz, tx, u->d_err);
    else
      k_conv3x3_wgrad_tma<16><<<tgrid, 128, wt_smem_bytes<16>(), u->stream>>>(a, tz, tx, u->d_err);
    const long long npx = (long long)n * h * wd;
    const unsigned bb = nblk(npx * (L.cout / 8)) < 148u * 4 ? nblk(npx * (L.cout / 8)) : 148u * 4;
    k_bias_grad<<<bb, 256, 0, u->stream>>>(dz, zcs, L.cout, npx, a.db);
    UCK(cudaGetLastError());
    return DS2D_OK;
  }
  if (u->use_tc && u->tc_wgrad && L.cin_pad % 16 == 0) {
    // tcgen05: CTAs of 128 output channels x kN input channels x one kernel row, 64-pixel chunks
    const int kn = L.cin_pad % 32 == 0 ? 32 : 16;
    const long long tchunks = (long long)n * h * ((wd + kWgP - 1) / kWgP);
    const long long ttiles = (long long)((L.cout + kWgM - 1) / kWgM) * (L.cin_pad / kn) * 3;
    long long ts = (4 * 148 + ttiles - 1) / ttiles;
    ts = ts > tchunks ? tchunks : (ts < 1 ? 1 : ts);
    a.chunks_per_cta = (int)((tchunks + ts - 1) / ts);
    ts = (tchunks + a.chunks_per_cta - 1) / a.chunks_per_cta;
    dim3 tgrid((L.cout + kWgM - 1) / kWgM, (L.cin_pad / kn) * 3, (unsigned)ts);
    if (kn == 32)
      k_conv3x3_wgrad_tc<32><<<tgrid, 128, wg_tc_smem_bytes<32>(), u->stream>>>(a, u->d_err);
    else
      k_conv3x3_wgrad_tc<16><<<tgrid, 128, wg_tc_smem_bytes<16>(), u->stream>>>(a, u->d_err);
    UCK(cudaGetLastError());
    return DS2D_OK;
  }
  dim3 grid(L.cout / 32, L.cin_pad / kci, (unsigned)splits);
  if (kci == 32)
    k_conv3x3_wgrad<2><<<grid, 128, 0, u->stream>>>(a);
  else
    k_conv3x3_wgrad<1><<<grid, 128, 0, u->stream>>>(a);
  UCK(cudaGetLastError());
  return DS2D_OK;
}

int refresh_weights(ds2d_unet *u) {
  if (!u->weights_dirty) return DS2D_OK;
  for (auto &L : u->layers) {
    if (L.k != 3) continue;
    const long long n = 9LL * L.cout * L.cin_pad;
    k_weights_bf16<<<nblk(n), 256, 0, u->stream>>>(u->params + L.w_off, 9, L.cout, L.cin,
                                                   L.cin_pad, L.wf, L.wb, L.wfb, L.wbb);
  }
  UCK(cudaGetLastError());
  u->weights_dirty = false;
  return DS2D_OK;
}

// Reads (and clears) the flag a tensor-core kernel raises when a bounded wait gave up.
int check_wait_flag(ds2d_unet *u) {
  int flag = 0;
  UCK(cudaMemcpyAsync(&flag, u->d_err, sizeof(int), cudaMemcpyDeviceToHost, u->stream));
  UCK(cudaStreamSynchronize(u->stream));
  if (flag) {
    UCK(cudaMemsetAsync(u->d_err, 0, sizeof(int), u->stream));
    return unet_fail(u, DS2D_E_CUDA, "tensor-core convolution: a bounded wait gave up");
  }
  return DS2D_OK;
}

int check_shape(ds2d_unet *u, int n, int h, int w) {
  if (n < 1 || n > u->max_n || h < 8 || w < 8 || h > u->max_h || w > u->max_w || h % 8 || w % 8)
    return unet_fail(u, DS2D_E_ARG,
                     "unet: need 1 <= n <= max_n, 8 <= h <= max_h, 8 <= w <= max_w, h and w "
                     "multiples of 8");
  return DS2D_OK;
}

// Forward pass: x [n][h][w] FP32 (device) -> u->y [n][h][w] FP32.
int forward(ds2d_unet *u, const float *x, int n, int h, int w) {
  int rc;
  if ((rc = refresh_weights(u))) return rc;
  using U = ds2d_unet;
  const long long npx = (long long)n * h * w;
  k_pack_input<<<nblk(npx), 256, 0, u->stream>>>(x, u->act[U::IN].p, npx);
  const int c[4] = {u->base, 2 * u->base, 4 * u->base, 8 * u->base};
  const int ea[4] = {U::E1A, U::E2A, U::E3A, U::E4A}, eb[4] = {U::E1B, U::E2B, U::E3B, U::E4B};
  const int pl[3] = {U::P1, U::P2, U::P3};
  int src = U::IN, cin = 16, hh = h, ww = w;
  for (int l = 0; l < 4; l++) {
    const auto &La = u->layers[2 * l], &Lb = u->layers[2 * l + 1];
    if ((rc = conv(u, La, u->act[src].p, La.wf, cin, c[l], u->params + La.b_off, u->act[ea[l]].p,
                   c[l], 0, nullptr, nullptr, 1, n, hh, ww)))
      return rc;
    if ((rc = conv(u, Lb, u->act[ea[l]].p, Lb.wf, c[l], c[l], u->params + Lb.b_off,
                   u->act[eb[l]].p, c[l], 0, nullptr, nullptr, 1, n, hh, ww)))
      return rc;
    if (l < 3) {
      k_pool<<<row_grid((long long)n * (hh / 2), (ww / 2) * (c[l] / 8)), 256, 0, u->stream>>>(
          u->act[eb[l]].p, u->act[pl[l]].p, n, hh, ww, c[l]);
      src = pl[l];
      hh /= 2;
      ww /= 2;
    }
    cin = c[l];
  }
  const int ca[3] = {U::C1, U::C2, U::C3}, da[3] = {U::D1A, U::D2A, U::D3A},
            db[3] = {U::D1B, U::D2B, U::D3B};
  int prev = U::E4B, cprev = c[3];
  for (int l = 2; l >= 0; l--) {
    hh *= 2;
    ww *= 2;
    const int cc = cprev + c[l];
    k_up_concat<<<row_grid((long long)n * hh, ww * (cc / 8)), 256, 0, u->stream>>>(
        u->act[prev].p, cprev, u->act[eb[l]].p, c[l], u->act[ca[l]].p, n, hh, ww);
    const int li = 8 + 2 * (2 - l);
    const auto &La = u->layers[li], &Lb = u->layers[li + 1];
    if ((rc = conv(u, La, u->act[ca[l]].p, La.wf, cc, c[l], u->params + La.b_off, u->act[da[l]].p,
                   c[l], 0, nullptr, nullptr, 1, n, hh, ww)))
      return rc;
    if ((rc = conv(u, Lb, u->act[da[l]].p, Lb.wf, c[l], c[l], u->params + Lb.b_off,
                   u->act[db[l]].p, c[l], 0, nullptr, nullptr, 1, n, hh, ww)))
      return rc;
    prev = db[l];
    cprev = c[l];
  }
  const auto &Lo = u->layers.back();
  if (c[0] == 32)
    k_out_fwd<32><<<nblk(npx), 256, 0, u->stream>>>(u->act[U::D1B].p, u->params + Lo.w_off,
                                                    u->params + Lo.b_off, u->y, npx);
  else
    k_out_fwd<64><<<nblk(npx), 256, 0, u->stream>>>(u->act[U::D1B].p, u->params + Lo.w_off,
                                                    u->params + Lo.b_off, u->y, npx);
  UCK(cudaGetLastError());
  return DS2D_OK;
}

// Backward pass from u->dy (dLoss/dy, FP32 [n][h][w]); parameter gradients into u->grads.
int backward(ds2d_unet *u, int n, int h, int w) {
  using U = ds2d_unet;
  int rc;
  const long long npx = (long long)n * h * w;
  const int c[4] = {u->base, 2 * u->base, 4 * u->base, 8 * u->base};
  UCK(cudaMemsetAsync(u->grads, 0, sizeof(float) * u->nparam, u->stream));
  const auto &Lo = u->layers.back();
  {
    const unsigned ob = nblk(npx) < 148u * 8 ? nblk(npx) : 148u * 8;  // grid-stride over pixels
    if (c[0] == 32)
      k_out_bwd<32><<<ob, 256, 0, u->stream>>>(u->act[U::D1B].p, u->dy, u->params + Lo.w_off,
                                               u->grad[U::D1B].p, u->grads + Lo.w_off,
                                               u->grads + Lo.b_off, npx);
    else
      k_out_bwd<64><<<ob, 256, 0, u->stream>>>(u->act[U::D1B].p, u->dy, u->params + Lo.w_off,
                                               u->grad[U::D1B].p, u->grads + Lo.w_off,
                                               u->grads + Lo.b_off, npx);
  }
  const int ca[3] = {U::C1, U::C2, U::C3}, da[3] = {U::D1A, U::D2A, U::D3A},
            db[3] = {U::D1B, U::D2B, U::D3B};
  const int ea[4] = {U::E1A, U::E2A, U::E3A, U::E4A}, eb[4] = {U::E1B, U::E2B, U::E3B, U::E4B};
  const int pl[3] = {U::P1, U::P2, U::P3};
  int hh = h, ww = w;
  // decoder, level 1 up to 3; the gradient arriving at db[l] is already ReLU-masked
  for (int l = 0; l < 3; l++) {
    const int li = 8 + 2 * (2 - l);
    const auto &La = u->layers[li], &Lb = u->layers[li + 1];
    const int cprev = l == 2 ? c[3] : c[l + 1];
    const int cc = cprev + c[l];
    // d(d_la output) = conv_bwd(d(db)) masked by d_la's output
    if ((rc = wgrad(u, Lb, u->grad[db[l]].p, c[l], u->act[da[l]].p, n, hh, ww))) return rc;
    if ((rc = conv(u, Lb, u->grad[db[l]].p, Lb.wb, c[l], c[l], nullptr, u->grad[da[l]].p, c[l], 0,
                   nullptr, u->act[da[l]].p, 0, n, hh, ww)))
      return rc;
    if ((rc = wgrad(u, La, u->grad[da[l]].p, c[l], u->act[ca[l]].p, n, hh, ww))) return rc;
    // d(concat) masked by the concat input (up(prev) and skip are both ReLU outputs)
    if ((rc = conv(u, La, u->grad[da[l]].p, La.wb, c[l], cc, nullptr, u->grad[ca[l]].p, cc, 0,
                   nullptr, u->act[ca[l]].p, 0, n, hh, ww)))
      return rc;
    // up part -> gradient of the coarser level's output
    const int prev = l == 2 ? U::E4B : db[l + 1];
    k_up_grad<<<row_grid((long long)n * (hh / 2), (ww / 2) * (cprev / 8)), 256, 0, u->stream>>>(
        u->grad[ca[l]].p, cc, u->grad[prev].p, cprev, n, hh, ww);
    hh /= 2;
    ww /= 2;
  }
  // encoder, level 4 down to 1; grad[eb[l]] holds the masked gradient of e{l}b's output
  for (int l = 3; l >= 0; l--) {
    const auto &La = u->layers[2 * l], &Lb = u->layers[2 * l + 1];
    if (l < 3) {
      // skip gradient: pool path (from level l+1's input) + concat path (channels cprev..)
      const int cprev = l == 2 ? c[3] : c[l + 1];
      k_pool_grad<<<row_grid((long long)n * hh, ww * (c[l] / 8)), 256, 0, u->stream>>>(
          u->grad[pl[l]].p, u->act[eb[l]].p, u->grad[ca[l]].p, cprev + c[l], cprev,
          u->grad[eb[l]].p, n, hh, ww, c[l]);
    }
    const int src = l == 0 ? U::IN : pl[l - 1];
    const int cin = l == 0 ? 16 : c[l - 1];
    if ((rc = wgrad(u, Lb, u->grad[eb[l]].p, c[l], u->act[ea[l]].p, n, hh, ww))) return rc;
    if ((rc = conv(u, Lb, u->grad[eb[l]].p, Lb.wb, c[l], c[l], nullptr, u->grad[ea[l]].p, c[l], 0,
                   nullptr, u->act[ea[l]].p, 0, n, hh, ww)))
      return rc;
    if (l == 0) {
      // first layer: cin padded 1 -> 16; weight gradient through the padded scratch, then
      // channel 0 of it is the real gradient
      UCK(cudaMemsetAsync(u->g0, 0, sizeof(float) * 9 * La.cout * La.cin_pad, u->stream));
      if ((rc = wgrad(u, La, u->grad[ea[l]].p, c[l], u->act[src].p, n, hh, ww, u->g0))) return rc;
      k_fold_first<<<nblk(9LL * La.cout), 256, 0, u->stream>>>(u->g0, u->grads + La.w_off,
                                                               9 * La.cout, La.cin_pad);
      break;
    }
    if ((rc = wgrad(u, La, u->grad[ea[l]].p, c[l], u->act[src].p, n, hh, ww))) return rc;
    // gradient of the pooled input (no mask: pooling output is not a ReLU output)
    if ((rc = conv(u, La, u->grad[ea[l]].p, La.wb, c[l], cin, nullptr, u->grad[src].p, cin, 0,
                   nullptr, nullptr, 0, n, hh, ww)))
      return rc;
    hh *= 2;
    ww *= 2;
  }
  UCK(cudaGetLastError());
  return DS2D_OK;
}

}  // namespace

extern "C" {

int ds2d_unet_create(int base, int max_n, int max_h, int max_w, int device, ds2d_unet **out) {
  if (!out) return DS2D_E_ARG;
  *out = nullptr;
  if (base != 32 && base != 64)
    return unet_fail(nullptr, DS2D_E_ARG, "unet base channels must be 32 or 64");
  if (max_n < 1 || max_h < 8 || max_w < 8 || max_h % 8 || max_w % 8)
    return unet_fail(nullptr, DS2D_E_ARG, "unet: max_n >= 1, max_h / max_w multiples of 8");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess)
    return unet_fail(nullptr, DS2D_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  ds2d_unet *u = new ds2d_unet();
  u->base = base; u->max_n = max_n; u->max_h = max_h; u->max_w = max_w; u->device = device;
  const int c[4] = {base, 2 * base, 4 * base, 8 * base};
  // layer table, same order as the oracle's layer_specs()
  auto add = [&](const char *name, int cin, int cout, int k) {
    ds2d_unet::Layer L;
    L.name = name; L.cin = cin; L.cout = cout; L.k = k;
    L.cin_pad = (cin + 15) / 16 * 16;
    L.nw = (long long)k * k * cout * cin;
    L.w_off = u->nparam;
    L.b_off = L.w_off + L.nw;
    u->nparam = L.b_off + cout;
    u->layers.push_back(L);
  };
  static const char *en[8] = {"e1a", "e1b", "e2a", "e2b", "e3a", "e3b", "e4a", "e4b"};
  int prev = 1;
  for (int l = 0; l < 4; l++) {
    add(en[2 * l], prev, c[l], 3);
    add(en[2 * l + 1], c[l], c[l], 3);
    prev = c[l];
  }
  static const char *dn[6] = {"d3a", "d3b", "d2a", "d2b", "d1a", "d1b"};
  for (int i = 0, l = 2; l >= 0; l--, i++) {
    add(dn[2 * i], prev + c[l], c[l], 3);
    add(dn[2 * i + 1], c[l], c[l], 3);
    prev = c[l];
  }
  add("out", c[0], 1, 1);
  int rc = DS2D_OK;
  auto A = [&](void **p, size_t bytes) {
    if (rc == DS2D_OK) rc = ualloc(u, p, bytes);
  };
  A((void **)&u->params, sizeof(float) * u->nparam);
  A((void **)&u->grads, sizeof(float) * u->nparam);
  A((void **)&u->m, sizeof(float) * u->nparam);
  A((void **)&u->v, sizeof(float) * u->nparam);
  for (auto &L : u->layers)
    if (L.k == 3) {
      A((void **)&L.wf, sizeof(bf16) * 9 * L.cout * L.cin_pad);
      A((void **)&L.wb, sizeof(bf16) * 9 * L.cout * L.cin);
      A((void **)&L.wfb, sizeof(bf16) * 9 * L.cout * L.cin_pad);
      A((void **)&L.wbb, sizeof(bf16) * 9 * L.cout * L.cin);
    }
  using U = ds2d_unet;
  const long long px0 = (long long)max_n * max_h * max_w;
  auto act = [&](int slot, int lev, int ch) {
    const long long px = px0 >> (2 * lev);
    u->act[slot].c = ch;
    u->grad[slot].c = ch;
    A((void **)&u->act[slot].p, sizeof(bf16) * px * ch);
    A((void **)&u->grad[slot].p, sizeof(bf16) * px * ch);
  };
  act(U::IN, 0, 16);
  act(U::E1A, 0, c[0]); act(U::E1B, 0, c[0]); act(U::P1, 1, c[0]);
  act(U::E2A, 1, c[1]); act(U::E2B, 1, c[1]); act(U::P2, 2, c[1]);
  act(U::E3A, 2, c[2]); act(U::E3B, 2, c[2]); act(U::P3, 3, c[2]);
  act(U::E4A, 3, c[3]); act(U::E4B, 3, c[3]);
  act(U::C3, 2, c[3] + c[2]); act(U::D3A, 2, c[2]); act(U::D3B, 2, c[2]);
  act(U::C2, 1, c[2] + c[1]); act(U::D2A, 1, c[1]); act(U::D2B, 1, c[1]);
  act(U::C1, 0, c[1] + c[0]); act(U::D1A, 0, c[0]); act(U::D1B, 0, c[0]);
  A((void **)&u->y, sizeof(float) * px0);
  A((void **)&u->dy, sizeof(float) * px0);
  A((void **)&u->part, sizeof(double) * kRedBlocks);
  A((void **)&u->g0, sizeof(float) * 9 * c[0] * 16);
  A((void **)&u->d_err, sizeof(int));
  if (rc == DS2D_OK) {
    cudaError_t ea = cudaFuncSetAttribute(k_conv3x3_tc<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          tc_smem_bytes<128>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_conv3x3_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                tc_smem_bytes<64>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_conv3x3_tc<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                tc_smem_bytes<32>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_conv3x3_tc<128, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                tc_smem_bytes<128, 2>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_conv3x3_tc<64, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                tc_smem_bytes<64, 2>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_conv3x3_tc<32, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                tc_smem_bytes<32, 2>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_conv3x3_tc<64, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                tc_smem_bytes<64, 4>());
    for (cudaError_t (*f)() : {tma_attr<128, 2, 3>, tma_attr<128, 2, 2>, tma_attr<128, 4, 3>,
                              tma_attr<128, 4, 2>, tma_attr<64, 2, 3>, tma_attr<64, 2, 2>,
                              tma_attr<64, 4, 3>, tma_attr<64, 4, 2>, tma_attr<32, 2, 3>,
                              tma_attr<32, 2, 2>, tma_attr<32, 4, 3>, tma_attr<32, 4, 2>,
                              tma_attr<96, 2, 2>, tma_attr<96, 2, 3>})
      if (ea == cudaSuccess) ea = f();
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_conv3x3_tc<32, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                tc_smem_bytes<32, 4>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_conv3x3_wgrad_tc<32>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, wg_tc_smem_bytes<32>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_conv3x3_wgrad_tc<16>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, wg_tc_smem_bytes<16>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_conv3x3_wgrad_tma<128>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, wt_smem_bytes<128>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_conv3x3_wgrad_tma<64>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, wt_smem_bytes<64>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_conv3x3_wgrad_tma<96>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, wt_smem_bytes<96>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_conv3x3_wgrad_tma<32>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, wt_smem_bytes<32>());
    if (ea == cudaSuccess)
      ea = cudaFuncSetAttribute(k_conv3x3_wgrad_tma<16>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, wt_smem_bytes<16>());
    if (ea != cudaSuccess)
      rc = unet_fail(u, DS2D_E_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(ea));
  }
  if (rc == DS2D_OK && cudaMallocHost((void **)&u->h_part, sizeof(double) * kRedBlocks) != cudaSuccess)
    rc = unet_fail(u, DS2D_E_NOMEM, "cudaMallocHost");
  if (rc != DS2D_OK) {
    g_unet_err = u->err;
    ds2d_unet_destroy(u);
    return rc;
  }
  *out = u;
  return DS2D_OK;
}

int ds2d_unet_destroy(ds2d_unet *u) {
  if (!u) return DS2D_OK;
  cudaSetDevice(u->device);
  if (u->stream) cudaStreamSynchronize(u->stream);
  for (void *p : u->allocs) cudaFree(p);
  if (u->h_part) cudaFreeHost(u->h_part);
  delete u;
  return DS2D_OK;
}

const char *ds2d_unet_last_error(const ds2d_unet *u) { return u ? u->err.c_str() : g_unet_err.c_str(); }

int ds2d_unet_set_stream(ds2d_unet *u, void *stream) {
  if (!u) return DS2D_E_ARG;
  u->stream = static_cast<cudaStream_t>(stream);
  return DS2D_OK;
}

long long ds2d_unet_num_params(const ds2d_unet *u) { return u ? u->nparam : 0; }

int ds2d_unet_set_params(ds2d_unet *u, const float *host, long long n) {
  if (!u || !host || n != u->nparam) return unet_fail(u, DS2D_E_ARG, "set_params: size mismatch");
  cudaSetDevice(u->device);
  UCK(cudaMemcpyAsync(u->params, host, sizeof(float) * n, cudaMemcpyHostToDevice, u->stream));
  UCK(cudaMemsetAsync(u->m, 0, sizeof(float) * n, u->stream));
  UCK(cudaMemsetAsync(u->v, 0, sizeof(float) * n, u->stream));
  UCK(cudaStreamSynchronize(u->stream));
  u->adam_t = 0;
  u->weights_dirty = true;
  return DS2D_OK;
}

int ds2d_unet_get_params(ds2d_unet *u, float *host, long long n) {
  if (!u || !host || n != u->nparam) return unet_fail(u, DS2D_E_ARG, "get_params: size mismatch");
  cudaSetDevice(u->device);
  UCK(cudaMemcpyAsync(host, u->params, sizeof(float) * n, cudaMemcpyDeviceToHost, u->stream));
  UCK(cudaStreamSynchronize(u->stream));
  return DS2D_OK;
}

int ds2d_unet_forward(ds2d_unet *u, const float *x, float *y, int n, int h, int w) {
  if (!u || !x || !y) return unet_fail(u, DS2D_E_ARG, "forward: null pointer");
  int rc;
  if ((rc = check_shape(u, n, h, w))) return rc;
  cudaSetDevice(u->device);
  if ((rc = forward(u, x, n, h, w))) return rc;
  UCK(cudaMemcpyAsync(y, u->y, sizeof(float) * n * h * w, cudaMemcpyDeviceToDevice, u->stream));
  return u->use_tc ? check_wait_flag(u) : DS2D_OK;
}

int ds2d_unet_set_option(ds2d_unet *u, const char *key, long long value) {
  if (!u || !key) return unet_fail(u, DS2D_E_ARG, "set_option: null argument");
  if (std::string(key) == "tcgen05") {
    u->use_tc = value != 0;
    return DS2D_OK;
  }
  if (std::string(key) == "tcgen05_wgrad") {
    u->tc_wgrad = value != 0;
    return DS2D_OK;
  }
  if (std::string(key) == "tcgen05_wgrad_tma") {
    u->tc_wgrad_tma = value != 0;
    return DS2D_OK;
  }
  if (std::string(key) == "tcgen05_tma") {
    u->tc_tma = value != 0;
    return DS2D_OK;
  }
  if (std::string(key) == "tcgen05_stages") {
    if (value != 2 && value != 3)
      return unet_fail(u, DS2D_E_ARG, "tcgen05_stages must be 2 or 3");
    u->tc_stages = (int)value;
    return DS2D_OK;
  }
  if (std::string(key) == "tcgen05_rows") {
    if (value != 1 && value != 2 && value != 4)
      return unet_fail(u, DS2D_E_ARG, "tcgen05_rows must be 1, 2 or 4");
    u->tc_rows = (int)value;
    return DS2D_OK;
  }
  return unet_fail(u, DS2D_E_ARG, std::string("unknown option ") + key);
}

int ds2d_unet_loss_grad(ds2d_unet *u, const float *x, const float *target, int n, int h, int w,
                        double *loss, float *grads_host) {
  if (!u || !x || !target) return unet_fail(u, DS2D_E_ARG, "loss_grad: null pointer");
  int rc;
  if ((rc = check_shape(u, n, h, w))) return rc;
  cudaSetDevice(u->device);
  if ((rc = forward(u, x, n, h, w))) return rc;
  const long long npx = (long long)n * h * w;
  k_mse<<<kRedBlocks, 256, 0, u->stream>>>(u->y, target, u->dy, npx, u->part);
  if ((rc = backward(u, n, h, w))) return rc;
  UCK(cudaMemcpyAsync(u->h_part, u->part, sizeof(double) * kRedBlocks, cudaMemcpyDeviceToHost,
                      u->stream));
  if (grads_host)
    UCK(cudaMemcpyAsync(grads_host, u->grads, sizeof(float) * u->nparam, cudaMemcpyDeviceToHost,
                        u->stream));
  UCK(cudaStreamSynchronize(u->stream));
  if (u->use_tc && (rc = check_wait_flag(u))) return rc;
  if (loss) {
    double s = 0;
    for (int i = 0; i < kRedBlocks; i++) s += u->h_part[i];
    *loss = s / (double)npx;
  }
  return DS2D_OK;
}

int ds2d_unet_adam_step(ds2d_unet *u, float lr, float beta1, float beta2, float eps) {
  if (!u) return DS2D_E_ARG;
  cudaSetDevice(u->device);
  u->adam_t++;
  const float c1 = 1.f - (float)std::pow((double)beta1, (double)u->adam_t);
  const float c2 = 1.f - (float)std::pow((double)beta2, (double)u->adam_t);
  k_adam<<<nblk(u->nparam), 256, 0, u->stream>>>(u->params, u->grads, u->m, u->v, u->nparam, lr,
                                                 beta1, beta2, eps, c1, c2);
  UCK(cudaGetLastError());
  u->weights_dirty = true;
  return DS2D_OK;
}

}  // extern "C"
