// Grouped BF16 or TF32 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a), FP32
// accumulation in tensor memory.  Used for the reverse-sketch contractions of
// tt_recursive_sketch (src/sketches.jl:1602-1638, :1648-1713) in the mixed-precision roundings:
//   C(i, j) = alpha * sum_k A(i, k) * B(j, k),   A and B K-major, BF16 (kind::f16) or FP32
//   read as TF32 (kind::tf32), row stride lda/ldb a multiple of 8 (BF16) or 4 (FP32)
//   elements, K zero padded to that multiple.
// Tile 128 x 128 x (128 bytes of K: 64 BF16 or 32 FP32), one CTA (4 warps) per output tile; the
// MMA's N is the tile's column count rounded up to 16, so narrow problems do not pay for 128.
// Operand tiles are staged with cp.async into the 128-byte-swizzled K-major layout that the
// UMMA shared-memory descriptors describe, in a two-stage ring: while one elected thread issues
// a stage's four tcgen05.mma (M=128, N<=128, 32 bytes of K each) and tcgen05.commit arrives on
// the stage's mbarrier, the next stage's loads are in flight.  The epilogue reads the
// accumulator with tcgen05.ld (32x32b) and writes FP64 / FP32 outputs and an operand-typed (BF16
// or FP32) output with arbitrary (split) row and column strides.
// Every mbarrier wait is bounded (by a device-wide limit that a test may lower): on timeout the
// kernel raises DFLAG_TIMEOUT, waits with the full limit for the MMAs it did issue, so that tensor
// memory is never released under them, frees its tensor memory and returns.
#include <cuda_bf16.h>

#include "kernels.cuh"

namespace ttc {
namespace {
// 128 x 128 tiles and a two-stage ring keep the shared memory at 65 KB, three CTAs per SM, so
// that one CTA's epilogue overlaps another's MMAs; measured on the config-5 sketch shapes, that
// beat a four-stage ring of 128 x 256 tiles at one CTA per SM by 1.7x to 2x.
constexpr int BM = 128, BN = 128, NT = 128, STAGES = 2;
constexpr int A_TILE = BM * 128;                        // 16 KB (128 B of K per row)
constexpr int B_TILE = BN * 128;                        // 16 KB
constexpr int STAGE_BYTES = A_TILE + B_TILE;
constexpr uint32_t TMEM_COLS = 128;
constexpr long long WAIT_LIMIT = 1LL << 24;             // bounded mbarrier polls
__device__ long long g_tc_wait_limit = WAIT_LIMIT;      // lowered only by a test hook

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async_16(uint32_t dst, const void* src, bool valid) {
  const int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait; returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit) {
  for (long long i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t make_sdesc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);            // start address
  d |= (uint64_t)1 << 16;                             // leading byte offset (unused for SW128 K-major)
  d |= (uint64_t)(1024 >> 4) << 32;                   // stride byte offset
  d |= (uint64_t)1 << 46;                             // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                             // layout: SWIZZLE_128B
  return d;
}

// Instruction descriptor: D=F32 (bits 4-5), A and B format (bits 7-9, 10-12: 1 = BF16 for
// kind::f16, 2 = TF32 for kind::tf32; A and B always the same type), both K-major, N>>3 at bit
// 17, M>>4 at bit 24.
template <bool TF32>
__host__ __device__ constexpr uint32_t idesc(int n_mma) {
  return (1u << 4) | ((TF32 ? 2u : 1u) << 7) | ((TF32 ? 2u : 1u) << 10) | ((uint32_t)(n_mma >> 3) << 17) |
         ((uint32_t)(BM >> 4) << 24);
}

template <bool TF32>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t id, uint32_t accumulate) {
  if constexpr (TF32)
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(id), "r"(accumulate)
        : "memory");
  else
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(id), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ int find_desc(const Bf16GemmDesc* __restrict__ d, int nd, long long tile) {
  int lo = 0, hi = nd - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (d[mid].tile_start <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}
}  // namespace

template <bool TF32>
__global__ void __launch_bounds__(NT, 1) gemm_bf16_tc_kernel(const Bf16GemmDesc* __restrict__ descs, int nd, int* flags) {
  constexpr int EB = TF32 ? 4 : 2;         // operand element bytes
  constexpr int BK = 128 / EB;             // K elements per 128-byte tile row
  constexpr int CH = 16 / EB;              // K elements per 16-byte chunk
  extern __shared__ __align__(1024) unsigned char dsm[];
  __shared__ uint64_t mbar[STAGES];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int s_last;                   // last iteration whose MMAs were issued (-1: none)
  // 1024-byte aligned operand ring: stage s holds A at s*STAGE_BYTES, B after it
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(dsm) + 1023) & ~uintptr_t(1023));

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long tile = blockIdx.x;
  const Bf16GemmDesc D = descs[find_desc(descs, nd, tile)];
  const int tm = (D.m + BM - 1) / BM, tn = (D.n + BN - 1) / BN;
  const long long local = tile - D.tile_start;
  if (local < 0 || local >= (long long)tm * tn) return;
  const int bm = (int)(local % tm), bn = (int)(local / tm);
  const int row0 = bm * BM, col0 = bn * BN;
  const int nk = (D.k + BK - 1) / BK;
  const int ncols = min(BN, D.n - col0);
  const int n_mma = (ncols + 15) & ~15;    // MMA N: the tile's columns rounded up to 16
  const uint32_t id = idesc<TF32>(n_mma);
  const long long wait_limit = g_tc_wait_limit;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(smem_u32(&mbar[s]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    s_last = -1;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  const char* Ag = reinterpret_cast<const char*>(D.A);
  const char* Bg = reinterpret_cast<const char*>(D.B);

  // A: 1024 16-byte chunks per tile (8 per thread); B: 8 chunks per row, n_mma rows
  auto load_stage = [&](int kt, int s) {
    const int k0 = kt * BK;
    const uint32_t sa = smem_u32(base + s * STAGE_BYTES), sb = sa + A_TILE;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const int idx = tid + NT * t;
      const int r = idx >> 3, c = idx & 7;
      const int kk = k0 + c * CH;
      const uint32_t off = (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4));
      const int gi = row0 + r;
      const bool va = (gi < D.m) && (kk < D.k);
      cp_async_16(sa + off, va ? (const void*)(Ag + ((long long)gi * D.lda + kk) * EB) : (const void*)Ag, va);
    }
    for (int idx = tid; idx < n_mma * 8; idx += NT) {
      const int r = idx >> 3, c = idx & 7;
      const int kk = k0 + c * CH;
      const uint32_t off = (uint32_t)(r * 128 + ((c ^ (r & 7)) << 4));
      const int gj = col0 + r;
      const bool vb = (gj < D.n) && (kk < D.k);
      cp_async_16(sb + off, vb ? (const void*)(Bg + ((long long)gj * D.ldb + kk) * EB) : (const void*)Bg, vb);
    }
    cp_async_commit();
  };

  // prologue: stages 0 .. STAGES-2 in flight (an empty group keeps the group count uniform)
#pragma unroll
  for (int p = 0; p < STAGES - 1; ++p) {
    if (p < nk) load_stage(p, p);
    else cp_async_commit();
  }
  bool ok = true;
  for (int kt = 0; kt < nk; ++kt) {
    const int s = kt % STAGES;
    const int next = kt + STAGES - 1;
    if (next < nk) {
      // the stage of `next` was read by the MMAs of iteration kt - 1
      if (kt >= 1) ok = ok && mbar_wait(smem_u32(&mbar[next % STAGES]), (uint32_t)(((kt - 1) / STAGES) & 1), wait_limit);
      load_stage(next, next % STAGES);
    } else {
      cp_async_commit();
    }
    cp_async_wait<STAGES - 1>();            // this iteration's stage has landed
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0 && ok) {
      tc_fence_after();
      const uint32_t sa = smem_u32(base + s * STAGE_BYTES), sb = sa + A_TILE;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)        // 32 bytes of K per MMA
        umma<TF32>(tmem, make_sdesc(sa + kk * 32), make_sdesc(sb + kk * 32), id, (kt > 0 || kk > 0) ? 1u : 0u);
      umma_commit(smem_u32(&mbar[s]));
      s_last = kt;
    }
    __syncthreads();
  }
  cp_async_wait<0>();
  if (nk > 0) ok = ok && mbar_wait(smem_u32(&mbar[(nk - 1) % STAGES]), (uint32_t)(((nk - 1) / STAGES) & 1), wait_limit);
  ok = __syncthreads_and(ok) != 0;
  if (!ok) {
    // drain with the full limit: the MMAs that were issued finish before tensor memory is freed
    const int last = s_last;
    if (last >= 0) mbar_wait(smem_u32(&mbar[last % STAGES]), (uint32_t)((last / STAGES) & 1), WAIT_LIMIT);
  }
  tc_fence_after();
  if (!ok) {
    if (tid == 0) atomicOr(flags, DFLAG_TIMEOUT);
  } else {
    // Epilogue: warp w owns accumulator rows 32w..32w+31 (TMEM lanes).
    const int row = row0 + warp * 32 + lane;
    const long long roff64 = (long long)(row % D.m0) * D.c_i0 + (long long)(row / D.m0) * D.c_i1;
    const long long roff16 = (long long)(row % D.m0) * D.h_i0 + (long long)(row / D.m0) * D.h_i1;
    for (int c0 = 0; c0 < n_mma; c0 += 16) {
      float v[16];
      if (nk > 0) tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      else {
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = 0.f;
      }
      if (row < D.m) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int col = col0 + c0 + i;
          if (col < D.n) {
            const double x = D.alpha * (double)v[i];
            const int j1 = D.n0 > 0 ? col / D.n0 : 0, j0 = col - j1 * D.n0;
            const long long co64 = (long long)j0 * D.c_j + (long long)j1 * D.c_j1;
            if (D.C64) D.C64[roff64 + co64] = x;
            if (D.C32) reinterpret_cast<float*>(D.C32)[roff64 + co64] = (float)x;
            if (D.C16) {   // operand-typed output
              const long long co16 = (long long)j0 * D.h_j + (long long)j1 * D.h_j1;
              if constexpr (TF32) reinterpret_cast<float*>(D.C16)[roff16 + co16] = round_tf32((float)x);
              else reinterpret_cast<__nv_bfloat16*>(D.C16)[roff16 + co16] = __double2bfloat16(x);
            }
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

long long bf16_gemm_tiles(const Bf16GemmDesc& d) {
  if (d.m <= 0 || d.n <= 0) return 0;
  return (long long)((d.m + BM - 1) / BM) * ((d.n + BN - 1) / BN);
}

namespace {
template <bool TF32>
void launch_tc(const Bf16GemmDesc* d, int nd, long long total_tiles, cudaStream_t s, int* d_flags) {
  const int smem = STAGES * STAGE_BYTES + 1024;
  static PerDeviceOnce attr_once;
  int dev = 0;
  TTC_CUDA(cudaGetDevice(&dev));
  attr_once.run(dev, [smem] {
    TTC_CUDA(cudaFuncSetAttribute(gemm_bf16_tc_kernel<TF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  });
  gemm_bf16_tc_kernel<TF32><<<(unsigned)total_tiles, NT, smem, s>>>(d, nd, d_flags);
  TTC_CHECK_LAUNCH();
}
}  // namespace

void set_tc_wait_limit(long long polls) {
  // 0: every wait gives up at once (a test of the timeout path; the drain of issued MMAs keeps
  // its full limit)
  TTC_REQUIRE(polls >= 0, TTC_EARG, "the tensor-core wait limit must not be negative");
  TTC_CUDA(cudaMemcpyToSymbol(g_tc_wait_limit, &polls, sizeof(polls)));
}

void launch_gemm_bf16_tc(const Bf16GemmDesc* d, int nd, long long total_tiles, cudaStream_t s, int* d_flags,
                         bool tf32) {
  if (nd <= 0 || total_tiles <= 0) return;
  if (tf32) launch_tc<true>(d, nd, total_tiles, s, d_flags);
  else launch_tc<false>(d, nd, total_tiles, s, d_flags);
}

}  // namespace ttc
