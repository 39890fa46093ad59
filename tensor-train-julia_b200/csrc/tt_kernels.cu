// Bandwidth-bound helper kernels of libttcuda: strided tensor copies (layout changes
// between the Julia core layout and the internal one), zero fills, sums of squares,
// the truncation rule, singular-vector selection, the MPO x TT apply and the Philox
// sketch generator.  Grids are sized in multiples of the SM count where they stream.
#include "kernels.cuh"

namespace ttc {
namespace {
constexpr int NT = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
}  // namespace

// ---------------------------------------------------------------- strided copy
// A 2-D copy that is contiguous along dim 0 on one side and along dim 1 on the other (a
// transpose) goes through 32 x 32 shared-memory tiles so both the loads and the stores are
// coalesced; every other copy maps consecutive threads to consecutive dim-0 elements, with
// 32-bit index arithmetic when the copy has fewer than 2^31 elements.
__global__ void __launch_bounds__(NT) copy4_kernel(const CopyDesc* __restrict__ descs) {
  __shared__ double tile[32][33];
  const CopyDesc D = descs[blockIdx.y];
  long long e0 = D.ext[0], e1 = D.ext[1];
  const long long e2 = D.ext[2], e3 = D.ext[3];
  long long s0 = D.ss[0], s1 = D.ss[1], d0 = D.ds[0], d1 = D.ds[1];
  if (e2 == 1 && e3 == 1 && s1 == 1 && d0 == 1 && s0 != 1) {   // orient: source contiguous along dim 0
    long long t = e0; e0 = e1; e1 = t;
    t = s0; s0 = s1; s1 = t;
    t = d0; d0 = d1; d1 = t;
  }
  if (e2 == 1 && e3 == 1 && s0 == 1 && d1 == 1 && d0 != 1 && e0 >= 32 && e1 >= 32) {
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;     // 32 x 8 threads
    const long long t0 = (e0 + 31) / 32, ntile = t0 * ((e1 + 31) / 32);
    for (long long ti = blockIdx.x; ti < ntile; ti += gridDim.x) {
      const long long b0 = (ti % t0) * 32, b1 = (ti / t0) * 32;
#pragma unroll
      for (int k = 0; k < 32; k += NT / 32) {
        const long long i0 = b0 + tx, i1 = b1 + ty + k;
        if (i0 < e0 && i1 < e1) tile[ty + k][tx] = D.src[i0 + i1 * s1];
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < 32; k += NT / 32) {
        const long long i0 = b0 + ty + k, i1 = b1 + tx;
        if (i0 < e0 && i1 < e1) D.dst[i0 * d0 + i1] = D.alpha * tile[tx][ty + k];
      }
      __syncthreads();
    }
    return;
  }
  const long long total = e0 * e1 * e2 * e3;
  if (total < (1LL << 31)) {
    const unsigned u0 = (unsigned)e0, u1 = (unsigned)e1, u2 = (unsigned)e2;
    for (unsigned e = blockIdx.x * NT + threadIdx.x; e < (unsigned)total; e += gridDim.x * NT) {
      unsigned r = e;
      const unsigned i0 = r % u0; r /= u0;
      const unsigned i1 = r % u1; r /= u1;
      const unsigned i2 = r % u2, i3 = r / u2;
      const double v = D.src[i0 * s0 + i1 * s1 + i2 * D.ss[2] + i3 * D.ss[3]];
      D.dst[i0 * d0 + i1 * d1 + i2 * D.ds[2] + i3 * D.ds[3]] = D.alpha * v;
    }
    return;
  }
  for (long long e = (long long)blockIdx.x * NT + threadIdx.x; e < total; e += (long long)gridDim.x * NT) {
    long long r = e;
    const long long i0 = r % e0; r /= e0;
    const long long i1 = r % e1; r /= e1;
    const long long i2 = r % e2; const long long i3 = r / e2;
    const double v = D.src[i0 * s0 + i1 * s1 + i2 * D.ss[2] + i3 * D.ss[3]];
    D.dst[i0 * d0 + i1 * d1 + i2 * D.ds[2] + i3 * D.ds[3]] = D.alpha * v;
  }
}

void launch_copy(const CopyDesc* d, int count, long long max_elems, cudaStream_t s) {
  if (count <= 0 || max_elems <= 0) return;
  // about four elements per thread; with `count` copies in the grid's y dimension
  const long long blocks = std::min<long long>((max_elems + 4 * NT - 1) / (4 * NT), 148LL * 8);
  dim3 grid((unsigned)blocks, (unsigned)count);
  copy4_kernel<<<grid, NT, 0, s>>>(d);
  TTC_CHECK_LAUNCH();
}

__global__ void zero_kernel(const ZeroDesc* __restrict__ descs) {
  const ZeroDesc D = descs[blockIdx.y];
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < D.n; e += (long long)gridDim.x * blockDim.x)
    D.p[e] = 0.0;
}

void launch_zero(const ZeroDesc* d, int count, long long max_n, cudaStream_t s) {
  if (count <= 0 || max_n <= 0) return;
  const long long blocks = std::min<long long>((max_n + NT - 1) / NT, 148LL * 8);
  zero_kernel<<<dim3((unsigned)blocks, (unsigned)count), NT, 0, s>>>(d);
  TTC_CHECK_LAUNCH();
}

// ---------------------------------------------------------------- sum of squares
__global__ void sumsq_kernel(const NormDesc* __restrict__ descs) {
  __shared__ double red[NT / 32];
  const NormDesc D = descs[blockIdx.x];
  double a = 0.0;
  for (long long e = threadIdx.x; e < D.n; e += NT) a = fma(D.p[e], D.p[e], a);
  a = warp_sum(a);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < NT / 32; ++i) s += red[i];
    *D.out = s;
  }
}

void launch_sumsq(const NormDesc* d, int count, cudaStream_t s) {
  if (count <= 0) return;
  sumsq_kernel<<<count, NT, 0, s>>>(d);
  TTC_CHECK_LAUNCH();
}

// ---------------------------------------------------------------- truncation rule
// floor(s, tol; degen_tol=1e-5) of src/tt_rounding.jl:297-315 on the sorted values, then
// k = min(k, rmax, #(s > 0)) (src/tt_rounding.jl:198-199).  One warp per problem: the lanes
// gather the sorted values into shared memory and count the positive ones; lane 0 then runs the
// rule as a sequential FP64 scan (the sums in the reference's order) over shared memory, eight
// loads in flight at a time.
constexpr int kTruncStage = 2048;
__global__ void __launch_bounds__(32) truncate_kernel(const TruncDesc* __restrict__ descs, int count, double tol,
                                                      long long rmax) {
  __shared__ double sv[kTruncStage];
  const int p = blockIdx.x, lane = threadIdx.x;
  if (p >= count) return;
  const TruncDesc D = descs[p];
  const int d = D.n;
  const bool staged = d <= kTruncStage;
  int npos = 0;
  for (int i = lane; i < d; i += 32) {
    if (staged) sv[i] = D.sigma[D.perm[i]];
    npos += (D.sigma[i] > 0.0);
  }
  npos = __reduce_add_sync(0xffffffffu, npos);
  __syncwarp();
  if (lane != 0) return;
  auto val = [&](int i) { return staged ? sv[i] : D.sigma[D.perm[i]]; };
  int k;
  if (d <= 0) { k = 0; }
  else if (tol == 0.0) { k = d; }
  else {
    double norm2 = 0.0;
#pragma unroll 8
    for (int i = 0; i < d; ++i) { const double v = val(i); norm2 = fma(v, v, norm2); }
    int i = d;
    double weight = 0.0;
    const double thr = tol * tol * norm2;
    while (i > 0 && weight < thr) {
      const double v = val(i - 1);
      weight = fma(v, v, weight);
      --i;
    }
    ++i;
    while (i < d) {
      const double a = val(i - 1), b = val(i);
      const double ratio = b / a;
      if (isfinite(ratio) && fabs(1.0 - ratio) <= 1e-5) ++i; else break;
    }
    k = i;
  }
  if (k > npos) k = npos;
  if ((long long)k > rmax) k = (int)rmax;
  *D.rank_out = k;
}

void launch_truncate(const TruncDesc* d, int count, double tol, long long rmax, cudaStream_t s) {
  if (count <= 0) return;
  truncate_kernel<<<count, 32, 0, s>>>(d, count, tol, rmax);
  TTC_CHECK_LAUNCH();
}

// ---------------------------------------------------------------- column selection
__global__ void select_kernel(const SelectDesc* __restrict__ descs) {
  const SelectDesc D = descs[blockIdx.y];
  const int k = *D.rank;
  const int rows = max(D.rows, D.zrows);
  const long long total = (long long)rows * D.cols;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e / rows), r = (int)(e - (long long)c * rows);
    double v = 0.0;
    if (c < k && r < D.rows) {
      const int src = D.perm[c];
      v = D.X[(long long)src * D.ldx + r];
      if (D.scale == 1) { const double s = D.sigma[src]; v = (s > 0.0) ? v / s : 0.0; }
      else if (D.scale == 2) v *= D.sigma[src];
    }
    D.U[(long long)c * D.ldu + r] = v;
  }
}

void launch_select(const SelectDesc* d, int count, int max_rows, int max_cols, cudaStream_t s) {
  if (count <= 0) return;
  const long long total = (long long)max_rows * max_cols;
  const long long blocks = std::max<long long>(1, std::min<long long>((total + NT - 1) / NT, 148LL * 4));
  select_kernel<<<dim3((unsigned)blocks, (unsigned)count), NT, 0, s>>>(d);
  TTC_CHECK_LAUNCH();
}

// ---------------------------------------------------------------- MPO x TT apply
// Y[(a + R*nu), i, (a' + R'*nu')] = sum_j H[a, i, j, a'] * V[nu, j, nu'] (internal layouts;
// src/tt_operations.jl:184).  HBM-bound on the output's write stream: the output core is R R'
// times the input core, and H and V are read a few times over from L2.
// Output column w = i + n (a' + R' nu') is a contiguous run of U = R r elements (u = a + R nu).  A
// CTA takes one nu' of one problem: it stages V[:, :, nu'] (n r values) in shared memory once, then
// for each (a', i) the n R operator entries H[:, i, :, a'], and writes the n R' columns of that nu'
// with consecutive threads on consecutive u (coalesced stores).  Each thread follows its (a, nu)
// through the column by constant increments (the block size divided by R), with no division per
// element; an element costs 2n shared-memory loads, n FMAs and one store.
__global__ void apply_kernel(const ApplyDesc* __restrict__ descs) {
  extern __shared__ double asm_[];
  const ApplyDesc D = descs[blockIdx.y];
  const int nun = blockIdx.x;
  if (nun >= D.rn) return;                         // uniform: the launch covers the largest rn
  const int R = D.R, n = D.n, Rn = D.Rn, r = D.r;
  const long long U = (long long)R * r;
  double* vs = asm_;                               // vs[j r + nu] = V[nu, j, nu']
  double* hs = asm_ + (size_t)n * r;               // hs[a + R (i + n j)] = H[a, i, j, a'] of one a'
  for (int e = threadIdx.x; e < n * r; e += blockDim.x) {
    const int j = e / r, nu = e - j * r;
    vs[e] = D.V[nu + (long long)r * (j + (long long)n * nun)];
  }
  const int stA = blockDim.x % R, stNu = blockDim.x / R;
  const int a0 = threadIdx.x % R, nu0 = threadIdx.x / R;
  const long long cstride = U;                     // output column i + 1 follows column i
  for (int an = 0; an < Rn; ++an) {
    __syncthreads();                               // the previous a's reads of hs are done
    const double* hsrc = D.H + (long long)R * n * n * an;   // H[:, :, :, a'] is contiguous
    for (int e = threadIdx.x; e < R * n * n; e += blockDim.x) hs[e] = hsrc[e];
    __syncthreads();
    // the n columns (i = 0 .. n-1) of this a' and nu' together: vs is read once per (u, j)
    double* y = D.Y + U * (long long)n * (an + (long long)Rn * nun);
    int a = a0, nu = nu0;
    for (long long u = threadIdx.x; u < U; u += blockDim.x) {
      if (n == 2) {
        const double v0 = vs[nu], v1 = vs[r + nu];
        y[u] = fma(hs[a + 2 * R], v1, hs[a] * v0);
        y[u + cstride] = fma(hs[a + 3 * R], v1, hs[a + R] * v0);
      } else {
        for (int i = 0; i < n; ++i) {
          double acc = 0.0;
          for (int j = 0; j < n; ++j) acc = fma(hs[a + R * (i + n * j)], vs[j * r + nu], acc);
          y[u + cstride * i] = acc;
        }
      }
      a += stA; nu += stNu;
      if (a >= R) { a -= R; ++nu; }
    }
  }
}

void launch_apply(const ApplyDesc* d, int count, int max_rn, int max_smem_doubles, cudaStream_t s) {
  if (count <= 0 || max_rn <= 0) return;
  const size_t smem = sizeof(double) * (size_t)std::max(1, max_smem_doubles);
  TTC_REQUIRE(smem <= 200 * 1024, TTC_EDIM, "apply: operator and vector ranks too large for the staged slices");
  static PerDeviceOnce attr_once;
  int dev = 0;
  TTC_CUDA(cudaGetDevice(&dev));
  attr_once.run(dev, [] {
    TTC_CUDA(cudaFuncSetAttribute(apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  });
  apply_kernel<<<dim3((unsigned)max_rn, (unsigned)count), NT, smem, s>>>(d);
  TTC_CHECK_LAUNCH();
}

// ---------------------------------------------------------------- Philox sketch generator
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11): counter (e/4, stream, 0, 0), key (seed lo, seed hi); Box-Muller on the word pairs.
// The oracle's philox_normals() computes the same sequence on the host.
__device__ __forceinline__ void philox10(unsigned c[4], unsigned k0, unsigned k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const unsigned long long p0 = 0xD2511F53ull * c[0];
    const unsigned long long p1 = 0xCD9E8D57ull * c[2];
    const unsigned hi0 = (unsigned)(p0 >> 32), lo0 = (unsigned)p0;
    const unsigned hi1 = (unsigned)(p1 >> 32), lo1 = (unsigned)p1;
    const unsigned n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
}

__global__ void philox_kernel(const PhiloxDesc* __restrict__ descs) {
  const PhiloxDesc D = descs[blockIdx.y];
  const long long nctr = (D.count + 3) / 4;
  const double inv = 1.0 / 4294967296.0;
  const double two_pi = 6.283185307179586476925286766559;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nctr; q += (long long)gridDim.x * blockDim.x) {
    unsigned c[4] = {(unsigned)q, D.stream, 0u, 0u};
    philox10(c, (unsigned)D.seed, (unsigned)(D.seed >> 32));
    const double u0 = (c[0] + 0.5) * inv, u1 = (c[1] + 0.5) * inv;
    const double u2 = (c[2] + 0.5) * inv, u3 = (c[3] + 0.5) * inv;
    const double r01 = sqrt(-2.0 * log(u0)), r23 = sqrt(-2.0 * log(u2));
    double s1, c1, s3, c3;
    sincos(two_pi * u1, &s1, &c1);
    sincos(two_pi * u3, &s3, &c3);
    const double z[4] = {r01 * c1, r01 * s1, r23 * c3, r23 * s3};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const long long e = 4 * q + t;
      if (e < D.count) D.dst[e] = D.scale * z[t];
    }
  }
}

void launch_philox(const PhiloxDesc* d, int count, long long max_count, cudaStream_t s) {
  if (count <= 0 || max_count <= 0) return;
  const long long blocks = std::min<long long>(((max_count + 3) / 4 + NT - 1) / NT, 148LL * 8);
  philox_kernel<<<dim3((unsigned)blocks, (unsigned)count), NT, 0, s>>>(d);
  TTC_CHECK_LAUNCH();
}

}  // namespace ttc
