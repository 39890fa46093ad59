// Plan execution, small control kernels, context and batch management of libttcuda.
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cmath>
#include <cuda_bf16.h>

#include "builder.cuh"
#include "regions.cuh"

namespace ttc {

// ---------------------------------------------------------------- control kernels
__global__ void zerochk_kernel(const ZeroChkDesc* d, int count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) *d[i].flag = (sqrt(*d[i].sumsq) < d[i].tol) ? 1 : 0;
}
void launch_zerochk(const ZeroChkDesc* d, int count, cudaStream_t s) {
  if (count <= 0) return;
  zerochk_kernel<<<(count + 127) / 128, 128, 0, s>>>(d, count);
  TTC_CHECK_LAUNCH();
}

// One CTA per problem: the largest sigma (block reduction), then the column scaling.
__global__ void pinv_scale_kernel(const PinvScaleDesc* descs) {
  const PinvScaleDesc D = descs[blockIdx.x];
  __shared__ double s_max[32];
  double mx = 0.0;
  for (int i = threadIdx.x; i < D.n; i += blockDim.x) mx = fmax(mx, D.sigma[i]);
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = mx;
  __syncthreads();
  mx = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mx = fmax(mx, s_max[w]);
  const double thr = D.eps * mx;
  for (long long e = threadIdx.x; e < (long long)D.m * D.n; e += blockDim.x) {
    const int i = (int)(e / D.m), r = (int)(e - (long long)i * D.m);
    const double s = D.sigma[i];
    double* x = D.X + (long long)i * D.ldx + r;
    *x = (s > thr) ? *x / (s * s) : 0.0;
  }
}
void launch_pinv_scale(const PinvScaleDesc* d, int count, cudaStream_t s) {
  if (count <= 0) return;
  pinv_scale_kernel<<<count, 256, 0, s>>>(d);
  TTC_CHECK_LAUNCH();
}

__global__ void final_kernel(const FinalDesc* descs) {
  const FinalDesc D = descs[blockIdx.y];
  if (*D.flag == 0) return;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < D.n; e += (long long)gridDim.x * blockDim.x)
    D.cores[e] = 0.0;
  if (blockIdx.x == 0)
    for (int i = threadIdx.x; i < D.nrks; i += blockDim.x) D.rks[i] = D.rks_restore[i];
}
void launch_final(const FinalDesc* d, int count, long long max_n, cudaStream_t s) {
  if (count <= 0) return;
  const long long blocks = std::max<long long>(1, std::min<long long>((max_n + 255) / 256, 148LL * 4));
  final_kernel<<<dim3((unsigned)blocks, (unsigned)count), 256, 0, s>>>(d);
  TTC_CHECK_LAUNCH();
}

__global__ void setrank_kernel(const SetRankDesc* d) {
  const SetRankDesc D = d[blockIdx.x];
  for (int i = threadIdx.x; i < D.n; i += blockDim.x) D.dst[i] = D.src[i];
}
void launch_setrank(const SetRankDesc* d, int count, cudaStream_t s) {
  if (count <= 0) return;
  setrank_kernel<<<count, 64, 0, s>>>(d);
  TTC_CHECK_LAUNCH();
}

__global__ void cvt_f32_kernel(const CvtDesc* descs) {
  const CvtDesc D = descs[blockIdx.y];
  const long long total = D.rows * D.cols;
  float* dst = reinterpret_cast<float*>(D.dst);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long i = e % D.rows, j = e / D.rows;
    dst[i * D.ds_i + j * D.ds_j] = (float)(D.alpha * D.src[i * D.ss_i + j * D.ss_j]);
  }
}
void launch_cvt_f32(const CvtDesc* d, int count, long long max_elems, cudaStream_t s) {
  if (count <= 0 || max_elems <= 0) return;
  const long long blocks = std::min<long long>((max_elems + 255) / 256, 148LL * 8);
  cvt_f32_kernel<<<dim3((unsigned)blocks, (unsigned)count), 256, 0, s>>>(d);
  TTC_CHECK_LAUNCH();
}
__global__ void widen_kernel(const CvtDesc* descs) {
  const CvtDesc D = descs[blockIdx.y];
  const long long total = D.rows * D.cols;
  const float* src = reinterpret_cast<const float*>(D.src);
  double* dst = reinterpret_cast<double*>(D.dst);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long i = e % D.rows, j = e / D.rows;
    dst[i * D.ds_i + j * D.ds_j] = D.alpha * (double)src[i * D.ss_i + j * D.ss_j];
  }
}
void launch_widen(const CvtDesc* d, int count, long long max_elems, cudaStream_t s) {
  if (count <= 0 || max_elems <= 0) return;
  const long long blocks = std::min<long long>((max_elems + 255) / 256, 148LL * 8);
  widen_kernel<<<dim3((unsigned)blocks, (unsigned)count), 256, 0, s>>>(d);
  TTC_CHECK_LAUNCH();
}

template <typename T>
__global__ void cvt_bf16_kernel(const CvtDesc* descs) {
  const CvtDesc D = descs[blockIdx.y];
  const long long total = D.rows * D.cols;
  T* dst = reinterpret_cast<T*>(D.dst);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long i = e % D.rows, j = e / D.rows;
    const double v = D.alpha * D.src[i * D.ss_i + j * D.ss_j];
    if constexpr (sizeof(T) == 4) dst[i * D.ds_i + j * D.ds_j] = round_tf32((float)v);   // TF32 operand
    else dst[i * D.ds_i + j * D.ds_j] = __double2bfloat16(v);
  }
}
void launch_cvt_bf16(const CvtDesc* d, int count, long long max_elems, cudaStream_t s, bool f32) {
  if (count <= 0 || max_elems <= 0) return;
  const long long blocks = std::min<long long>((max_elems + 255) / 256, 148LL * 8);
  if (f32) cvt_bf16_kernel<float><<<dim3((unsigned)blocks, (unsigned)count), 256, 0, s>>>(d);
  else cvt_bf16_kernel<__nv_bfloat16><<<dim3((unsigned)blocks, (unsigned)count), 256, 0, s>>>(d);
  TTC_CHECK_LAUNCH();
}

// ---------------------------------------------------------------- plan
Plan::~Plan() {
  if (gexec) cudaGraphExecDestroy(gexec);
  if (d_blob) { region_remove(d_blob); cudaFree(d_blob); }
}

static void launch_op(ttc_context* c, const Plan& p, const Op& op);

// stages = false leaves the stage events out (graph capture: the whole run is timed by the
// begin/end events around the graph launch instead)
static void launch_ops(ttc_context* c, Plan& p, bool stages) {
  for (const Op& op : p.ops)
    if (stages || op.kind != OP_STAGE) launch_op(c, p, op);
}

static void launch_op(ttc_context* c, const Plan& p, const Op& op) {
  cudaStream_t s = c->stream;
  {
    const unsigned char* d = p.d_blob + op.off;
    switch (op.kind) {
      case OP_GEMM: launch_gemm_f64((const GemmDesc*)d, op.count, op.total, s); break;
      case OP_QR: launch_qr((const QRDesc*)d, op.count, op.a, s, c->d_flags); break;
      case OP_QAPPLY: launch_qr_apply((const QApplyDesc*)d, op.count, op.a, s); break;
      case OP_JACOBI:
        launch_jacobi((const JacobiDesc*)d, op.count, op.a, op.b, op.total != 0, s, c->d_flags, op.iw, (int)op.rmax);
        break;
      case OP_TRUNC: launch_truncate((const TruncDesc*)d, op.count, op.tol, op.rmax, s); break;
      case OP_SELECT: launch_select((const SelectDesc*)d, op.count, op.a, op.b, s); break;
      case OP_COPY: launch_copy((const CopyDesc*)d, op.count, op.total, s); break;
      case OP_ZERO: launch_zero((const ZeroDesc*)d, op.count, op.total, s); break;
      case OP_SUMSQ: launch_sumsq((const NormDesc*)d, op.count, s); break;
      case OP_APPLY: launch_apply((const ApplyDesc*)d, op.count, op.a, op.b, s); break;
      case OP_GEMM32: launch_gemm_f32((const GemmDesc*)d, op.count, op.total, s); break;
      case OP_CVT32: launch_cvt_f32((const CvtDesc*)d, op.count, op.total, s); break;
      case OP_WIDEN: launch_widen((const CvtDesc*)d, op.count, op.total, s); break;
      case OP_PHILOX: launch_philox((const PhiloxDesc*)d, op.count, op.total, s); break;
      case OP_BF16GEMM: launch_gemm_bf16_tc((const Bf16GemmDesc*)d, op.count, op.total, s, c->d_flags, op.a != 0); break;
      case OP_ZEROCHK: launch_zerochk((const ZeroChkDesc*)d, op.count, s); break;
      case OP_PINV_SCALE: launch_pinv_scale((const PinvScaleDesc*)d, op.count, s); break;
      case OP_FINAL: launch_final((const FinalDesc*)d, op.count, op.total, s); break;
      case OP_SETRANK: launch_setrank((const SetRankDesc*)d, op.count, s); break;
      case OP_CVT_BF16: launch_cvt_bf16((const CvtDesc*)d, op.count, op.total, s, op.a != 0); break;
      case OP_STAGE: TTC_CUDA(cudaEventRecord(c->ev[op.a], s)); break;
    }
  }
}

long long count_launches(const Plan& p) {
  long long n = 0;
  for (const Op& op : p.ops) n += (op.kind != OP_STAGE) + (op.kind == OP_JACOBI && op.iw ? 1 : 0);   // + order kernel
  return n;
}

static int op_kind(OpKind k) {
  switch (k) {
    case OP_GEMM: return TTC_KERN_GEMM_F64;
    case OP_GEMM32: return TTC_KERN_GEMM_F64;
    case OP_QR: return TTC_KERN_QR;
    case OP_QAPPLY: return TTC_KERN_QR;
    case OP_JACOBI: return TTC_KERN_JACOBI;
    case OP_BF16GEMM: return TTC_KERN_GEMM_BF16;
    case OP_APPLY: return TTC_KERN_APPLY;
    default: return TTC_KERN_OTHER;
  }
}

// Algorithmic FLOPs of one launch at the sizes its descriptors run with.  Without device
// bounds these are the capacity shapes the builder counts; with them (`val` reads a bound that
// the run wrote), the bounded block: the QR, Q application and Jacobi of the SVD sweep work on
// the rows left by the kept rank of the next bond, a GEMM with n_dev on its first *n_dev columns.
static double qr_flops(double m, double n, bool with_q) {
  const double k = std::min(m, n);
  return (with_q ? 2.0 : 1.0) * (2.0 * m * k * k - 2.0 * k * k * k / 3.0) + 2.0 * m * k * (n - k);
}
static double qapply_flops(double m, double K, double nb) { return 4.0 * m * K * nb - 2.0 * K * K * nb; }
static double jacobi_flops(double m, double n) { return 4.0 * m * n * n + 8.0 * n * n * n; }

static double bounded_flops(const Plan& p, const Op& op, const std::function<int(const int*)>& val) {
  const unsigned char* d = p.blob.data() + op.off;
  auto bnd = [&](int cap, const int* ptr, int mult) {
    return ptr ? std::min(cap, std::max(0, mult * val(ptr))) : cap;
  };
  double f = 0.0;
  switch (op.kind) {
    case OP_QR:
      for (int i = 0; i < op.count; ++i) {
        const QRDesc& q = ((const QRDesc*)d)[i];
        f += qr_flops(bnd(q.m, q.m_dev, q.m_mult), bnd(q.n, q.n_dev, q.n_mult), q.Q != nullptr);
      }
      return f;
    case OP_QAPPLY:
      for (int i = 0; i < op.count; ++i) {
        const QApplyDesc& q = ((const QApplyDesc*)d)[i];
        const int m = bnd(q.m, q.m_dev, q.m_mult);
        f += qapply_flops(m, std::min(q.K, m), bnd(q.nb, q.n_dev, 1));
      }
      return f;
    case OP_JACOBI:
      for (int i = 0; i < op.count; ++i) {
        const JacobiDesc& j = ((const JacobiDesc*)d)[i];
        const int m = bnd(j.m, j.m_dev, j.m_mult);
        f += jacobi_flops(m, j.m_dev ? std::min(j.n, m) : j.n);   // a bounded factor is m x m at most
      }
      return f;
    case OP_GEMM:
      for (int i = 0; i < op.count; ++i) {
        const GemmDesc& g = ((const GemmDesc*)d)[i];
        f += 2.0 * g.m * bnd(g.n, g.n_dev, 1) * (double)g.k * std::max(1, g.batch);
      }
      return f;
    default:
      return op.flops;
  }
}

// Profiled execution: an event pair around every launch, times accumulated per kernel family.
static void run_plan_profiled(ttc_context* c, Plan& p) {
  std::vector<cudaEvent_t> ev;
  std::vector<int> kinds;
  std::vector<double> flops;
  for (const Op& op : p.ops) {
    if (op.kind == OP_STAGE) continue;
    flops.push_back(op.flops);
    cudaEvent_t a, b;
    TTC_CUDA(cudaEventCreate(&a));
    TTC_CUDA(cudaEventCreate(&b));
    ev.push_back(a);
    ev.push_back(b);
    kinds.push_back(op_kind(op.kind));
  }
  size_t i = 0;
  for (const Op& op : p.ops) {
    if (op.kind == OP_STAGE) {
      TTC_CUDA(cudaEventRecord(c->ev[op.a], c->stream));
      continue;
    }
    TTC_CUDA(cudaEventRecord(ev[2 * i], c->stream));
    launch_op(c, p, op);
    TTC_CUDA(cudaEventRecord(ev[2 * i + 1], c->stream));
    ++i;
  }
  TTC_CUDA(cudaStreamSynchronize(c->stream));
  // FLOPs at the sizes the launches ran with (device bounds read back once per address)
  std::unordered_map<const int*, int> bound_cache;
  auto val = [&](const int* ptr) {
    auto it = bound_cache.find(ptr);
    if (it != bound_cache.end()) return it->second;
    int v = 0;
    TTC_CUDA(cudaMemcpy(&v, ptr, sizeof(int), cudaMemcpyDeviceToHost));
    bound_cache[ptr] = v;
    return v;
  };
  {
    size_t j = 0;
    for (const Op& op : p.ops)
      if (op.kind != OP_STAGE) flops[j++] = bounded_flops(p, op, val);
  }
  for (int k = 0; k < 8; ++k) { c->stats.kind_ms[k] = 0; c->stats.kind_launches[k] = 0; c->stats.kind_flops[k] = 0; }
  // TTC_PROFILE_TRACE=<file>: one line per launch appended (op kind, problems, the kernel-specific
  // size arguments a, b and total, device ms, algorithmic FLOPs)
  FILE* trace = getenv("TTC_PROFILE_TRACE") ? fopen(getenv("TTC_PROFILE_TRACE"), "a") : nullptr;
  size_t j = 0;
  for (const Op& op : p.ops) {
    if (op.kind == OP_STAGE) continue;
    float ms = 0;
    TTC_CUDA(cudaEventElapsedTime(&ms, ev[2 * j], ev[2 * j + 1]));
    c->stats.kind_ms[kinds[j]] += ms;
    c->stats.kind_launches[kinds[j]] += 1;
    c->stats.kind_flops[kinds[j]] += flops[j];
    if (trace) fprintf(trace, "%d %d %d %d %lld %.4f %.4g\n", (int)op.kind, op.count, op.a, op.b, op.total, ms, flops[j]);
    ++j;
  }
  if (trace) fclose(trace);
  for (auto e : ev) cudaEventDestroy(e);
  // Jacobi sweep counters written into the plan blob
  c->stats.jacobi_problems = 0; c->stats.jacobi_sweeps_sum = 0; c->stats.jacobi_sweeps_max = 0;
  for (const auto& dg : p.diag) {
    std::vector<int> v((size_t)dg.second);
    TTC_CUDA(cudaMemcpy(v.data(), p.d_blob + dg.first, v.size() * sizeof(int), cudaMemcpyDeviceToHost));
    for (int x : v) {
      if (x == 0) continue;   // problem not run (empty)
      const int sw = x < 0 ? -x : x;
      c->stats.jacobi_problems += 1;
      c->stats.jacobi_sweeps_sum += sw;
      c->stats.jacobi_sweeps_max = std::max<int64_t>(c->stats.jacobi_sweeps_max, sw);
    }
  }
}

void run_plan(ttc_context* c, Plan& p) {
  c->stats.kernel_launches = count_launches(p);
  c->last_run_graph = false;
  TTC_CUDA(cudaEventRecord(c->ev[kEvRunBegin], c->stream));
  if (c->profiling) {
    run_plan_profiled(c, p);
    TTC_CUDA(cudaEventRecord(c->ev[kEvRunEnd], c->stream));
    return;
  }
  if (p.gexec && p.graph_stream == c->stream) {
    TTC_CUDA(cudaGraphLaunch(p.gexec, c->stream));
    c->last_run_graph = true;
    TTC_CUDA(cudaEventRecord(c->ev[kEvRunEnd], c->stream));
    return;
  }
  if (c->use_graphs && p.launches > 0) {
    // second and later runs: capture once, then replay the graph
    cudaGraph_t g = nullptr;
    TTC_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    try {
      launch_ops(c, p, false);
    } catch (...) {
      cudaStreamEndCapture(c->stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    TTC_CUDA(cudaStreamEndCapture(c->stream, &g));
    cudaGraphExec_t ge = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    TTC_CUDA(e);
    if (p.gexec) cudaGraphExecDestroy(p.gexec);
    p.gexec = ge;
    p.graph_stream = c->stream;
    TTC_CUDA(cudaGraphLaunch(p.gexec, c->stream));
    c->last_run_graph = true;
    TTC_CUDA(cudaEventRecord(c->ev[kEvRunEnd], c->stream));
    return;
  }
  launch_ops(c, p, true);
  p.launches++;
  TTC_CUDA(cudaEventRecord(c->ev[kEvRunEnd], c->stream));
}

// ---------------------------------------------------------------- builder
namespace {
inline void chk(bool on, const void* p, long long elems, size_t esz, const char* what) {
  if (on && elems > 0) region_check(p, (size_t)elems * esz, what);
}
inline long long sp2(long long e0, long long s0, long long e1, long long s1) {
  const long long e[2] = {e0, e1}, s[2] = {s0, s1};
  return span_elems(e, s, 2);
}
void check_gemm(const GemmDesc& d, size_t esz = 8) {
  const long long mi0 = std::min(d.m, d.m0), mi1 = (d.m - 1) / d.m0 + 1;
  const long long ni0 = std::min(d.n, d.n0), ni1 = (d.n - 1) / d.n0 + 1;
  const long long ki0 = std::min(d.k, d.k0e), ki1 = (d.k - 1) / d.k0e + 1;
  if (d.k > 0) {
    const long long ea[5] = {mi0, mi1, ki0, ki1, d.batch}, sa[5] = {d.a_i0, d.a_i1, d.a_k0, d.a_k1, d.a_b};
    region_check(d.A, esz * (size_t)span_elems(ea, sa, 5), "gemm A");
    const long long eb[5] = {ki0, ki1, ni0, ni1, d.batch}, sb[5] = {d.b_k0, d.b_k1, d.b_j0, d.b_j1, d.b_b};
    region_check(d.B, esz * (size_t)span_elems(eb, sb, 5), "gemm B");
  }
  const long long ec[5] = {mi0, mi1, ni0, ni1, d.batch}, sc[5] = {d.c_i0, d.c_i1, d.c_j0, d.c_j1, d.c_b};
  region_check(d.C, esz * (size_t)span_elems(ec, sc, 5), "gemm C");
  if (d.n_dev) region_check(d.n_dev, sizeof(int), "gemm n_dev");
}
}  // namespace

double* Builder::wd(size_t n) {
  const size_t o = (wsoff + 255) & ~size_t(255);
  wsoff = o + std::max<size_t>(n, 1) * sizeof(double);
  wshw = std::max(wshw, wsoff);
  return reinterpret_cast<double*>(wsbase + o);
}
int* Builder::wi(size_t n) {
  const size_t o = (wsoff + 255) & ~size_t(255);
  wsoff = o + std::max<size_t>(n, 1) * sizeof(int);
  wshw = std::max(wshw, wsoff);
  return reinterpret_cast<int*>(wsbase + o);
}
int* Builder::diag_ints(int n) {
  const size_t o = plan->push(std::vector<int>((size_t)std::max(n, 1), 0));
  plan->diag.push_back({o, std::max(n, 1)});
  return reinterpret_cast<int*>(blob_base + o);
}
void Builder::stage(int id) {
  Op op; op.kind = OP_STAGE; op.a = id;
  plan->ops.push_back(op);
}
const int* Builder::const_ints(const std::vector<int>& v) {
  const size_t o = plan->push(v);
  return reinterpret_cast<const int*>(blob_base + o);
}
void Builder::gemm(std::vector<GemmDesc> v) {
  std::vector<GemmDesc> w;
  long long out_tiles = 0;
  for (auto& d : v) {
    d.ksplit = 1; d.ws = nullptr; d.cnt = nullptr;
    out_tiles += gemm_tiles(d);
  }
  const int nsm = current_sm_count();
  long long t = 0;
  for (auto& d : v) {
    if (gemm_tiles(d) == 0) continue;
    if (d.m0 <= 0) d.m0 = std::max(d.m, 1);
    if (d.n0 <= 0) d.n0 = std::max(d.n, 1);
    if (d.k0e <= 0) d.k0e = std::max(d.k, 1);
    if (wsbase) check_gemm(d);
    const long long tiles_out = gemm_tiles(d);
    d.ksplit = gemm_pick_ksplit(d, out_tiles, nsm);
    if (d.ksplit > 1) {
      d.ws = wd((size_t)gemm_split_ws_doubles(d));
      // one counter per output tile, zero in the plan blob; the kernel leaves them zero
      const size_t o = plan->push(std::vector<unsigned>((size_t)tiles_out, 0u));
      d.cnt = reinterpret_cast<unsigned*>(blob_base + o);
      if (wsbase) {
        region_check(d.ws, sizeof(double) * (size_t)gemm_split_ws_doubles(d), "gemm split-K partials");
        region_check(d.cnt, sizeof(unsigned) * (size_t)tiles_out, "gemm split-K counters");
      }
    }
    d.tile_start = t;
    t += gemm_tiles(d);
    w.push_back(d);
  }
  if (w.empty()) return;
  Op op; op.kind = OP_GEMM; op.off = plan->push(w); op.count = (int)w.size(); op.total = t;
  for (auto& d : w) op.flops += 2.0 * d.m * d.n * d.k * std::max(1, d.batch);
  plan->ops.push_back(op);
}
void Builder::gemm32(std::vector<GemmDesc> v) {
  std::vector<GemmDesc> w;
  long long t = 0;
  for (auto& d : v) {
    const long long n = gemm_tiles(d);
    if (n == 0) continue;
    if (d.m0 <= 0) d.m0 = std::max(d.m, 1);
    if (d.n0 <= 0) d.n0 = std::max(d.n, 1);
    if (d.k0e <= 0) d.k0e = std::max(d.k, 1);
    if (wsbase) check_gemm(d, 4);
    d.tile_start = t;
    t += n;
    w.push_back(d);
  }
  if (w.empty()) return;
  Op op; op.kind = OP_GEMM32; op.off = plan->push(w); op.count = (int)w.size(); op.total = t;
  for (auto& d : w) op.flops += 2.0 * d.m * d.n * d.k * std::max(1, d.batch);
  plan->ops.push_back(op);
}
void Builder::cvt_f32(const std::vector<CvtDesc>& v) {
  if (v.empty()) return;
  long long mx = 0;
  for (auto& d : v) {
    mx = std::max(mx, d.rows * d.cols);
    if (wsbase) {
      region_check(d.src, 8 * (size_t)sp2(d.rows, d.ss_i, d.cols, d.ss_j), "cvt32 src");
      region_check(d.dst, 4 * (size_t)sp2(d.rows, d.ds_i, d.cols, d.ds_j), "cvt32 dst");
    }
  }
  Op op; op.kind = OP_CVT32; op.off = plan->push(v); op.count = (int)v.size(); op.total = mx;
  plan->ops.push_back(op);
}
void Builder::widen(const std::vector<CvtDesc>& v) {
  if (v.empty()) return;
  long long mx = 0;
  for (auto& d : v) {
    mx = std::max(mx, d.rows * d.cols);
    if (wsbase) {
      region_check(d.src, 4 * (size_t)sp2(d.rows, d.ss_i, d.cols, d.ss_j), "widen src");
      region_check(d.dst, 8 * (size_t)sp2(d.rows, d.ds_i, d.cols, d.ds_j), "widen dst");
    }
  }
  Op op; op.kind = OP_WIDEN; op.off = plan->push(v); op.count = (int)v.size(); op.total = mx;
  plan->ops.push_back(op);
}
void Builder::qr(const std::vector<QRDesc>& v) {
  if (v.empty()) return;
  int mm = 0, nn = 0;
  for (auto& d : v) {
    mm = std::max(mm, d.m);
    nn = std::max(nn, d.n);
    const int K = std::min(d.m, d.n);
    const bool on = wsbase != nullptr;
    chk(on, d.A, (long long)d.lda * (d.n - 1) + d.m, 8, "qr A");
    if (d.Q) chk(on, d.Q, (long long)d.ldq * (K - 1) + d.m, 8, "qr Q");
    if (d.R) chk(on, d.R, d.r_trans ? (long long)d.ldr * (K - 1) + d.n : (long long)d.ldr * (d.n - 1) + K, 8, "qr R");
    if (d.Rt) chk(on, d.Rt, (long long)d.ldrt * (K - 1) + d.n, 8, "qr R^T");
    TTC_REQUIRE(!d.Rt || (d.R && d.ldrt >= d.n), TTC_EINTERNAL, "qr: the transposed copy of R needs R");
    if (d.Tws) chk(on, d.Tws, (long long)((K + 15) / 16) * 256, 8, "qr Tws");
    TTC_REQUIRE(d.m <= QR_MAX_M, TTC_EDIM, "qr: row count exceeds the supported maximum (1536)");
    TTC_REQUIRE(!d.Q || d.Tws, TTC_EINTERNAL, "qr: forming Q needs the block-reflector workspace");
    TTC_REQUIRE(d.lda >= d.m && (!d.Q || d.ldq >= d.m) && (!d.R || d.ldr >= (d.r_trans ? d.n : K)), TTC_EINTERNAL,
                "qr: leading dims");
  }
  // largest problems first (the hardware starts clusters in index order): a launch whose
  // clusters outnumber the resident slots runs the long problems in the first wave
  std::vector<QRDesc> w(v);
  std::stable_sort(w.begin(), w.end(), [](const QRDesc& a, const QRDesc& b) {
    return qr_flops(a.m, a.n, a.Q != nullptr) > qr_flops(b.m, b.n, b.Q != nullptr);
  });
  Op op; op.kind = OP_QR; op.off = plan->push(w); op.count = (int)w.size(); op.a = mm; op.b = nn;
  for (auto& d : w) op.flops += qr_flops(d.m, d.n, d.Q != nullptr);
  plan->ops.push_back(op);
}
void Builder::qapply(const std::vector<QApplyDesc>& v) {
  if (v.empty()) return;
  int mm = 0;
  for (auto& d : v) {
    mm = std::max(mm, d.m);
    const bool on = wsbase != nullptr;
    chk(on, d.A, (long long)d.lda * (d.K - 1) + d.m, 8, "qr apply A");
    chk(on, d.Tws, (long long)((d.K + 15) / 16) * 256, 8, "qr apply Tws");
    chk(on, d.B, (long long)d.ldb * (d.nb - 1) + d.m, 8, "qr apply B");
    if (d.n_dev) chk(on, d.n_dev, 1, 4, "qr apply n_dev");
    TTC_REQUIRE(d.lda >= d.m && d.ldb >= d.m && d.K <= d.m, TTC_EINTERNAL, "qr apply: leading dims");
  }
  Op op; op.kind = OP_QAPPLY; op.off = plan->push(v); op.count = (int)v.size(); op.a = mm;
  for (auto& d : v) op.flops += qapply_flops(d.m, d.K, d.nb);
  plan->ops.push_back(op);
}
void Builder::jacobi(const std::vector<JacobiDesc>& v) {
  if (v.empty()) return;
  int mm = 0, nn = 0;
  for (auto& d : v) {
    mm = std::max(mm, d.m); nn = std::max(nn, d.n);
    const bool on = wsbase != nullptr;
    chk(on, d.X, (long long)d.ldx * (d.n - 1) + d.m, 8, "jacobi X");
    if (d.W) chk(on, d.W, (long long)d.ldw * (d.n - 1) + d.n, 8, "jacobi W");
    chk(on, d.sigma, d.n, 8, "jacobi sigma");
    chk(on, d.perm, d.n, 4, "jacobi perm");
    if (d.info) chk(on, d.info, 1, 4, "jacobi info");
    TTC_REQUIRE(d.ldx >= d.m && (!d.W || d.ldw >= d.n), TTC_EINTERNAL, "jacobi: leading dims");
    TTC_REQUIRE(2LL * 1 * (d.m + (d.W ? d.n : 0)) <= 25600 && d.n <= 25600, TTC_EDIM, "jacobi: matrix too large");
  }
  Op op; op.kind = OP_JACOBI; op.off = plan->push(v); op.count = (int)v.size(); op.a = mm; op.b = nn;
  op.rmax = ctx->jacobi_max_sweeps;              // the sweep cap (plans are rebuilt when it changes)
  op.iw = (int)v.size() <= kJacobiOrderMax ? wi(v.size()) : nullptr;   // largest problems first
  for (auto& d : v) op.total |= (d.W != nullptr);
  for (auto& d : v) op.flops += jacobi_flops(d.m, d.n);
  plan->ops.push_back(op);
}
void Builder::trunc(const std::vector<TruncDesc>& v, double tol, long long rmax) {
  if (v.empty()) return;
  for (auto& d : v) {
    const bool on = wsbase != nullptr;
    chk(on, d.sigma, d.n, 8, "trunc sigma");
    chk(on, d.perm, d.n, 4, "trunc perm");
    chk(on, d.rank_out, 1, 4, "trunc rank");
  }
  Op op; op.kind = OP_TRUNC; op.off = plan->push(v); op.count = (int)v.size(); op.tol = tol; op.rmax = rmax;
  plan->ops.push_back(op);
}
void Builder::select(const std::vector<SelectDesc>& v) {
  if (v.empty()) return;
  int mr = 0, mc = 0;
  for (auto& d : v) {
    const int rows = std::max(d.rows, d.zrows);
    mr = std::max(mr, rows); mc = std::max(mc, d.cols);
    const bool on = wsbase != nullptr;
    chk(on, d.X, (long long)d.ldx * (d.src_cols - 1) + d.rows, 8, "select X");
    chk(on, d.sigma, d.src_cols, 8, "select sigma");
    chk(on, d.perm, d.src_cols, 4, "select perm");
    chk(on, d.rank, 1, 4, "select rank");
    chk(on, d.U, (long long)d.ldu * (d.cols - 1) + rows, 8, "select U");
    TTC_REQUIRE(d.ldx >= d.rows && d.ldu >= rows, TTC_EINTERNAL, "select: leading dims");
  }
  Op op; op.kind = OP_SELECT; op.off = plan->push(v); op.count = (int)v.size(); op.a = mr; op.b = mc;
  plan->ops.push_back(op);
}
void Builder::copy(const std::vector<CopyDesc>& v) {
  std::vector<CopyDesc> w;
  long long mx = 0;
  for (auto& d : v) {
    const long long n = d.ext[0] * d.ext[1] * d.ext[2] * d.ext[3];
    if (n <= 0) continue;
    if (wsbase) {
      region_check(d.src, 8 * (size_t)span_elems(d.ext, d.ss, 4), "copy src");
      region_check(d.dst, 8 * (size_t)span_elems(d.ext, d.ds, 4), "copy dst");
    }
    mx = std::max(mx, n);
    w.push_back(d);
  }
  if (w.empty()) return;
  Op op; op.kind = OP_COPY; op.off = plan->push(w); op.count = (int)w.size(); op.total = mx;
  plan->ops.push_back(op);
}
void Builder::zero(const std::vector<ZeroDesc>& v) {
  std::vector<ZeroDesc> w;
  long long mx = 0;
  for (auto& d : v) if (d.n > 0) {
    chk(wsbase != nullptr, d.p, d.n, 8, "zero");
    w.push_back(d); mx = std::max(mx, d.n);
  }
  if (w.empty()) return;
  Op op; op.kind = OP_ZERO; op.off = plan->push(w); op.count = (int)w.size(); op.total = mx;
  plan->ops.push_back(op);
}
void Builder::sumsq(const std::vector<NormDesc>& v) {
  if (v.empty()) return;
  for (auto& d : v) { chk(wsbase != nullptr, d.p, d.n, 8, "sumsq src"); chk(wsbase != nullptr, d.out, 1, 8, "sumsq out"); }
  Op op; op.kind = OP_SUMSQ; op.off = plan->push(v); op.count = (int)v.size();
  plan->ops.push_back(op);
}
void Builder::apply(const std::vector<ApplyDesc>& v) {
  if (v.empty()) return;
  long long mx = 0;
  int max_rn = 0;
  long long max_sm = 0;
  for (auto& d : v) {
    mx = std::max(mx, (long long)d.R * d.r * d.n * d.Rn * d.rn);
    max_rn = std::max(max_rn, d.rn);
    max_sm = std::max<long long>(max_sm, apply_smem_doubles(d));
    const bool on = wsbase != nullptr;
    chk(on, d.H, (long long)d.R * d.n * d.n * d.Rn, 8, "apply H");
    chk(on, d.V, (long long)d.r * d.n * d.rn, 8, "apply V");
    chk(on, d.Y, (long long)d.R * d.r * d.n * d.Rn * d.rn, 8, "apply Y");
  }
  Op op; op.kind = OP_APPLY; op.off = plan->push(v); op.count = (int)v.size(); op.total = mx;
  TTC_REQUIRE(max_sm <= 25600, TTC_EDIM, "apply: operator and vector ranks too large for the staged slices");
  op.a = max_rn; op.b = (int)max_sm;
  plan->ops.push_back(op);
}
void Builder::philox(const std::vector<PhiloxDesc>& v) {
  if (v.empty()) return;
  long long mx = 0;
  for (auto& d : v) { mx = std::max(mx, d.count); chk(wsbase != nullptr, d.dst, d.count, 8, "philox dst"); }
  Op op; op.kind = OP_PHILOX; op.off = plan->push(v); op.count = (int)v.size(); op.total = mx;
  plan->ops.push_back(op);
}
void Builder::bf16gemm(std::vector<Bf16GemmDesc> v, bool tf32) {
  std::vector<Bf16GemmDesc> w;
  long long t = 0;
  const long long esz = tf32 ? 4 : 2, chunk = 16 / esz;   // operand bytes, elements per 16 bytes
  for (auto& d : v) {
    const long long n = bf16_gemm_tiles(d);
    if (n == 0) continue;
    if (wsbase) {
      TTC_REQUIRE(d.lda % chunk == 0 && d.ldb % chunk == 0 && d.lda >= d.k && d.ldb >= d.k && d.m0 >= 1,
                  TTC_EINTERNAL, "tensor-core gemm: leading dims must be multiples of 16 bytes covering K");
      TTC_REQUIRE(((uintptr_t)d.A % 16) == 0 && ((uintptr_t)d.B % 16) == 0, TTC_EINTERNAL, "bf16 gemm: 16-byte alignment");
      const long long kp = (d.k + chunk - 1) / chunk * chunk;
      region_check(d.A, esz * (size_t)(d.lda * (d.m - 1) + kp), "bf16 A");
      region_check(d.B, esz * (size_t)(d.ldb * (d.n - 1) + kp), "bf16 B");
      const long long mi0 = std::min(d.m, d.m0), mi1 = (d.m - 1) / d.m0 + 1;
      TTC_REQUIRE(d.n0 >= 0, TTC_EINTERNAL, "bf16 gemm: negative column split");
      const long long nj0 = d.n0 > 0 ? std::min(d.n, d.n0) : d.n, nj1 = d.n0 > 0 ? (d.n - 1) / d.n0 + 1 : 1;
      if (d.C64 || d.C32) {
        const long long e[4] = {mi0, mi1, nj0, nj1}, s[4] = {d.c_i0, d.c_i1, d.c_j, d.c_j1};
        if (d.C64) region_check(d.C64, 8 * (size_t)span_elems(e, s, 4), "bf16 C64");
        if (d.C32) region_check(d.C32, 4 * (size_t)span_elems(e, s, 4), "bf16 C32");
      }
      if (d.C16) {
        const long long e[4] = {mi0, mi1, nj0, nj1}, s[4] = {d.h_i0, d.h_i1, d.h_j, d.h_j1};
        region_check(d.C16, esz * (size_t)span_elems(e, s, 4), "bf16 C16");
      }
    }
    d.tile_start = t;
    t += n;
    w.push_back(d);
  }
  if (w.empty()) return;
  Op op; op.kind = OP_BF16GEMM; op.off = plan->push(w); op.count = (int)w.size(); op.total = t; op.a = tf32;
  for (auto& d : w) op.flops += 2.0 * d.m * d.n * d.k;
  plan->ops.push_back(op);
}
void Builder::cvt_bf16(const std::vector<CvtDesc>& v, bool f32) {
  if (v.empty()) return;
  long long mx = 0;
  for (auto& d : v) {
    mx = std::max(mx, d.rows * d.cols);
    if (wsbase) {
      region_check(d.src, 8 * (size_t)sp2(d.rows, d.ss_i, d.cols, d.ss_j), "cvt src");
      region_check(d.dst, (f32 ? 4 : 2) * (size_t)sp2(d.rows, d.ds_i, d.cols, d.ds_j), "cvt dst");
    }
  }
  Op op; op.kind = OP_CVT_BF16; op.off = plan->push(v); op.count = (int)v.size(); op.total = mx; op.a = f32;
  plan->ops.push_back(op);
}
void Builder::pinv_scale(const std::vector<PinvScaleDesc>& v) {
  if (v.empty()) return;
  for (auto& d : v) {
    chk(wsbase != nullptr, d.X, (long long)d.ldx * std::max(d.n - 1, 0) + d.m, 8, "pinv_scale X");
    chk(wsbase != nullptr, d.sigma, d.n, 8, "pinv_scale sigma");
  }
  Op op; op.kind = OP_PINV_SCALE; op.off = plan->push(v); op.count = (int)v.size();
  plan->ops.push_back(op);
}
void Builder::zerochk(const std::vector<ZeroChkDesc>& v) {
  if (v.empty()) return;
  for (auto& d : v) { chk(wsbase != nullptr, d.sumsq, 1, 8, "zerochk"); chk(wsbase != nullptr, d.flag, 1, 4, "zerochk flag"); }
  Op op; op.kind = OP_ZEROCHK; op.off = plan->push(v); op.count = (int)v.size();
  plan->ops.push_back(op);
}
void Builder::finalize(const std::vector<FinalDesc>& v) {
  if (v.empty()) return;
  long long mx = 0;
  for (auto& d : v) {
    mx = std::max(mx, d.n);
    const bool on = wsbase != nullptr;
    chk(on, d.cores, d.n, 8, "final cores");
    chk(on, d.rks, d.nrks, 4, "final rks");
    chk(on, d.rks_restore, d.nrks, 4, "final rks src");
    chk(on, d.flag, 1, 4, "final flag");
  }
  Op op; op.kind = OP_FINAL; op.off = plan->push(v); op.count = (int)v.size(); op.total = mx;
  plan->ops.push_back(op);
}
void Builder::setrank(const std::vector<SetRankDesc>& v) {
  if (v.empty()) return;
  for (auto& d : v) { chk(wsbase != nullptr, d.dst, d.n, 4, "setrank dst"); chk(wsbase != nullptr, d.src, d.n, 4, "setrank src"); }
  Op op; op.kind = OP_SETRANK; op.off = plan->push(v); op.count = (int)v.size();
  plan->ops.push_back(op);
}

GemmDesc gd(int m, int n, int k, const double* A, long long a_i, long long a_k, const double* B, long long b_k,
            long long b_j, double* C, long long c_i, long long c_j, double alpha, double beta) {
  GemmDesc d{};
  d.m = m; d.n = n; d.k = k; d.batch = 1;
  d.m0 = std::max(m, 1); d.n0 = std::max(n, 1); d.k0e = std::max(k, 1);
  d.A = A; d.a_i0 = a_i; d.a_k0 = a_k;
  d.B = B; d.b_k0 = b_k; d.b_j0 = b_j;
  d.C = C; d.c_i0 = c_i; d.c_j0 = c_j;
  d.alpha = alpha; d.beta = beta;
  return d;
}

CopyDesc cd2(const double* src, double* dst, long long e0, long long e1, long long s0, long long s1, long long d0,
             long long d1, double alpha) {
  CopyDesc c{};
  c.src = src; c.dst = dst;
  c.ext[0] = e0; c.ext[1] = e1; c.ext[2] = 1; c.ext[3] = 1;
  c.ss[0] = s0; c.ss[1] = s1; c.ds[0] = d0; c.ds[1] = d1;
  c.alpha = alpha;
  return c;
}

CopyDesc cd3(const double* src, double* dst, long long e0, long long e1, long long e2, long long s0, long long s1,
             long long s2, long long d0, long long d1, long long d2, double alpha) {
  CopyDesc c = cd2(src, dst, e0, e1, s0, s1, d0, d1, alpha);
  c.ext[2] = e2; c.ss[2] = s2; c.ds[2] = d2;
  return c;
}

// Two passes: measure (workspace and blob sizes), allocate, then build for real.
Plan* get_plan(ttc_context* c, const std::string& key, const std::function<void(Builder&)>& fn) {
  auto it = c->plans.find(key);
  if (it != c->plans.end() && it->second->ws_base == (void*)c->ws) return it->second.get();
  std::unique_ptr<Plan> meas(new Plan());
  {
    Builder b;
    b.ctx = c; b.plan = meas.get(); b.wsbase = nullptr; b.blob_base = nullptr;
    fn(b);
    meas->ws_needed = b.wshw;
  }
  ensure_workspace(c, meas->ws_needed);
  std::unique_ptr<Plan> p(new Plan());
  const size_t blob_cap = meas->blob.size() + 256;
  TTC_CUDA(cudaMalloc(&p->d_blob, blob_cap));
  region_add(p->d_blob, blob_cap);
  p->d_blob_cap = blob_cap;
  {
    Builder b;
    b.ctx = c; b.plan = p.get(); b.wsbase = c->ws; b.blob_base = p->d_blob;
    fn(b);
    p->ws_needed = b.wshw;
  }
  TTC_REQUIRE(p->blob.size() <= blob_cap, TTC_EINTERNAL, "plan blob grew between passes");
  TTC_CUDA(cudaMemcpy(p->d_blob, p->blob.data(), p->blob.size(), cudaMemcpyHostToDevice));
  p->ws_base = c->ws;
  Plan* raw = p.get();
  c->stats.plans_built += 1;
  if (c->plans.size() > 64) c->plans.clear();
  c->plans[key] = std::move(p);
  return raw;
}

void ensure_workspace(ttc_context* c, size_t bytes) {
  if (bytes <= c->ws_bytes) return;
  TTC_CUDA(cudaStreamSynchronize(c->stream));
  if (c->ws) { region_remove(c->ws); TTC_CUDA(cudaFree(c->ws)); }
  c->ws = nullptr;
  c->ws_bytes = 0;
  const size_t nb = bytes + bytes / 4 + (1 << 20);
  if (cudaMalloc(&c->ws, nb) != cudaSuccess) {
    cudaGetLastError();
    throw Error(TTC_ENOMEM, "workspace allocation of " + std::to_string(nb) + " bytes failed");
  }
  c->ws_bytes = nb;
  region_add(c->ws, nb);
  c->plans.clear();   // descriptors point into the old workspace
}

int current_sm_count() {
  static std::mutex mu;
  static int count[kMaxDevices] = {};
  int dev = 0;
  TTC_CUDA(cudaGetDevice(&dev));
  TTC_REQUIRE(dev >= 0 && dev < kMaxDevices, TTC_EARG, "device index out of range");
  std::lock_guard<std::mutex> lk(mu);
  if (count[dev] == 0) TTC_CUDA(cudaDeviceGetAttribute(&count[dev], cudaDevAttrMultiProcessorCount, dev));
  return count[dev];
}

void check_device_flags(ttc_context* c) {
  int f = 0;
  TTC_CUDA(cudaMemcpyAsync(&f, c->d_flags, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  TTC_CUDA(cudaStreamSynchronize(c->stream));
  if (f) {
    TTC_CUDA(cudaMemsetAsync(c->d_flags, 0, sizeof(int), c->stream));
    if (f & DFLAG_NONFINITE) throw Error(TTC_ENONFINITE, "NaN or Inf met in a factorisation input");
    if (f & DFLAG_JACOBI_NOCONV) throw Error(TTC_ENOCONV, "one-sided Jacobi SVD did not converge within the sweep cap");
    if (f & DFLAG_BAD_DESC) throw Error(TTC_EINTERNAL, "a kernel skipped an inconsistent descriptor");
    if (f & DFLAG_TIMEOUT) throw Error(TTC_EINTERNAL, "a bounded device wait gave up (tensor-core pipeline stalled)");
  }
}

// ---------------------------------------------------------------- batches
ttc_batch* batch_create(ttc_context* c, int count, int N, const long long* dims, const int* cap) {
  TTC_REQUIRE(count > 0 && N > 0, TTC_EARG, "batch: count and N must be positive");
  std::unique_ptr<ttc_batch> b(new ttc_batch());
  b->ctx = c; b->count = count; b->N = N;
  b->dims.assign(dims, dims + N);
  for (int k = 0; k < N; ++k) TTC_REQUIRE(dims[k] > 0, TTC_EARG, "batch: dims must be positive");
  b->cap.assign(cap, cap + (size_t)count * (N + 1));
  b->off.resize((size_t)count * N);
  b->tt_off.resize(count + 1);
  long long o = 0;
  for (int t = 0; t < count; ++t) {
    b->tt_off[t] = o;
    TTC_REQUIRE(b->capr(t, 0) >= 1 && b->capr(t, N) >= 1, TTC_EARG, "batch: boundary capacities must be >= 1");
    for (int k = 0; k < N; ++k) {
      TTC_REQUIRE(b->capr(t, k) >= 1, TTC_EARG, "batch: capacities must be >= 1");
      b->off[(size_t)t * N + k] = o;
      o += (long long)b->capr(t, k) * dims[k] * b->capr(t, k + 1);
      o = (o + 31) & ~31LL;    // 256-byte aligned cores
    }
  }
  b->tt_off[count] = o;
  b->total = o;
  if (cudaMalloc(&b->d_cores, sizeof(double) * std::max<long long>(o, 1)) != cudaSuccess) {
    cudaGetLastError();
    throw Error(TTC_ENOMEM, "batch allocation failed");
  }
  TTC_CUDA(cudaMalloc(&b->d_rks, sizeof(int) * (size_t)count * (N + 1)));
  TTC_CUDA(cudaMalloc(&b->d_zero, sizeof(int) * count));
  region_add(b->d_cores, sizeof(double) * std::max<long long>(o, 1));
  region_add(b->d_rks, sizeof(int) * (size_t)count * (N + 1));
  region_add(b->d_zero, sizeof(int) * count);
  TTC_CUDA(cudaMemsetAsync(b->d_cores, 0, sizeof(double) * std::max<long long>(o, 1), c->stream));
  TTC_CUDA(cudaMemsetAsync(b->d_zero, 0, sizeof(int) * count, c->stream));
  b->h_rks.assign((size_t)count * (N + 1), 1);
  b->h_ot.assign((size_t)count * N, 0);
  TTC_CUDA(cudaMemcpyAsync(b->d_rks, b->h_rks.data(), sizeof(int) * b->h_rks.size(), cudaMemcpyHostToDevice, c->stream));
  TTC_CUDA(cudaStreamSynchronize(c->stream));
  return b.release();
}

void batch_sync_ranks(ttc_batch* b) {
  if (!b->rks_dirty) return;
  ttc_context* c = b->ctx;
  TTC_CUDA(cudaMemcpyAsync(b->h_rks.data(), b->d_rks, sizeof(int) * b->h_rks.size(), cudaMemcpyDeviceToHost, c->stream));
  std::vector<int> z(b->count);
  TTC_CUDA(cudaMemcpyAsync(z.data(), b->d_zero, sizeof(int) * b->count, cudaMemcpyDeviceToHost, c->stream));
  TTC_CUDA(cudaStreamSynchronize(c->stream));
  for (int t = 0; t < b->count; ++t)
    if (z[t])
      for (int k = 0; k < b->N; ++k) b->h_ot[(size_t)t * b->N + k] = 0;
  b->rks_dirty = false;
  batch_rehash(b);   // plans that read the batch are keyed on its rank state, not on its history
}

void batch_destroy(ttc_batch* b) {
  if (!b) return;
  region_remove(b->d_cores); region_remove(b->d_rks); region_remove(b->d_zero);
  if (b->d_cores) cudaFree(b->d_cores);
  if (b->d_rks) cudaFree(b->d_rks);
  if (b->d_zero) cudaFree(b->d_zero);
  // plans keyed on this batch stay valid only while it lives
  ttc_context* c = b->ctx;
  const std::string tag = "@" + std::to_string((unsigned long long)(uintptr_t)b) + ":";
  for (auto it = c->plans.begin(); it != c->plans.end();) {
    if (it->first.find(tag) != std::string::npos) it = c->plans.erase(it); else ++it;
  }
  delete b;
}

std::string batch_key(const ttc_batch* b) {
  return "@" + std::to_string((unsigned long long)(uintptr_t)b) + ":" + std::to_string(b->version) + ";";
}

std::string batch_out_key(const ttc_batch* b) {
  return "@" + std::to_string((unsigned long long)(uintptr_t)b) + ":out;";
}

void batch_rehash(ttc_batch* b) {
  unsigned long long h = 1469598103934665603ull;   // FNV-1a over the host rank and ot state
  for (int v : b->h_rks) h = (h ^ (unsigned)v) * 1099511628211ull;
  for (int v : b->h_ot) h = (h ^ (unsigned)(v + 7)) * 1099511628211ull;
  b->version = h;
}

}  // namespace ttc
