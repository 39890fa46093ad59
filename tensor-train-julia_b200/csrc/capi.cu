// extern "C" boundary of libttcuda (declared in include/ttcuda.h).  Converts exceptions to
// status codes, moves host tensors in the reference's column-major layout to and from the
// internal device layout (one pinned staging copy per call, packed by several host threads;
// permutation on the device).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "api_impl.cuh"
#include "regions.cuh"

using namespace ttc;

namespace ttc {

static thread_local std::string g_err_noctx;
// Message of ttc_last_error(NULL) for entry points that take no context.
void set_noctx_error(const std::string& msg) { g_err_noctx = msg; }

template <class F>
int guard(ttc_context* c, F&& f) {
  try {
    if (c) TTC_CUDA(cudaSetDevice(c->device));
    f();
    return TTC_OK;
  } catch (const Error& e) {
    if (c) c->err = e.what(); else g_err_noctx = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    if (c) c->err = "host allocation failed"; else g_err_noctx = "host allocation failed";
    return TTC_ENOMEM;
  } catch (const std::exception& e) {
    if (c) c->err = e.what(); else g_err_noctx = e.what();
    return TTC_EINTERNAL;
  }
}

void ensure_stage(ttc_context* c, size_t bytes) {
  if (bytes <= c->stage_bytes) return;
  TTC_CUDA(cudaStreamSynchronize(c->stream));
  if (c->d_stage) { region_remove(c->d_stage); cudaFree(c->d_stage); }
  if (c->h_stage) cudaFreeHost(c->h_stage);
  c->d_stage = nullptr; c->h_stage = nullptr; c->stage_bytes = 0;
  const size_t nb = bytes + bytes / 4 + (1 << 16);
  if (cudaMalloc(&c->d_stage, nb) != cudaSuccess) { cudaGetLastError(); throw Error(TTC_ENOMEM, "staging allocation failed"); }
  if (cudaMallocHost(&c->h_stage, nb) != cudaSuccess) { cudaGetLastError(); throw Error(TTC_ENOMEM, "pinned staging allocation failed"); }
  c->stage_bytes = nb;
  region_add(c->d_stage, nb);
}

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Host copies of a transfer (dst, src, bytes), split over host threads: packing hundreds of MB
// into the pinned staging buffer is bound by host memory bandwidth, which one thread does not
// reach.  Small transfers stay on the calling thread.
struct HostCopy { void* dst; const void* src; size_t bytes; };
// Host staging is done in chunks of about this many bytes, each chunk's transfer overlapping
// the staging of the next.
constexpr size_t kStageChunk = 48u << 20;

static void parallel_memcpy(const std::vector<HostCopy>& cps) {
  size_t total = 0;
  for (const auto& c : cps) total += c.bytes;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned nt = (unsigned)std::min<size_t>(std::min(hw, 16u), total / (8u << 20) + 1);
  if (nt <= 1) {
    for (const auto& c : cps) std::memcpy(c.dst, c.src, c.bytes);
    return;
  }
  // split the byte range [0, total) evenly; a copy may be cut between two threads
  auto work = [&](size_t lo, size_t hi) {
    size_t base = 0;
    for (const auto& c : cps) {
      const size_t a = std::max(lo, base), e = std::min(hi, base + c.bytes);
      if (a < e) std::memcpy((char*)c.dst + (a - base), (const char*)c.src + (a - base), e - a);
      base += c.bytes;
      if (base >= hi) break;
    }
  };
  std::vector<std::thread> th;
  for (unsigned i = 1; i < nt; ++i) th.emplace_back(work, total * i / nt, total * (i + 1) / nt);
  work(0, total / nt);
  for (auto& t : th) t.join();
}

void validate_ttv(const ttc_ttv* x) {
  TTC_REQUIRE(x && x->N > 0 && x->dims && x->rks && x->cores, TTC_EARG, "TTvector: null field");
  for (int k = 0; k < x->N; ++k) {
    TTC_REQUIRE(x->dims[k] > 0, TTC_EARG, "TTvector: dims must be positive");
    TTC_REQUIRE(x->cores[k] != nullptr, TTC_EARG, "TTvector: null core");
  }
  TTC_REQUIRE(x->rks[0] == 1 && x->rks[x->N] == 1, TTC_EDIM, "TTvector: boundary ranks must be 1");
  for (int k = 0; k <= x->N; ++k) TTC_REQUIRE(x->rks[k] >= 1, TTC_EDIM, "TTvector: ranks must be >= 1");
}

// Device address of the host range [p, p + bytes) when all of it lies in page-locked host
// memory mapped into the device address space (cudaHostAlloc, cudaHostRegister), so that a
// kernel can read or write it directly over the host link; nullptr otherwise (pageable memory).
static const void* mapped_host_view(const void* p, size_t bytes) {
  if (!p || bytes == 0) return nullptr;
  cudaPointerAttributes a{}, e{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return nullptr; }
  if (a.type != cudaMemoryTypeHost || !a.devicePointer) return nullptr;
  const char* last = (const char*)p + bytes - 1;
  if (cudaPointerGetAttributes(&e, last) != cudaSuccess) { cudaGetLastError(); return nullptr; }
  if (e.type != cudaMemoryTypeHost || !e.devicePointer) return nullptr;
  if ((const char*)e.devicePointer - (const char*)a.devicePointer != (std::ptrdiff_t)(bytes - 1)) return nullptr;
  return a.devicePointer;
}

// Upload many TTs into consecutive slots [first, first+m) of a batch.  Cores in page-locked
// memory are copied by DMA straight into the device staging area, one copy per run of cores
// adjacent in host memory; pageable cores are first packed into the context's pinned buffer.
// A layout kernel then moves the staged cores into the batch slots.
void batch_upload_many(ttc_batch* b, int first, int m, const ttc_ttv* xs, bool reverse) {
  ttc_context* c = b->ctx;
  const int N = b->N;
  size_t data = 0;
  for (int i = 0; i < m; ++i) {
    const ttc_ttv& x = xs[i];
    validate_ttv(&x);
    TTC_REQUIRE(x.N == N, TTC_EDIM, "upload: N differs from the batch");
    for (int k = 0; k < N; ++k)
      TTC_REQUIRE(x.dims[reverse ? N - 1 - k : k] == b->dims[k], TTC_EDIM, "upload: dims differ from the batch");
    for (int k = 0; k <= N; ++k)
      TTC_REQUIRE(x.rks[reverse ? N - k : k] <= b->capr(first + i, k), TTC_EDIM, "upload: rank exceeds the batch capacity");
    for (int k = 0; k < N; ++k) data += (size_t)x.dims[k] * x.rks[k] * x.rks[k + 1];
  }
  bool direct = true;   // every core page-locked (validated above)
  for (int i = 0; i < m && direct; ++i)
    for (int k = 0; k < N && direct; ++k) {
      const size_t cnt = (size_t)xs[i].dims[k] * xs[i].rks[k] * xs[i].rks[k + 1];
      direct = mapped_host_view(xs[i].cores[k], cnt * sizeof(double)) != nullptr;
    }
  const size_t nd = (size_t)m * N;
  const size_t off_desc = align_up(data * sizeof(double), 256);
  const size_t off_rk = align_up(off_desc + nd * sizeof(CopyDesc), 256);
  const size_t total = off_rk + (size_t)m * (N + 1) * sizeof(int);
  ensure_stage(c, total);
  unsigned char* h = (unsigned char*)c->h_stage;
  unsigned char* d = (unsigned char*)c->d_stage;
  double* hd = (double*)h;
  CopyDesc* hc = (CopyDesc*)(h + off_desc);
  int* hr = (int*)(h + off_rk);
  size_t o = 0, ci = 0;
  long long maxe = 0;
  std::vector<HostCopy> hcp;
  for (int i = 0; i < m; ++i) {
    const ttc_ttv& x = xs[i];
    const int t = first + i;
    for (int k = 0; k < N; ++k) {
      const int kx = reverse ? N - 1 - k : k;     // host core feeding slot core k
      const long long n = x.dims[kx], r0 = x.rks[kx], r1 = x.rks[kx + 1], cap0 = b->capr(t, k);
      const size_t cnt = (size_t)n * r0 * r1;
      hcp.push_back({hd + o, x.cores[kx], cnt * sizeof(double)});
      // Julia (i, a, b) at i + n*(a + r0*b)  ->  internal (a, i, b) at a + cap0*(i + n*b);
      // reversed: internal (b, i, a) at b + cap0*(i + n*a)
      if (!reverse)
        hc[ci++] = cd3((const double*)(d) + o, b->core(t, k), n, r0, r1, 1, n, n * r0, cap0, 1, cap0 * n);
      else
        hc[ci++] = cd3((const double*)(d) + o, b->core(t, k), n, r0, r1, 1, n, n * r0, cap0, cap0 * n, 1);
      maxe = std::max<long long>(maxe, (long long)cnt);
      o += cnt;
    }
    for (int k = 0; k <= N; ++k) hr[(size_t)i * (N + 1) + k] = (int)x.rks[reverse ? N - k : k];
  }
  // zero the slots (padding must be 0); stage the cores chunk by chunk, each chunk's transfer
  // running while the next one is staged; then the descriptors and ranks
  TTC_CUDA(cudaMemsetAsync(b->core(first, 0), 0, sizeof(double) * (b->tt_off[first + m] - b->tt_off[first]), c->stream));
  size_t sent = 0;
  if (direct) {
    for (size_t gi = 0; gi < hcp.size();) {      // runs of cores adjacent in host memory
      size_t gj = gi + 1, bytes = hcp[gi].bytes;
      while (gj < hcp.size() && (const char*)hcp[gj].src == (const char*)hcp[gi].src + bytes) bytes += hcp[gj++].bytes;
      TTC_CUDA(cudaMemcpyAsync(d + sent, hcp[gi].src, bytes, cudaMemcpyHostToDevice, c->stream));
      sent += bytes;
      gi = gj;
    }
  } else {
    for (size_t gi = 0; gi < hcp.size();) {
      size_t gj = gi, bytes = 0;
      while (gj < hcp.size() && (gj == gi || bytes < kStageChunk)) bytes += hcp[gj++].bytes;
      parallel_memcpy(std::vector<HostCopy>(hcp.begin() + (long)gi, hcp.begin() + (long)gj));
      TTC_CUDA(cudaMemcpyAsync(d + sent, h + sent, bytes, cudaMemcpyHostToDevice, c->stream));
      sent += bytes;
      gi = gj;
    }
  }
  TTC_CUDA(cudaMemcpyAsync(d + off_desc, h + off_desc, total - off_desc, cudaMemcpyHostToDevice, c->stream));
  launch_copy((const CopyDesc*)(d + off_desc), (int)ci, maxe, c->stream);
  TTC_CUDA(cudaMemcpyAsync(b->drk(first, 0), d + off_rk, (size_t)m * (N + 1) * sizeof(int), cudaMemcpyDeviceToDevice,
                           c->stream));
  TTC_CUDA(cudaMemsetAsync(b->d_zero + first, 0, sizeof(int) * m, c->stream));
  TTC_CUDA(cudaStreamSynchronize(c->stream));   // the pinned staging is reused by the next call
  for (int i = 0; i < m; ++i) {
    const ttc_ttv& x = xs[i];
    const int t = first + i;
    for (int k = 0; k <= N; ++k) b->h_rks[(size_t)t * (N + 1) + k] = (int)x.rks[reverse ? N - k : k];
    for (int k = 0; k < N; ++k)
      b->h_ot[(size_t)t * N + k] = x.ot ? (reverse ? -(int)x.ot[N - 1 - k] : (int)x.ot[k]) : 0;
  }
  batch_rehash(b);
  b->rks_dirty = false;
}

void batch_download_many(ttc_batch* b, int first, int m, ttc_ttv_out* ys, bool reverse) {
  ttc_context* c = b->ctx;
  const int N = b->N;
  batch_sync_ranks(b);
  size_t data = 0;
  for (int i = 0; i < m; ++i) {
    const int t = first + i;
    TTC_REQUIRE(ys[i].N == N && ys[i].rks && ys[i].cores, TTC_EARG, "download: bad output descriptor");
    for (int k = 0; k <= N; ++k)
      if (ys[i].rks_cap)
        TTC_REQUIRE(b->rk(t, reverse ? N - k : k) <= ys[i].rks_cap[k], TTC_EDIM,
                    "download: output capacity smaller than the result rank");
    for (int k = 0; k < N; ++k) data += (size_t)b->dims[k] * b->rk(t, k) * b->rk(t, k + 1);
  }
  // output cores in mapped page-locked memory are written by the layout kernel itself
  std::vector<void*> views;
  bool direct = true;
  for (int i = 0; i < m && direct; ++i)
    for (int ko = 0; ko < N && direct; ++ko) {
      const int k = reverse ? N - 1 - ko : ko;
      const size_t cnt = (size_t)b->dims[k] * b->rk(first + i, k) * b->rk(first + i, k + 1);
      views.push_back(const_cast<void*>(mapped_host_view(ys[i].cores[ko], cnt * sizeof(double))));
      direct = views.back() != nullptr;
    }
  if (direct) data = 0;
  const size_t nd = (size_t)m * N;
  const size_t off_desc = align_up(data * sizeof(double), 256);
  const size_t total = off_desc + nd * sizeof(CopyDesc);
  ensure_stage(c, total);
  unsigned char* h = (unsigned char*)c->h_stage;
  unsigned char* d = (unsigned char*)c->d_stage;
  CopyDesc* hc = (CopyDesc*)(h + off_desc);
  size_t o = 0, ci = 0;
  long long maxe = 0;
  std::vector<size_t> offs;
  for (int i = 0; i < m; ++i) {
    const int t = first + i;
    for (int ko = 0; ko < N; ++ko) {           // output core ko
      const int k = reverse ? N - 1 - ko : ko;  // batch core holding it
      const long long n = b->dims[k], r0 = b->rk(t, k), r1 = b->rk(t, k + 1), cap0 = b->capr(t, k);
      double* dst = direct ? (double*)views[(size_t)i * N + ko] : (double*)d + o;
      if (!reverse)
        hc[ci++] = cd3(b->core(t, k), dst, n, r0, r1, cap0, 1, cap0 * n, 1, n, n * r0);
      else  // output (i, a, b) with a < r1, b < r0 from internal (b, i, a)
        hc[ci++] = cd3(b->core(t, k), dst, n, r1, r0, cap0, cap0 * n, 1, 1, n, n * r1);
      maxe = std::max<long long>(maxe, n * r0 * r1);
      offs.push_back(o);
      if (!direct) o += (size_t)n * r0 * r1;
    }
  }
  TTC_CUDA(cudaMemcpyAsync(d + off_desc, h + off_desc, nd * sizeof(CopyDesc), cudaMemcpyHostToDevice, c->stream));
  launch_copy((const CopyDesc*)(d + off_desc), (int)ci, maxe, c->stream);
  if (direct) {
    TTC_CUDA(cudaStreamSynchronize(c->stream));
  } else {
    size_t q = 0;
    std::vector<HostCopy> hcp;
    for (int i = 0; i < m; ++i) {
      const int t = first + i;
      for (int ko = 0; ko < N; ++ko) {
        const int k = reverse ? N - 1 - ko : ko;
        const size_t cnt = (size_t)b->dims[k] * b->rk(t, k) * b->rk(t, k + 1);
        hcp.push_back({ys[i].cores[ko], (double*)h + offs[q++], cnt * sizeof(double)});
      }
    }
    // transfer chunk by chunk, an event after each; unpack a chunk while the next ones arrive
    std::vector<std::pair<size_t, size_t>> groups;   // [gi, gj) of hcp
    std::vector<cudaEvent_t> evs;
    size_t sent = 0;
    try {
      for (size_t gi = 0; gi < hcp.size();) {
        size_t gj = gi, bytes = 0;
        while (gj < hcp.size() && (gj == gi || bytes < kStageChunk)) bytes += hcp[gj++].bytes;
        cudaEvent_t e;
        TTC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        evs.push_back(e);
        TTC_CUDA(cudaMemcpyAsync(h + sent, d + sent, bytes, cudaMemcpyDeviceToHost, c->stream));
        TTC_CUDA(cudaEventRecord(e, c->stream));
        groups.push_back({gi, gj});
        sent += bytes;
        gi = gj;
      }
      for (size_t g = 0; g < groups.size(); ++g) {
        TTC_CUDA(cudaEventSynchronize(evs[g]));
        parallel_memcpy(std::vector<HostCopy>(hcp.begin() + (long)groups[g].first, hcp.begin() + (long)groups[g].second));
      }
    } catch (...) {
      cudaStreamSynchronize(c->stream);
      for (auto e : evs) cudaEventDestroy(e);
      throw;
    }
    TTC_CUDA(cudaStreamSynchronize(c->stream));
    for (auto e : evs) cudaEventDestroy(e);
  }
  for (int i = 0; i < m; ++i) {
    const int t = first + i;
    for (int k = 0; k <= N; ++k) ys[i].rks[k] = b->rk(t, reverse ? N - k : k);
    if (ys[i].ot)
      for (int k = 0; k < N; ++k)
        ys[i].ot[k] = reverse ? -b->h_ot[(size_t)t * N + (N - 1 - k)] : b->h_ot[(size_t)t * N + k];
  }
}

// A one-TT batch holding the host tensor x, with capacities max(cap, x.rks).
ttc_batch* batch_from_host(ttc_context* c, const ttc_ttv* x, const std::vector<int>* cap, bool reverse) {
  validate_ttv(x);
  const int N = x->N;
  std::vector<long long> dims(N);
  for (int k = 0; k < N; ++k) dims[k] = x->dims[reverse ? N - 1 - k : k];
  std::vector<int> cp(N + 1);
  for (int k = 0; k <= N; ++k) cp[k] = std::max<int>((int)x->rks[reverse ? N - k : k], cap ? (*cap)[k] : 1);
  ttc_batch* b = batch_create(c, 1, N, dims.data(), cp.data());
  try {
    batch_upload_many(b, 0, 1, x, reverse);
  } catch (...) {
    batch_destroy(b);
    throw;
  }
  return b;
}

ttc_batch* oneshot_batch(ttc_context* c, const std::string& key, const std::function<ttc_batch*()>& make) {
  auto& v = c->oneshot;
  for (size_t i = 0; i < v.size(); ++i)
    if (v[i].first == key) {
      auto e = v[i];
      v.erase(v.begin() + (long)i);
      v.push_back(e);
      return e.second;
    }
  ttc_batch* b = make();
  v.emplace_back(key, b);
  constexpr size_t kKeep = 8;
  while (v.size() > kKeep) {
    TTC_CUDA(cudaStreamSynchronize(c->stream));
    ttc_batch* old = v.front().second;
    v.erase(v.begin());
    batch_destroy(old);            // drops the plans that name it as well
  }
  return b;
}

void oneshot_clear(ttc_context* c) {
  for (auto& e : c->oneshot) batch_destroy(e.second);
  c->oneshot.clear();
}

ttc_batch* batch_empty_like(ttc_context* c, int count, int N, const std::vector<long long>& dims,
                            const std::vector<int>& cap_per_tt) {
  std::vector<int> cp;
  for (int t = 0; t < count; ++t) cp.insert(cp.end(), cap_per_tt.begin(), cap_per_tt.end());
  return batch_create(c, count, N, dims.data(), cp.data());
}



void set_jacobi_max_sweeps(ttc_context* c, int sweeps) {
  TTC_REQUIRE(sweeps >= 1, TTC_EARG, "the Jacobi sweep cap must be at least 1");
  if (c->jacobi_max_sweeps == sweeps) return;
  TTC_CUDA(cudaStreamSynchronize(c->stream));     // no plan of the old cap still running
  c->jacobi_max_sweeps = sweeps;
  c->plans.clear();
}

void record_stats(ttc_context* c, int nstages) {
  TTC_CUDA(cudaStreamSynchronize(c->stream));
  // an event pair that cannot be timed reports 0 (its error is consumed here, so that it is
  // not picked up by a later launch check)
  auto elapsed = [](cudaEvent_t a, cudaEvent_t b) {
    float v = 0.0f;
    if (cudaEventElapsedTime(&v, a, b) != cudaSuccess) {
      cudaGetLastError();
      v = 0.0f;
    }
    return v;
  };
  float ms[8] = {0};
  if (!c->last_run_graph)   // stage events are recorded only outside CUDA graphs
    for (int i = 0; i + 1 < nstages; ++i) ms[i] = elapsed(c->ev[i], c->ev[i + 1]);
  const float tot = elapsed(c->ev[kEvRunBegin], c->ev[kEvRunEnd]);
  c->stats.total_ms = tot;
  c->stats.sketch_ms = 0; c->stats.orth_ms = 0; c->stats.svd_ms = 0;
  if (nstages == 3) { c->stats.orth_ms = ms[0]; c->stats.svd_ms = ms[1]; }
  if (nstages == 4) { c->stats.sketch_ms = ms[0]; c->stats.orth_ms = ms[1]; c->stats.svd_ms = ms[2]; }
}

std::vector<const double*> upload_host_blocks(ttc_context* c, const std::vector<long long>& dims, const SketchPlan& sp,
                                              const double* const* blocks, std::string& key) {
  std::vector<const double*> out;
  if (!blocks) return out;
  const int N = (int)dims.size();
  size_t total = 0;
  for (int k = 0; k < N; ++k) total += (size_t)sp.b[k + 1] * dims[k] * sp.b[k] * sp.p[k];
  if (total > c->sk_cap) {
    if (c->d_sk) { region_remove(c->d_sk); cudaFree(c->d_sk); }
    c->d_sk = nullptr;
    TTC_CUDA(cudaMalloc(&c->d_sk, total * sizeof(double)));
    region_add(c->d_sk, total * sizeof(double));
    c->sk_cap = total;
  }
  size_t o = 0;
  for (int k = 0; k < N; ++k) {
    TTC_REQUIRE(blocks[k] != nullptr, TTC_EARG, "sketch_blocks: null block");
    const size_t cnt = (size_t)sp.b[k + 1] * dims[k] * sp.b[k] * sp.p[k];
    TTC_CUDA(cudaMemcpyAsync(c->d_sk + o, blocks[k], cnt * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    out.push_back(c->d_sk + o);
    o += cnt;
  }
  TTC_CUDA(cudaStreamSynchronize(c->stream));
  key = "hostsk:" + std::to_string((unsigned long long)(uintptr_t)c->d_sk) + ":";
  return out;
}

std::vector<long long> rks_vec(const int64_t* rks, int N) {
  TTC_REQUIRE(rks != nullptr, TTC_EARG, "rks is null");
  return std::vector<long long>(rks, rks + N + 1);
}

}  // namespace ttc

// ================================================================= extern "C"
extern "C" {

const char* ttc_version(void) { return "libttcuda 0.1 sm_100a (tcgen05 BF16 sketch, FP64 QR/Jacobi)"; }

int ttc_create(ttc_context** out, int device) {
  if (!out) return TTC_EARG;
  ttc_context* c = new (std::nothrow) ttc_context();
  if (!c) return TTC_ENOMEM;
  c->device = device;
  const int st = guard(c, [&] {
    int n = 0;
    TTC_CUDA(cudaGetDeviceCount(&n));
    TTC_REQUIRE(device >= 0 && device < n, TTC_EARG, "ttc_create: no such device");
    TTC_CUDA(cudaSetDevice(device));
    TTC_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = true;
    TTC_CUDA(cudaMalloc(&c->d_flags, 64));
    region_add(c->d_flags, 64);
    TTC_CUDA(cudaMemset(c->d_flags, 0, 64));
    TTC_CUDA(cudaMalloc(&c->d_one, 64));
    region_add(c->d_one, 64);
    const double one[8] = {1.0, 0, 0, 0, 0, 0, 0, 0};
    TTC_CUDA(cudaMemcpy(c->d_one, one, sizeof(one), cudaMemcpyHostToDevice));
    for (auto& e : c->ev) TTC_CUDA(cudaEventCreate(&e));
  });
  if (st != TTC_OK) {
    g_err_noctx = c->err;
    delete c;
    return st;
  }
  *out = c;
  return TTC_OK;
}

int ttc_destroy(ttc_context* c) {
  if (!c) return TTC_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  c->plans.clear();
  try {
    oneshot_clear(c);
  } catch (...) {
  }
  for (void* p : {(void*)c->ws, c->d_stage, (void*)c->d_sk, (void*)c->d_flags, (void*)c->d_one}) region_remove(p);
  if (c->ws) cudaFree(c->ws);
  if (c->d_stage) cudaFree(c->d_stage);
  if (c->h_stage) cudaFreeHost(c->h_stage);
  if (c->d_sk) cudaFree(c->d_sk);
  if (c->d_flags) cudaFree(c->d_flags);
  if (c->d_one) cudaFree(c->d_one);
  for (auto& e : c->ev) if (e) cudaEventDestroy(e);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return TTC_OK;
}

int ttc_set_stream(ttc_context* c, void* stream) {
  if (!c) return TTC_EARG;
  return guard(c, [&] {
    TTC_CUDA(cudaStreamSynchronize(c->stream));
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
  });
}

const char* ttc_last_error(const ttc_context* c) { return c ? c->err.c_str() : g_err_noctx.c_str(); }

int ttc_get_stats(const ttc_context* c, ttc_stats* out) {
  if (!c || !out) return TTC_EARG;
  *out = c->stats;
  return TTC_OK;
}

int ttc_set_profiling(ttc_context* c, int on) {
  if (!c) return TTC_EARG;
  c->profiling = (on != 0);
  return TTC_OK;
}

int ttc_synchronize(ttc_context* c) {
  if (!c) return TTC_EARG;
  return guard(c, [&] {
    TTC_CUDA(cudaStreamSynchronize(c->stream));
    check_device_flags(c);
  });
}

int ttc_batch_create(ttc_context* c, int32_t count, int32_t N, const int64_t* dims, const int64_t* rks_cap,
                     ttc_batch** out) {
  if (!c || !out || !dims || !rks_cap) return TTC_EARG;
  return guard(c, [&] {
    std::vector<long long> d(dims, dims + N);
    std::vector<int> cp((size_t)count * (N + 1));
    for (size_t i = 0; i < cp.size(); ++i) {
      TTC_REQUIRE(rks_cap[i] >= 1 && rks_cap[i] < (1 << 20), TTC_EARG, "batch: bad capacity");
      cp[i] = (int)rks_cap[i];
    }
    for (int t = 0; t < count; ++t)
      TTC_REQUIRE(cp[(size_t)t * (N + 1)] == 1 && cp[(size_t)t * (N + 1) + N] == 1, TTC_EDIM,
                  "batch: boundary capacities must be 1");
    *out = batch_create(c, count, N, d.data(), cp.data());
  });
}

int ttc_batch_destroy(ttc_batch* b) {
  if (!b) return TTC_OK;
  ttc_context* c = b->ctx;
  return guard(c, [&] {
    TTC_CUDA(cudaStreamSynchronize(c->stream));
    batch_destroy(b);
  });
}

int ttc_batch_upload(ttc_batch* b, int32_t index, const ttc_ttv* x) {
  if (!b || !x) return TTC_EARG;
  return guard(b->ctx, [&] {
    TTC_REQUIRE(index >= 0 && index < b->count, TTC_EARG, "upload: index out of range");
    batch_upload_many(b, index, 1, x);
  });
}

int ttc_host_alloc(size_t bytes, void** out) {
  if (!out || bytes == 0) return TTC_EARG;
  *out = nullptr;
  const cudaError_t e = cudaHostAlloc(out, bytes, cudaHostAllocMapped | cudaHostAllocPortable);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    ttc::set_noctx_error(std::string("ttc_host_alloc: ") + cudaGetErrorString(e));
    return TTC_ENOMEM;
  }
  return TTC_OK;
}

int ttc_host_free(void* p) {
  if (!p) return TTC_OK;
  const cudaError_t e = cudaFreeHost(p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    ttc::set_noctx_error(std::string("ttc_host_free: ") + cudaGetErrorString(e));
    return TTC_ECUDA;
  }
  return TTC_OK;
}

int ttc_batch_upload_all(ttc_batch* b, const ttc_ttv* xs) {
  if (!b || !xs) return TTC_EARG;
  return guard(b->ctx, [&] { batch_upload_many(b, 0, b->count, xs); });
}

int ttc_batch_download(ttc_batch* b, int32_t index, ttc_ttv_out* y) {
  if (!b || !y) return TTC_EARG;
  return guard(b->ctx, [&] {
    TTC_REQUIRE(index >= 0 && index < b->count, TTC_EARG, "download: index out of range");
    check_device_flags(b->ctx);
    batch_download_many(b, index, 1, y);
  });
}

int ttc_batch_download_all(ttc_batch* b, ttc_ttv_out* ys) {
  if (!b || !ys) return TTC_EARG;
  return guard(b->ctx, [&] {
    check_device_flags(b->ctx);
    batch_download_many(b, 0, b->count, ys);
  });
}

int ttc_batch_ranks(ttc_batch* b, int32_t index, int64_t* rks) {
  if (!b || !rks) return TTC_EARG;
  return guard(b->ctx, [&] {
    TTC_REQUIRE(index >= 0 && index < b->count, TTC_EARG, "ranks: index out of range");
    batch_sync_ranks(b);
    for (int k = 0; k <= b->N; ++k) rks[k] = b->rk(index, k);
  });
}

size_t ttc_batch_bytes(const ttc_batch* b) {
  if (!b) return 0;
  return sizeof(double) * (size_t)b->total + sizeof(int) * (b->h_rks.size() + b->count);
}

int ttc_batch_round_det(ttc_context* c, ttc_batch* x, const ttc_round_opts* opts, ttc_batch* y) {
  if (!c || !x || !y || !opts) return TTC_EARG;
  return guard(c, [&] {
    with_svd_retry(c, [&] {
      round_det(c, x, *opts, y);
      record_stats(c, 3);
      check_device_flags(c);
    });
  });
}

int ttc_batch_round_det_async(ttc_context* c, ttc_batch* x, const ttc_round_opts* opts, ttc_batch* y) {
  if (!c || !x || !y || !opts) return TTC_EARG;
  return guard(c, [&] { round_det(c, x, *opts, y); });
}

int ttc_batch_round_rand(ttc_context* c, ttc_batch* x, const int64_t* rks, const ttc_sketch_opts* sk,
                         const ttc_round_opts* after, ttc_batch* y) {
  if (!c || !x || !y || !sk) return TTC_EARG;
  return guard(c, [&] {
    std::string key;
    const auto r = rks_vec(rks, x->N);
    const auto raw = upload_host_blocks(c, x->dims, sketch_plan(x->dims, r, sk->block_rks), sk->sketch_blocks, key);
    with_svd_retry(c, [&] {
      round_rand(c, x, r, *sk, after, y, raw, key);
      record_stats(c, 4);
      check_device_flags(c);
    });
  });
}

int ttc_batch_round_rand_async(ttc_context* c, ttc_batch* x, const int64_t* rks, const ttc_sketch_opts* sk,
                               const ttc_round_opts* after, ttc_batch* y) {
  if (!c || !x || !y || !sk) return TTC_EARG;
  return guard(c, [&] {
    TTC_REQUIRE(sk->sketch_blocks == nullptr, TTC_EARG, "async rounding takes device-generated sketches only");
    round_rand(c, x, rks_vec(rks, x->N), *sk, after, y, {}, "");
  });
}

int ttc_tt_rounding(ttc_context* c, const ttc_ttv* x, const ttc_round_opts* opts, ttc_ttv_out* y) {
  if (!c || !x || !opts || !y) return TTC_EARG;
  return guard(c, [&] { tt_rounding_host(c, x, *opts, y); });
}

int ttc_orthogonalize(ttc_context* c, const ttc_ttv* x, int32_t i, ttc_ttv_out* y) {
  if (!c || !x || !y) return TTC_EARG;
  return guard(c, [&] { orthogonalize_host(c, x, i, y); });
}

int ttc_norm(ttc_context* c, const ttc_ttv* x, double* out) {
  if (!c || !x || !out) return TTC_EARG;
  return guard(c, [&] { *out = norm_host(c, x); });
}

int ttc_recursive_sketch(ttc_context* c, const ttc_ttv* A, const int64_t* rks, const ttc_sketch_opts* sk,
                         double* const* W_out, int64_t* sketch_rks) {
  if (!c || !A || !sk || !W_out || !sketch_rks) return TTC_EARG;
  return guard(c, [&] { recursive_sketch_host(c, A, nullptr, rks, *sk, W_out, sketch_rks); });
}

int ttc_recursive_sketch_op(ttc_context* c, const ttc_tto* H, const ttc_ttv* A, const int64_t* rks,
                            const ttc_sketch_opts* sk, double* const* W_out, int64_t* sketch_rks) {
  if (!c || !H || !A || !sk || !W_out || !sketch_rks) return TTC_EARG;
  return guard(c, [&] { recursive_sketch_host(c, A, H, rks, *sk, W_out, sketch_rks); });
}

int ttc_ttrand_rounding(ttc_context* c, const ttc_ttv* x, const int64_t* rks, const ttc_sketch_opts* sk, ttc_ttv_out* y) {
  if (!c || !x || !sk || !y) return TTC_EARG;
  return guard(c, [&] {
    const double one = 1.0;
    rand_rounding_host(c, 1, &one, nullptr, x, nullptr, rks, *sk, y);
  });
}

int ttc_ttrand_rounding_lincomb(ttc_context* c, int32_t m, const double* alpha, const ttc_ttv* ys, const int64_t* rks,
                                const ttc_sketch_opts* sk, ttc_ttv_out* y) {
  if (!c || m < 1 || !alpha || !ys || !sk || !y) return TTC_EARG;
  return guard(c, [&] { rand_rounding_host(c, m, alpha, nullptr, ys, nullptr, rks, *sk, y); });
}

int ttc_ttrand_rounding_hadamard(ttc_context* c, int32_t m, const ttc_ttv* ys, const int64_t* rks,
                                 const ttc_sketch_opts* sk, ttc_ttv_out* y) {
  if (!c || m < 1 || !ys || !rks || !sk || !y) return TTC_EARG;
  return guard(c, [&] {
    if (m == 1) {
      const double one = 1.0;
      rand_rounding_host(c, 1, &one, nullptr, ys, nullptr, rks, *sk, y);
    } else {
      hadamard_rounding_host(c, m, ys, rks, *sk, y);
    }
  });
}

int ttc_stta(ttc_context* c, int32_t m, const double* alpha, const ttc_ttv* ys, const int64_t* rks, uint64_t seed_left,
             uint64_t seed_right, int32_t orthogonal, int64_t block_rks, ttc_ttv_out* y) {
  if (!c || m < 1 || !alpha || !ys || !rks || !y) return TTC_EARG;
  return guard(c, [&] { stta_host(c, m, alpha, ys, rks, seed_left, seed_right, orthogonal, block_rks, y); });
}

int ttc_ttrand_rounding_op(ttc_context* c, int32_t m, const double* alpha, const ttc_tto* A, const ttc_ttv* ys,
                           const int64_t* rks, const ttc_sketch_opts* sk, ttc_ttv_out* y) {
  if (!c || m < 1 || !alpha || !A || !ys || !sk || !y) return TTC_EARG;
  return guard(c, [&] { rand_rounding_host(c, m, alpha, A, ys, nullptr, rks, *sk, y); });
}

int ttc_ttrand_rounding_residual(ttc_context* c, const ttc_tto* A, const ttc_ttv* x, const ttc_ttv* b,
                                 const int64_t* rks, const ttc_sketch_opts* sk, ttc_ttv_out* y) {
  if (!c || !A || !x || !b || !sk || !y) return TTC_EARG;
  return guard(c, [&] {
    const double al[2] = {1.0, -1.0};
    const ttc_ttv ys[2] = {*x, *b};
    rand_rounding_host(c, 2, al, A, ys, nullptr, rks, *sk, y);
  });
}

int ttc_mpo_apply(ttc_context* c, const ttc_tto* A, const ttc_ttv* x, ttc_ttv_out* y) {
  if (!c || !A || !x || !y) return TTC_EARG;
  return guard(c, [&] { mpo_apply_host(c, A, x, y); });
}

int ttc_dot(ttc_context* c, const ttc_ttv* A, const ttc_ttv* B, double* out) {
  if (!c || !A || !B || !out) return TTC_EARG;
  return guard(c, [&] { *out = dot_host(c, A, B, nullptr, 1); });
}

int ttc_partial_contraction(ttc_context* c, const ttc_ttv* A, const ttc_ttv* B, int32_t reverse, double* const* W_out) {
  if (!c || !A || !B || !W_out) return TTC_EARG;
  return guard(c, [&] { dot_host(c, A, B, W_out, reverse); });
}

int ttc_dot_operator(ttc_context* c, const ttc_ttv* psi, const ttc_tto* H, const ttc_ttv* phi, double* out) {
  if (!c || !psi || !H || !phi || !out) return TTC_EARG;
  return guard(c, [&] { *out = dot_operator_host(c, psi, H, phi); });
}

int ttc_tt_add(ttc_context* c, const ttc_ttv* x, const ttc_ttv* y, ttc_ttv_out* out) {
  if (!c || !x || !y || !out) return TTC_EARG;
  return guard(c, [&] { tt_add_host(c, x, y, out); });
}

int ttc_tt_scale(ttc_context* c, double a, const ttc_ttv* x, ttc_ttv_out* out) {
  if (!c || !x || !out) return TTC_EARG;
  return guard(c, [&] { tt_scale_host(c, a, x, out); });
}

int ttc_rayleigh_grad(ttc_context* c, const ttc_tto* H, const ttc_ttv* x, int32_t ckpt_every, double* value,
                      double* const* grads) {
  if (!c || !H || !x || !value || !grads) return TTC_EARG;
  return guard(c, [&] { rayleigh_grad_host(c, H, x, ckpt_every, value, grads); });
}

int ttc_rayleigh_grad_prec(ttc_context* c, const ttc_tto* H, const ttc_ttv* x, int32_t ckpt_every, int32_t precision,
                           double* value, double* const* grads) {
  if (!c || !H || !x || !value || !grads) return TTC_EARG;
  return guard(c, [&] {
    TTC_REQUIRE(precision == TTC_PREC_FP64 || precision == TTC_PREC_FP32, TTC_EARG,
                "rayleigh_grad: precision must be TTC_PREC_FP64 or TTC_PREC_FP32");
    rayleigh_grad_host(c, H, x, ckpt_every, value, grads, precision == TTC_PREC_FP32);
  });
}

}  // extern "C"
