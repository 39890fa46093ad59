// Kernel-level test entry points: run one device kernel on host arrays so the tests can
// check it against numpy in isolation.  They are exported for the test suite only and are
// not part of the public ABI in include/ttcuda.h.
#include <cstring>

#include "api_impl.cuh"
#include "regions.cuh"

using namespace ttc;

namespace {
struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
  explicit DevBuf(size_t bytes) : n(bytes) {
    if (bytes == 0) bytes = 8;
    TTC_CUDA(cudaMalloc(&p, bytes));
    TTC_CUDA(cudaMemset(p, 0, bytes));
    region_add(p, bytes);
  }
  ~DevBuf() { region_remove(p); cudaFree(p); }
  template <class T> T* as() const { return (T*)p; }
};

template <class F>
int hook(ttc_context* c, F&& f) {
  try {
    TTC_CUDA(cudaSetDevice(c->device));
    f();
    TTC_CUDA(cudaStreamSynchronize(c->stream));
    check_device_flags(c);
    return TTC_OK;
  } catch (const Error& e) {
    c->err = e.what();
    return e.status;
  } catch (const std::exception& e) {
    c->err = e.what();
    return TTC_EINTERNAL;
  }
}

void run_plan_once(ttc_context* c, const std::function<void(Builder&)>& fn) {
  static unsigned long long serial = 0;
  const std::string key = "hook:" + std::to_string(++serial);
  Plan* p = get_plan(c, key, fn);
  run_plan(c, *p);
  TTC_CUDA(cudaStreamSynchronize(c->stream));
  c->plans.erase(key);
}
}  // namespace

extern "C" {

// Sets the context's Jacobi SVD sweep cap (default 40), so that the tests can make the sweep run
// out of sweeps (TTC_ENOCONV) on purpose and watch the retry.
int ttc_test_set_jacobi_max_sweeps(ttc_context* c, int sweeps) {
  try {
    set_jacobi_max_sweeps(c, sweeps);
    return TTC_OK;
  } catch (const Error& e) {
    c->err = e.what();
    return e.status;
  }
}

// Sets the poll limit of the tensor-core GEMM's bounded mbarrier waits on the context's device
// (default 2^24), so that a test can make the waits run out on purpose.
int ttc_test_set_tc_wait_limit(ttc_context* c, long long polls) {
  return hook(c, [&] { set_tc_wait_limit(polls); });
}

// Device-resident timing of the tcgen05 GEMM C = A B^T (M x N, K; BF16 operands, or FP32 read as
// TF32) for kernel benchmarks: operands filled on the device, `reps` launches of one plan timed
// with events on the context stream after one warm-up launch; *ms_out = milliseconds per launch.
int ttc_test_tc_gemm_bench(ttc_context* c, int m, int n, int k, int tf32, int reps, double* ms_out) {
  return hook(c, [&] {
    TTC_REQUIRE(m > 0 && n > 0 && k > 0 && reps > 0 && ms_out, TTC_EARG, "tc gemm bench: bad arguments");
    const long long esz = tf32 ? 4 : 2, chunk = 16 / esz;
    const long long ld = (k + chunk - 1) / chunk * chunk;
    DevBuf dA((size_t)(m * ld * esz)), dB((size_t)(n * ld * esz)), dC((size_t)m * n * 4), dS((size_t)std::max(m, n) * ld * 8);
    // operands: a smooth deterministic pattern converted from FP64 on the device
    run_plan_once(c, [&](Builder& B) {
      std::vector<PhiloxDesc> ph{{dS.as<double>(), (long long)std::max(m, n) * ld, 7ull, 0u, 0.1}};
      B.philox(ph);
      CvtDesc a{}, b{};
      a.src = dS.as<double>(); a.dst = dA.p; a.rows = k; a.cols = m; a.ss_i = 1; a.ss_j = ld; a.ds_i = 1; a.ds_j = ld; a.alpha = 1.0;
      b = a; b.dst = dB.p; b.cols = n;
      B.cvt_bf16({a, b}, tf32 != 0);
    });
    std::string key = "tcbench:" + std::to_string(m) + ":" + std::to_string(n) + ":" + std::to_string(k);
    Plan* p = get_plan(c, key, [&](Builder& B) {
      Bf16GemmDesc d{};
      d.m = m; d.n = n; d.k = k; d.m0 = m;
      d.A = dA.p; d.lda = ld; d.B = dB.p; d.ldb = ld;
      d.C32 = dC.as<float>(); d.c_i0 = 1; d.c_i1 = 0; d.c_j = m;
      d.alpha = 1.0;
      B.bf16gemm({d}, tf32 != 0);
    });
    run_plan(c, *p);
    TTC_CUDA(cudaEventRecord(c->ev[0], c->stream));
    for (int i = 0; i < reps; ++i) run_plan(c, *p);
    TTC_CUDA(cudaEventRecord(c->ev[1], c->stream));
    TTC_CUDA(cudaEventSynchronize(c->ev[1]));
    float ms = 0.f;
    TTC_CUDA(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
    *ms_out = ms / reps;
    TTC_CUDA(cudaStreamSynchronize(c->stream));
    c->plans.erase(key);
  });
}

// Builds a plan whose copy descriptor points `offset` bytes past the end of the context's
// workspace: the host-side registry check refuses it (TTC_EINTERNAL) before any launch.
int ttc_test_bad_descriptor(ttc_context* c, long long offset) {
  return hook(c, [&] {
    ensure_workspace(c, 1 << 20);
    double* past = reinterpret_cast<double*>(c->ws + c->ws_bytes + offset);
    // the address must lie outside every registered allocation, or the plan below would run
    bool registered = true;
    try {
      region_check(past, 4 * sizeof(double), "probe");
    } catch (const Error&) {
      registered = false;
    }
    TTC_REQUIRE(!registered, TTC_EARG, "test address lies inside a registered allocation");
    run_plan_once(c, [&](Builder& B) { B.copy({cd2(past, past, 4, 1, 1, 4, 1, 4)}); });
  });
}

// C = alpha * A * B + beta * C with split strides (a_str = {i0, i1, k0, k1, b}, ...), the plan
// run `runs` times (with beta == 0 every run writes the same C; the repeats check that the
// split-K tile counters are left zero for the next launch).  *ksplit_out (when given) receives
// the split count the planner chose.
int ttc_test_gemm_runs(ttc_context* c, int m, int n, int k, int batch, int m0, int n0, int k0e, const double* A,
                       long long a_len, const long long* as, const double* Bh, long long b_len, const long long* bs,
                       double* Ch, long long c_len, const long long* cs, double alpha, double beta, int runs,
                       int* ksplit_out) {
  return hook(c, [&] {
    TTC_REQUIRE(runs >= 1 && (runs == 1 || beta == 0.0), TTC_EARG, "repeated runs need beta == 0");
    DevBuf dA(a_len * 8), dB(b_len * 8), dC(c_len * 8);
    TTC_CUDA(cudaMemcpy(dA.p, A, a_len * 8, cudaMemcpyHostToDevice));
    TTC_CUDA(cudaMemcpy(dB.p, Bh, b_len * 8, cudaMemcpyHostToDevice));
    TTC_CUDA(cudaMemcpy(dC.p, Ch, c_len * 8, cudaMemcpyHostToDevice));
    static unsigned long long serial = 0;
    const std::string key = "hook-gemm:" + std::to_string(++serial);
    int ks = 1;
    Plan* p = get_plan(c, key, [&](Builder& B) {
      GemmDesc d{};
      d.m = m; d.n = n; d.k = k; d.batch = batch; d.m0 = m0; d.n0 = n0; d.k0e = k0e;
      d.A = dA.as<double>(); d.a_i0 = as[0]; d.a_i1 = as[1]; d.a_k0 = as[2]; d.a_k1 = as[3]; d.a_b = as[4];
      d.B = dB.as<double>(); d.b_k0 = bs[0]; d.b_k1 = bs[1]; d.b_j0 = bs[2]; d.b_j1 = bs[3]; d.b_b = bs[4];
      d.C = dC.as<double>(); d.c_i0 = cs[0]; d.c_i1 = cs[1]; d.c_j0 = cs[2]; d.c_j1 = cs[3]; d.c_b = cs[4];
      d.alpha = alpha; d.beta = beta;
      B.gemm({d});
      ks = gemm_pick_ksplit(d, gemm_tiles(d), current_sm_count());
    });
    for (int r = 0; r < runs; ++r) run_plan(c, *p);
    TTC_CUDA(cudaStreamSynchronize(c->stream));
    c->plans.erase(key);
    if (ksplit_out) *ksplit_out = ks;
    TTC_CUDA(cudaMemcpy(Ch, dC.p, c_len * 8, cudaMemcpyDeviceToHost));
  });
}

int ttc_test_gemm(ttc_context* c, int m, int n, int k, int batch, int m0, int n0, int k0e, const double* A,
                  long long a_len, const long long* as, const double* Bh, long long b_len, const long long* bs,
                  double* Ch, long long c_len, const long long* cs, double alpha, double beta) {
  return ttc_test_gemm_runs(c, m, n, k, batch, m0, n0, k0e, A, a_len, as, Bh, b_len, bs, Ch, c_len, cs, alpha, beta,
                            1, nullptr);
}

// Householder QR of A (m x n, col-major): Q (m x K), R (K x n).
int ttc_test_qr(ttc_context* c, int m, int n, const double* A, double* Q, double* R) {
  return hook(c, [&] {
    const int K = std::min(m, n);
    DevBuf dA((size_t)m * n * 8), dQ((size_t)m * K * 8), dR((size_t)K * n * 8), dT((size_t)((K + 15) / 16 + 1) * 256 * 8);
    TTC_CUDA(cudaMemcpy(dA.p, A, (size_t)m * n * 8, cudaMemcpyHostToDevice));
    run_plan_once(c, [&](Builder& B) {
      B.qr({{m, n, dA.as<double>(), m, dQ.as<double>(), m, dR.as<double>(), K, dT.as<double>()}});
    });
    TTC_CUDA(cudaMemcpy(Q, dQ.p, (size_t)m * K * 8, cudaMemcpyDeviceToHost));
    TTC_CUDA(cudaMemcpy(R, dR.p, (size_t)K * n * 8, cudaMemcpyDeviceToHost));
  });
}

// One-sided Jacobi of X (m x n): X <- X W (orthogonal columns), sigma, perm; W if accw.
// *sweeps receives the sweeps used (negative when the cap was hit; not raised as an error here).
int ttc_test_jacobi(ttc_context* c, int m, int n, double* X, int accw, double* W, double* sigma, int* perm,
                    int* sweeps) {
  return hook(c, [&] {
    DevBuf dX((size_t)m * n * 8), dW((size_t)n * n * 8), ds((size_t)n * 8), dp((size_t)n * 4), di(8);
    TTC_CUDA(cudaMemcpy(dX.p, X, (size_t)m * n * 8, cudaMemcpyHostToDevice));
    run_plan_once(c, [&](Builder& B) {
      JacobiDesc d{m, n, dX.as<double>(), m, accw ? dW.as<double>() : nullptr, n, ds.as<double>(), dp.as<int>(),
                   di.as<int>()};
      B.jacobi({d});
    });
    TTC_CUDA(cudaMemcpy(X, dX.p, (size_t)m * n * 8, cudaMemcpyDeviceToHost));
    if (accw) TTC_CUDA(cudaMemcpy(W, dW.p, (size_t)n * n * 8, cudaMemcpyDeviceToHost));
    TTC_CUDA(cudaMemcpy(sigma, ds.p, (size_t)n * 8, cudaMemcpyDeviceToHost));
    TTC_CUDA(cudaMemcpy(perm, dp.p, (size_t)n * 4, cudaMemcpyDeviceToHost));
    TTC_CUDA(cudaMemcpy(sweeps, di.p, 4, cudaMemcpyDeviceToHost));
    TTC_CUDA(cudaMemset(c->d_flags, 0, sizeof(int)));
  });
}

// The batched Jacobi SVD alone: `count` m x n problems (X, column-major, one after another) are
// copied into a work array and factored, `reps` times in one plan run; *ms receives the device time
// per repetition (copy included) and sweeps[i] the sweeps problem i used in the last repetition.
int ttc_test_jacobi_bench(ttc_context* c, int count, int m, int n, const double* X, int reps, double* ms,
                          int* sweeps) {
  return hook(c, [&] {
    TTC_REQUIRE(count >= 1 && m >= n && n >= 1 && reps >= 1, TTC_EARG, "jacobi bench: bad sizes");
    const size_t per = (size_t)m * n;
    DevBuf d0(per * count * 8), dX(per * count * 8), ds((size_t)n * count * 8), dp((size_t)n * count * 4),
        di((size_t)count * 4);
    TTC_CUDA(cudaMemcpy(d0.p, X, per * count * 8, cudaMemcpyHostToDevice));
    static unsigned long long serial = 0;
    const std::string key = "hook-jacobi:" + std::to_string(++serial);
    Plan* p = get_plan(c, key, [&](Builder& B) {
      for (int r = 0; r < reps; ++r) {
        if (r == 0) B.stage(0);
        B.copy({cd2(d0.as<double>(), dX.as<double>(), (long long)(per * count), 1, 1, 0, 1, 0)});
        std::vector<JacobiDesc> v;
        for (int i = 0; i < count; ++i)
          v.push_back({m, n, dX.as<double>() + per * i, m, nullptr, n, ds.as<double>() + (size_t)n * i,
                       dp.as<int>() + (size_t)n * i, di.as<int>() + i, nullptr, 0});
        B.jacobi(v);
      }
      B.stage(1);
    });
    // the first run loads the kernels and the second captures the graph: time the third, a
    // replay of the whole plan
    for (int run = 0; run < 3; ++run) {
      run_plan(c, *p);
      TTC_CUDA(cudaStreamSynchronize(c->stream));
    }
    float t = 0.f;
    TTC_CUDA(cudaEventElapsedTime(&t, c->ev[kEvRunBegin], c->ev[kEvRunEnd]));
    *ms = (double)t / reps;
    TTC_CUDA(cudaMemcpy(sweeps, di.p, (size_t)count * 4, cudaMemcpyDeviceToHost));
    c->plans.erase(key);
    TTC_CUDA(cudaMemset(c->d_flags, 0, sizeof(int)));
  });
}

// tcgen05 BF16 GEMM: C (m x n, col-major, FP64 out) = alpha * bf16(A) bf16(B)^T with A (m x k)
// and B (n x k) given row-major in FP64 (converted to BF16 on the device).
int ttc_test_bf16_gemm(ttc_context* c, int m, int n, int k, const double* A, const double* Bh, double* C,
                       double alpha) {
  return hook(c, [&] {
    const long long lda = (k + 7) / 8 * 8;
    DevBuf dA((size_t)m * k * 8), dB((size_t)n * k * 8), dC((size_t)m * n * 8);
    DevBuf a16((size_t)m * lda * 2 + 64), b16((size_t)n * lda * 2 + 64);
    TTC_CUDA(cudaMemcpy(dA.p, A, (size_t)m * k * 8, cudaMemcpyHostToDevice));
    TTC_CUDA(cudaMemcpy(dB.p, Bh, (size_t)n * k * 8, cudaMemcpyHostToDevice));
    run_plan_once(c, [&](Builder& B) {
      CvtDesc ca{dA.as<double>(), a16.p, m, k, k, 1, lda, 1, 1.0};
      CvtDesc cb{dB.as<double>(), b16.p, n, k, k, 1, lda, 1, 1.0};
      B.cvt_bf16({ca, cb});
      Bf16GemmDesc d{};
      d.m = m; d.n = n; d.k = k; d.m0 = std::max(m, 1);
      d.A = a16.p; d.lda = lda; d.B = b16.p; d.ldb = lda;
      d.C64 = dC.as<double>(); d.c_i0 = 1; d.c_i1 = 0; d.c_j = m;
      d.alpha = alpha;
      B.bf16gemm({d});
    });
    TTC_CUDA(cudaMemcpy(C, dC.p, (size_t)m * n * 8, cudaMemcpyDeviceToHost));
  });
}

// tcgen05 TF32 GEMM: as ttc_test_bf16_gemm with the operands converted to FP32 and read by the
// tensor cores as TF32 (kind::tf32).
int ttc_test_tf32_gemm(ttc_context* c, int m, int n, int k, const double* A, const double* Bh, double* C,
                       double alpha) {
  return hook(c, [&] {
    const long long lda = (k + 3) / 4 * 4;
    DevBuf dA((size_t)m * k * 8), dB((size_t)n * k * 8), dC((size_t)m * n * 8);
    DevBuf a32((size_t)m * lda * 4 + 64), b32((size_t)n * lda * 4 + 64);
    TTC_CUDA(cudaMemcpy(dA.p, A, (size_t)m * k * 8, cudaMemcpyHostToDevice));
    TTC_CUDA(cudaMemcpy(dB.p, Bh, (size_t)n * k * 8, cudaMemcpyHostToDevice));
    TTC_CUDA(cudaMemset(a32.p, 0, (size_t)m * lda * 4 + 64));
    TTC_CUDA(cudaMemset(b32.p, 0, (size_t)n * lda * 4 + 64));
    run_plan_once(c, [&](Builder& B) {
      CvtDesc ca{dA.as<double>(), a32.p, m, k, k, 1, lda, 1, 1.0};
      CvtDesc cb{dB.as<double>(), b32.p, n, k, k, 1, lda, 1, 1.0};
      B.cvt_bf16({ca, cb}, true);
      Bf16GemmDesc d{};
      d.m = m; d.n = n; d.k = k; d.m0 = std::max(m, 1);
      d.A = a32.p; d.lda = lda; d.B = b32.p; d.ldb = lda;
      d.C64 = dC.as<double>(); d.c_i0 = 1; d.c_i1 = 0; d.c_j = m;
      d.alpha = alpha;
      B.bf16gemm({d}, true);
    });
    TTC_CUDA(cudaMemcpy(C, dC.p, (size_t)m * n * 8, cudaMemcpyDeviceToHost));
  });
}

}  // extern "C"
