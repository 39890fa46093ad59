// Operator-aware and environment contractions on the device: the operator sketch
// (src/sketches.jl:1648-1713), rounding of linear combinations and of A y + sum y_j
// (src/tt_randtools.jl:169-354), the MPO apply (src/tt_operations.jl:170-194), dot and
// partial_contraction (src/tt_operations.jl:302-323, src/sketches.jl:1047-1070),
// dot_operator (src/tt_operations.jl:390-421), the direct sum and scaling
// (src/tt_operations.jl:81-112, :428-441), orthogonalize with any root
// (src/tt_rounding.jl:65-97), norm (:107-114) and the Rayleigh-quotient gradient built from
// the ALS environments (src/als.jl:9-25).  All contractions are split-index FP64 GEMMs.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "api_impl.cuh"
#include "regions.cuh"

namespace ttc {

static inline int qr_tws2(int m, int n) { return ((std::min(m, n) + 15) / 16) * 256 + 256; }

// Build, run and drop a plan (for one-shot calls on temporary buffers).
static void run_once(ttc_context* c, const std::function<void(Builder&)>& fn) {
  static unsigned long long serial = 0;
  const std::string key = "once:" + std::to_string(++serial);
  Plan* p = get_plan(c, key, fn);
  run_plan(c, *p);
  TTC_CUDA(cudaStreamSynchronize(c->stream));
  c->plans.erase(key);
  check_device_flags(c);
}

// ---------------------------------------------------------------- TToperator upload
DevTTO::~DevTTO() {
  if (d) { region_remove(d); cudaFree(d); }
}

DevTTO* tto_upload(ttc_context* c, const ttc_tto* H) {
  TTC_REQUIRE(H && H->N > 0 && H->dims && H->rks && H->cores, TTC_EARG, "TToperator: null field");
  std::unique_ptr<DevTTO> D(new DevTTO());
  const int N = H->N;
  D->N = N;
  D->dims.assign(H->dims, H->dims + N);
  D->rks.assign(H->rks, H->rks + N + 1);
  TTC_REQUIRE(D->rks[0] == 1, TTC_EDIM, "TToperator: first rank must be 1");
  D->off.resize(N);
  long long o = 0;
  for (int k = 0; k < N; ++k) {
    TTC_REQUIRE(D->dims[k] > 0 && D->rks[k] > 0 && D->rks[k + 1] > 0 && H->cores[k], TTC_EARG, "TToperator: bad core");
    D->off[k] = o;
    o += (D->rks[k] * D->dims[k] * D->dims[k] * (long long)D->rks[k + 1] + 31) & ~31LL;
  }
  TTC_CUDA(cudaMalloc(&D->d, sizeof(double) * std::max<long long>(o, 1)));
  region_add(D->d, sizeof(double) * std::max<long long>(o, 1));
  ensure_stage(c, sizeof(double) * o + 256 + sizeof(CopyDesc) * N);
  double* hs = (double*)c->h_stage;
  std::vector<CopyDesc> cp;
  long long maxe = 0;
  for (int k = 0; k < N; ++k) {
    const long long n = D->dims[k], R0 = D->rks[k], R1 = D->rks[k + 1];
    const long long cnt = n * n * R0 * R1;
    std::memcpy(hs + D->off[k], H->cores[k], cnt * sizeof(double));
    // Julia (i, j, a, a') at i + n*(j + n*(a + R0*a'))  ->  internal (a, i, j, a') at a + R0*(i + n*(j + n*a'))
    CopyDesc d{};
    d.src = (double*)c->d_stage + D->off[k]; d.dst = D->core(k);
    d.ext[0] = n; d.ext[1] = n; d.ext[2] = R0; d.ext[3] = R1;
    d.ss[0] = 1; d.ss[1] = n; d.ss[2] = n * n; d.ss[3] = n * n * R0;
    d.ds[0] = R0; d.ds[1] = R0 * n; d.ds[2] = 1; d.ds[3] = R0 * n * n;
    d.alpha = 1.0;
    cp.push_back(d);
    maxe = std::max(maxe, cnt);
  }
  const size_t doff = ((size_t)o * sizeof(double) + 255) & ~size_t(255);
  std::memcpy((unsigned char*)c->h_stage + doff, cp.data(), cp.size() * sizeof(CopyDesc));
  TTC_CUDA(cudaMemcpyAsync(c->d_stage, c->h_stage, doff + cp.size() * sizeof(CopyDesc), cudaMemcpyHostToDevice, c->stream));
  launch_copy((const CopyDesc*)((unsigned char*)c->d_stage + doff), N, maxe, c->stream);
  TTC_CUDA(cudaStreamSynchronize(c->stream));
  return D.release();
}

// ---------------------------------------------------------------- operator sketch
// One site of the operator contraction W[a,b,c] = sum A[a,z,al] H[b,ze,z,be] S[ze,ga,c] V[al,be,ga]
// (internal layouts; S given by strides: S(kappa = ze + n*ga, c) at S[kappa*s_k + c*s_c]).
struct OpEnvStep {
  const double* A; int r, xc;        // TT core (r, n, r1) in a slab with left capacity xc
  int r1;
  const double* H; int R, R1;        // MPO core (R, n, n, R1)
  const double* S; long long s_k, s_c; int g, cdim;   // S kappa range n*g, output third dim cdim
  const double* V;                   // (r1, R1, g) packed
  double* W;                         // (r, R, cdim) packed
  int n;
  int batch; long long v_b, s_b, w_b;  // block batching (sketch blocks)
};

static void emit_op_env(Builder& B, const std::vector<OpEnvStep>& steps, bool f32 = false) {
  std::vector<GemmDesc> g1, g2, g3;
  for (const auto& st : steps) {
    const int r = st.r, r1 = st.r1, R = st.R, R1 = st.R1, n = st.n, g = st.g;
    double* T1 = B.wd((size_t)r * n * R1 * g * st.batch);
    double* T2 = B.wd((size_t)r * R * n * g * st.batch);
    // 1. T1[(a,z), (be,ga)] = sum_al A[a,z,al] V[al,(be,ga)]
    GemmDesc d1 = gd(r * n, R1 * g, r1, st.A, 1, (long long)st.xc * n, st.V, 1, r1, T1, 1, (long long)r * n);
    d1.m0 = r; d1.a_i0 = 1; d1.a_i1 = st.xc; d1.c_i0 = 1; d1.c_i1 = r;
    d1.batch = st.batch; d1.b_b = st.v_b; d1.c_b = (long long)r * n * R1 * g;
    g1.push_back(d1);
    // 2. T2[a, b, ze, ga] = sum_{z,be} T1[a,z,be,ga] H[b,ze,z,be]
    GemmDesc d2{};
    d2.m = r * g; d2.n = R * n; d2.k = n * R1; d2.batch = st.batch;
    d2.m0 = r; d2.n0 = R; d2.k0e = n;
    d2.A = T1; d2.a_i0 = 1; d2.a_i1 = (long long)r * n * R1; d2.a_k0 = r; d2.a_k1 = (long long)r * n;
    d2.a_b = (long long)r * n * R1 * g;
    d2.B = st.H; d2.b_k0 = (long long)R * n; d2.b_k1 = (long long)R * n * n; d2.b_j0 = 1; d2.b_j1 = R;
    d2.C = T2; d2.c_i0 = 1; d2.c_i1 = (long long)r * R * n; d2.c_j0 = r; d2.c_j1 = (long long)r * R;
    d2.c_b = (long long)r * R * n * g;
    d2.alpha = 1.0; d2.beta = 0.0;
    g2.push_back(d2);
    // 3. W[(a,b), c] = sum_{(ze,ga)} T2[(a,b),(ze,ga)] S[(ze,ga), c]
    GemmDesc d3 = gd(r * R, st.cdim, n * g, T2, 1, (long long)r * R, st.S, st.s_k, st.s_c, st.W, 1, (long long)r * R);
    d3.batch = st.batch; d3.a_b = (long long)r * R * n * g; d3.b_b = st.s_b; d3.c_b = st.w_b;
    g3.push_back(d3);
  }
  if (f32) {
    B.gemm32(g1);
    B.gemm32(g2);
    B.gemm32(g3);
  } else {
    B.gemm(g1);
    B.gemm(g2);
    B.gemm(g3);
  }
}

void emit_sketch_op_f64(Builder& B, const DevTTO& H, ttc_batch* x, int t, const SketchPlan& sp,
                        const std::vector<double*>& S, std::vector<double*>& W) {
  const int N = x->N;
  W.assign(N + 1, nullptr);
  for (int k = 0; k < N; ++k) W[k] = B.wd((size_t)x->rk(t, k) * H.rks[k] * sp.b[k] * sp.p[k]);
  W[N] = B.ctx->d_one;
  for (int k = N - 1; k >= 0; --k) {
    const size_t mk = B.mark();
    OpEnvStep st{};
    st.A = x->core(t, k); st.r = x->rk(t, k); st.xc = x->capr(t, k); st.r1 = x->rk(t, k + 1);
    st.H = H.core(k); st.R = H.rks[k]; st.R1 = H.rks[k + 1];
    st.n = (int)x->dims[k];
    st.g = sp.b[k + 1]; st.cdim = sp.b[k];
    st.S = S[k]; st.s_k = 1; st.s_c = (long long)st.n * st.g;
    st.V = W[k + 1];
    st.W = W[k];
    st.batch = sp.p[k];
    st.v_b = (k < N - 1) ? (long long)st.r1 * st.R1 * st.g : 0;
    st.s_b = (long long)st.n * st.g * st.cdim;
    st.w_b = (long long)st.r * st.R * st.cdim;
    emit_op_env(B, {st});
    B.release(mk);
  }
}

// The operator sketch on the tcgen05 tensor cores (BF16 operands, or FP32 operands read as
// TF32), FP32 accumulation: per site and block, the three contractions of
// contract_sketch_core_backwards!(W, A, B, S, V) (src/sketches.jl:1648-1713) as three GEMMs,
//   G1  T1[(a,z), (be,ga)] = sum_al A[a,z,al] V[al,(be,ga)]
//   G2  T2[(a,ga), (b,ze)] = sum_{(z,be)} T1[a,z,be,ga] H[b,ze,z,be]
//   G3  W[(a,b), c]        = sum_{(ze,ga)} T2[a,b,ze,ga] S[(ze,ga), c]
// each epilogue writing the next GEMM's K-major operand directly (split row and column strides),
// G3 also W in FP64 (for the FP64 range finder) and the next site's V operand.  Operands are
// zero-padded to 16-byte rows; the TT core, the MPO core and the sketch blocks are converted
// once per call.
// Precision policy (as for the TT sketch): the range finder stays exact under a perturbed sketch
// only where the right interface of H y has full row rank.  Where it is structurally rank
// deficient -- rho_k = min(r_k R_k, n_k rho_{k+1}) < r_k R_k, the bonds near the end whose
// combined rank exceeds the dimension of the right part -- W_k must keep the form R_k X, which
// rounding the operands breaks, so those levels are contracted in FP64 (from the FP64 W_{k+1})
// and only their result is converted for the next tensor-core level.
static inline long long pad_k(long long v, bool tf32) { const long long c = tf32 ? 4 : 8; return (v + c - 1) / c * c; }

void emit_sketch_op_tc(Builder& B, const DevTTO& H, ttc_batch* x, int t, const SketchPlan& sp,
                       const std::vector<double*>& S, std::vector<double*>& W, bool tf32) {
  const int N = x->N;
  const long long esz = tf32 ? 4 : 2;
  W.assign(N + 1, nullptr);
  std::vector<ZeroDesc> zr;
  auto buf = [&](long long elems) -> void* {
    const long long nd = (elems * esz + 7) / 8;
    double* p = B.wd((size_t)nd);
    zr.push_back({p, nd});
    return (void*)p;
  };
  auto at = [&](const void* p, long long elems) -> void* { return (void*)((const char*)p + elems * esz); };
  std::vector<void*> A16(N), H16(N), S16(N), V16(N + 1);
  std::vector<long long> ldv(N + 1);
  std::vector<CvtDesc> cv;
  std::vector<char> f64lvl(N + 1, 0);
  {
    long long rho = 1;
    for (int k = N - 1; k >= 0; --k) {
      const long long full = (long long)x->rk(t, k) * H.rks[k];
      rho = std::min<long long>(full, x->dims[k] * rho);
      f64lvl[k] = rho < full;
    }
  }
  for (int k = 0; k < N; ++k) {
    const long long n = x->dims[k], r = x->rk(t, k), r1 = x->rk(t, k + 1), xc = x->capr(t, k);
    const long long R = H.rks[k], R1 = H.rks[k + 1], g = sp.b[k + 1], cd = sp.b[k], pk = sp.p[k];
    W[k] = B.wd((size_t)(r * R * cd * pk));
    ldv[k] = pad_k(r, tf32);
    V16[k] = (k > 0) ? buf(ldv[k] * R * cd * pk) : nullptr;
    if (f64lvl[k]) continue;       // contracted in FP64: no operand copies
    // A16: row (a + r z), K = al
    const long long lda = pad_k(r1, tf32);
    A16[k] = buf(r * n * lda);
    for (long long z = 0; z < n; ++z) {
      CvtDesc c{};
      c.src = x->core(t, k) + z * xc; c.dst = at(A16[k], r * z * lda);
      c.rows = r; c.cols = r1; c.ss_i = 1; c.ss_j = xc * n; c.ds_i = lda; c.ds_j = 1; c.alpha = 1.0;
      cv.push_back(c);
    }
    // H16: row (b + R ze), K = (z + n be); internal H (b, ze, z, be) at b + R (ze + n (z + n be))
    const long long ldh = pad_k(n * R1, tf32);
    H16[k] = buf(R * n * ldh);
    {
      CvtDesc c{};
      c.src = H.core(k); c.dst = H16[k];
      c.rows = R * n; c.cols = n * R1; c.ss_i = 1; c.ss_j = R * n; c.ds_i = ldh; c.ds_j = 1; c.alpha = 1.0;
      cv.push_back(c);
    }
    // S16: row c, K = (ze + n ga); block j of S at S[k] + j n g cd
    const long long lds = pad_k(n * g, tf32);
    S16[k] = buf(lds * cd * pk);
    for (long long j = 0; j < pk; ++j) {
      CvtDesc c{};
      c.src = S[k] + j * n * g * cd; c.dst = at(S16[k], j * lds * cd);
      c.rows = n * g; c.cols = cd; c.ss_i = 1; c.ss_j = n * g; c.ds_i = 1; c.ds_j = lds; c.alpha = 1.0;
      cv.push_back(c);
    }
  }
  W[N] = B.ctx->d_one;
  ldv[N] = pad_k(1, tf32);
  V16[N] = buf(ldv[N]);
  {
    CvtDesc one{};
    one.src = B.ctx->d_one; one.dst = V16[N];
    one.rows = 1; one.cols = 1; one.ss_i = 0; one.ss_j = 0; one.ds_i = 1; one.ds_j = 1; one.alpha = 1.0;
    cv.push_back(one);
  }
  B.zero(zr);
  B.cvt_bf16(cv, tf32);
  for (int k = N - 1; k >= 0; --k) {
    const size_t mk = B.mark();
    zr.clear();
    std::vector<Bf16GemmDesc> g1, g2, g3;
    const long long n = x->dims[k], r = x->rk(t, k), r1 = x->rk(t, k + 1);
    const long long R = H.rks[k], R1 = H.rks[k + 1], g = sp.b[k + 1], cd = sp.b[k], pk = sp.p[k];
    if (f64lvl[k]) {
      OpEnvStep st{};
      st.A = x->core(t, k); st.r = (int)r; st.xc = x->capr(t, k); st.r1 = (int)r1;
      st.H = H.core(k); st.R = (int)R; st.R1 = (int)R1;
      st.n = (int)n;
      st.g = (int)g; st.cdim = (int)cd;
      st.S = S[k]; st.s_k = 1; st.s_c = n * g;
      st.V = W[k + 1];
      st.W = W[k];
      st.batch = (int)pk;
      st.v_b = (k < N - 1) ? r1 * R1 * g : 0;
      st.s_b = n * g * cd;
      st.w_b = r * R * cd;
      emit_op_env(B, {st});
      if (k > 0) {                                   // the next (tensor-core) level's V operand
        CvtDesc c{};
        c.src = W[k]; c.dst = V16[k];
        c.rows = r; c.cols = R * cd * pk; c.ss_i = 1; c.ss_j = r; c.ds_i = 1; c.ds_j = ldv[k]; c.alpha = 1.0;
        B.cvt_bf16({c}, tf32);
      }
      B.release(mk);
      continue;
    }
    const long long ldt1 = pad_k(n * R1, tf32), ldt2 = pad_k(n * g, tf32), lda = pad_k(r1, tf32);
    const long long lds = pad_k(n * g, tf32), ldh = pad_k(n * R1, tf32);
    for (long long j = 0; j < pk; ++j) {
      void* T1 = buf(r * g * ldt1);
      void* T2 = buf(r * R * ldt2);
      const long long jn = (k < N - 1) ? j : 0;     // W_N is the single constant block
      Bf16GemmDesc d1{};
      d1.m = (int)(r * n); d1.n = (int)(R1 * g); d1.k = (int)r1; d1.m0 = (int)r;
      d1.A = A16[k]; d1.lda = lda;
      d1.B = at(V16[k + 1], jn * ldv[k + 1] * R1 * g); d1.ldb = ldv[k + 1];
      d1.C16 = T1; d1.h_i0 = ldt1; d1.h_i1 = 1;                  // row (a + r ga), K (z + n be)
      d1.n0 = (int)R1; d1.h_j = n; d1.h_j1 = r * ldt1;
      d1.alpha = 1.0;
      g1.push_back(d1);
      Bf16GemmDesc d2{};
      d2.m = (int)(r * g); d2.n = (int)(R * n); d2.k = (int)(n * R1); d2.m0 = (int)r;
      d2.A = T1; d2.lda = ldt1;
      d2.B = H16[k]; d2.ldb = ldh;
      d2.C16 = T2; d2.h_i0 = ldt2; d2.h_i1 = n;                  // row (a + r b), K (ze + n ga)
      d2.n0 = (int)R; d2.h_j = r * ldt2; d2.h_j1 = 1;
      d2.alpha = 1.0;
      g2.push_back(d2);
      Bf16GemmDesc d3{};
      d3.m = (int)(r * R); d3.n = (int)cd; d3.k = (int)(n * g); d3.m0 = (int)r;
      d3.A = T2; d3.lda = ldt2;
      d3.B = at(S16[k], j * lds * cd); d3.ldb = lds;
      d3.C64 = W[k] + j * r * R * cd; d3.c_i0 = 1; d3.c_i1 = r; d3.c_j = r * R;
      if (k > 0) {                                               // next site's V: (a, b, c) at a + ldv (b + R c)
        d3.C16 = at(V16[k], j * ldv[k] * R * cd); d3.h_i0 = 1; d3.h_i1 = ldv[k]; d3.h_j = ldv[k] * R;
      }
      d3.alpha = 1.0;
      g3.push_back(d3);
    }
    B.zero(zr);
    B.bf16gemm(g1, tf32);
    B.bf16gemm(g2, tf32);
    B.bf16gemm(g3, tf32);
    B.release(mk);
  }
}

// ---------------------------------------------------------------- general randomized rounding
// ttrand_rounding(alpha, [A,] ys, rks) (src/tt_randtools.jl:223-354) and the residual form
// A y - b (:169-214, here alpha = [1, -1]).  Term 0 is A*ys[0] when A is given.
void rand_rounding_general(ttc_context* c, int m, const double* alpha, const ttc_tto* Ah, const ttc_ttv* ys,
                           const int64_t* rks, const ttc_sketch_opts& sk, ttc_ttv_out* y) {
  check_precision(sk.precision);
  TTC_REQUIRE(m >= 1, TTC_EARG, "ttrand_rounding: empty combination");
  const int N = ys[0].N;
  for (int j = 0; j < m; ++j) {
    validate_ttv(&ys[j]);
    TTC_REQUIRE(ys[j].N == N, TTC_EDIM, "ttrand_rounding: terms differ in N");
    for (int k = 0; k < N; ++k) TTC_REQUIRE(ys[j].dims[k] == ys[0].dims[k], TTC_EDIM, "ttrand_rounding: terms differ in dims");
  }
  const auto r = rks_vec(rks, N);
  TTC_REQUIRE(r[N] == 1, TTC_EDIM, "ttrand_rounding: rks[N+1] must be 1");
  std::vector<long long> dims(ys[0].dims, ys[0].dims + N);
  const SketchPlan sp = sketch_plan(dims, r, sk.block_rks);
  if (sk.orthogonal)
    for (int k = 0; k < N; ++k)
      TTC_REQUIRE(sp.b[k] <= dims[k] * sp.b[k + 1], TTC_EARG, "generate_sketch_blocks: right_rank > dim*left_rank");
  // all terms in one batch (capacity = their own ranks)
  std::vector<int> cap;
  for (int j = 0; j < m; ++j)
    for (int k = 0; k <= N; ++k) cap.push_back((int)ys[j].rks[k]);
  BatchHolder BH;
  ttc_batch* X = BH.add(batch_create(c, m, N, dims.data(), cap.data()));
  batch_upload_many(X, 0, m, ys, false);
  std::unique_ptr<DevTTO> H;
  if (Ah) {
    H.reset(tto_upload(c, Ah));
    TTC_REQUIRE(H->N == N && H->dims == dims, TTC_EDIM, "ttrand_rounding: operator and TT dims differ");
    TTC_REQUIRE(H->rks[N] == 1, TTC_EDIM, "ttrand_rounding: last operator rank must be 1");
  }
  const std::vector<int> rho = rand_out_ranks(dims, sp);
  ttc_batch* Y = BH.add(batch_create(c, 1, N, dims.data(), rho.data()));
  std::string rawkey;
  const auto raw = upload_host_blocks(c, dims, sp, sk.sketch_blocks, rawkey);
  const bool op = (H != nullptr);
  // q_j[k]: width of term j's projected core at bond k
  auto qdim = [&](int j, int k) { return (op && j == 0) ? X->rk(0, k) * H->rks[k] : X->rk(j, k); };
  run_once(c, [&](Builder& B) {
    B.stage(0);
    emit_zero_tts(B, Y, {0});
    emit_set_ranks(B, Y, {0}, {rho});
    std::vector<double*> S;
    emit_sketch_blocks(B, dims, sp, sk, raw, S);
    std::vector<std::vector<double*>> W(m);
    std::vector<int> tt_terms;
    for (int j = op ? 1 : 0; j < m; ++j) tt_terms.push_back(j);
    if (!tt_terms.empty()) {
      std::vector<std::vector<double*>> Wt;
      if (tensor_core_sketch(sk.precision)) emit_sketch_bf16(B, X, tt_terms, sp, S, Wt, sk.precision == TTC_PREC_TF32);
      else emit_sketch_f64(B, X, tt_terms, sp, S, Wt);
      for (size_t i = 0; i < tt_terms.size(); ++i) W[tt_terms[i]] = Wt[i];
    }
    if (op) {
      if (tensor_core_sketch(sk.precision)) emit_sketch_op_tc(B, *H, X, 0, sp, S, W[0], sk.precision == TTC_PREC_TF32);
      else emit_sketch_op_f64(B, *H, X, 0, sp, S, W[0]);
    }
    B.stage(1);
    // projected cores, ping-pong buffers per term
    std::vector<double*> Yc(m), Yn(m);
    for (int j = 0; j < m; ++j) {
      size_t mx = 1;
      for (int k = 0; k < N; ++k) mx = std::max(mx, (size_t)((long long)rho[k] * dims[k] * qdim(j, k + 1)));
      Yc[j] = B.wd(mx);
      Yn[j] = B.wd(mx);
    }
    {  // k = 0: alpha_j * first cores (term 0 of the operator form: alpha_0 * (A_1 y_1))
      std::vector<GemmDesc> g;
      std::vector<CopyDesc> cp;
      for (int j = 0; j < m; ++j) {
        const int n = (int)dims[0];
        if (op && j == 0) {
          const int r1 = X->rk(0, 1), R1 = H->rks[1];
          GemmDesc d = gd(n, r1, n, H->core(0), 1, n, X->core(0, 0), 1, n, Yc[0], 1, n, alpha[0]);
          d.batch = R1; d.a_b = (long long)n * n; d.b_b = 0; d.c_b = (long long)n * r1;
          g.push_back(d);
        } else {
          cp.push_back(cd2(X->core(j, 0), Yc[j], n, X->rk(j, 1), 1, (long long)n * X->capr(j, 0), 1, n, alpha[j]));
        }
      }
      B.gemm(g);
      B.copy(cp);
    }
    for (int k = 0; k + 1 < N; ++k) {
      const size_t mk = B.mark();
      const int n = (int)dims[k], nn = (int)dims[k + 1];
      const int rh = rho[k], rhn = rho[k + 1], s = sp.s[k + 1];
      const double ws = 1.0 / std::sqrt((double)sp.p[k + 1]);
      double* Z = B.wd((size_t)rh * n * s);
      double* Q = B.wd((size_t)rh * n * rhn);
      double* Tws = B.wd(qr_tws2(rh * n, s));
      for (int j = 0; j < m; ++j) {   // Z = sum_j Y_j W_j[k+1]  (one launch per term: accumulation)
        const int q = qdim(j, k + 1);
        B.gemm({gd(rh * n, s, q, Yc[j], 1, (long long)rh * n, W[j][k + 1], 1, q, Z, 1, (long long)rh * n, ws,
                   j == 0 ? 0.0 : 1.0)});
      }
      B.qr({{rh * n, s, Z, rh * n, Q, rh * n, nullptr, 0, Tws}});
      const int yc = Y->capr(0, k);
      B.copy({cd3(Q, Y->core(0, k), rh, n, rhn, 1, rh, (long long)rh * n, 1, yc, (long long)yc * n)});
      std::vector<GemmDesc> gp, gu, gv;
      std::vector<double*> P(m), U(m);
      for (int j = 0; j < m; ++j) {
        const int q = qdim(j, k + 1);
        P[j] = B.wd((size_t)rhn * q);
        gp.push_back(gd(rhn, q, rh * n, Q, (long long)rh * n, 1, Yc[j], 1, (long long)rh * n, P[j], 1, rhn));
        if (op && j == 0) {
          const int r1 = X->rk(0, k + 1), r2 = X->rk(0, k + 2), R1 = H->rks[k + 1], R2 = H->rks[k + 2];
          const int xc = X->capr(0, k + 1);
          U[0] = B.wd((size_t)rhn * nn * r2 * R1);
          // U[rho', j, a', be] = sum_a P[rho', a, be] y[a, j, a']   (batched over be)
          GemmDesc d = gd(rhn, nn * r2, r1, P[0], 1, rhn, X->core(0, k + 1), 1, xc, U[0], 1, rhn);
          d.batch = R1; d.a_b = (long long)rhn * r1; d.b_b = 0; d.c_b = (long long)rhn * nn * r2;
          gu.push_back(d);
          // Ay'[rho', i', (a' + r2 be')] = sum_{j,be} U[rho', j, a', be] H[be, i', j, be']
          GemmDesc e{};
          e.m = rhn * r2; e.n = nn * R2; e.k = nn * R1; e.batch = 1;
          e.m0 = rhn; e.n0 = nn; e.k0e = nn;
          e.A = U[0]; e.a_i0 = 1; e.a_i1 = (long long)rhn * nn; e.a_k0 = rhn; e.a_k1 = (long long)rhn * nn * r2;
          e.B = H->core(k + 1); e.b_k0 = (long long)R1 * nn; e.b_k1 = 1; e.b_j0 = R1; e.b_j1 = (long long)R1 * nn * nn;
          e.C = Yn[0]; e.c_i0 = 1; e.c_i1 = (long long)rhn * nn; e.c_j0 = rhn; e.c_j1 = (long long)rhn * nn * r2;
          e.alpha = 1.0; e.beta = 0.0;
          gv.push_back(e);
        } else {
          const int r2 = X->rk(j, k + 2);
          gu.push_back(gd(rhn, nn * r2, q, P[j], 1, rhn, X->core(j, k + 1), 1, X->capr(j, k + 1), Yn[j], 1, rhn));
        }
      }
      B.gemm(gp);
      B.gemm(gu);
      B.gemm(gv);
      std::swap(Yc, Yn);
      B.release(mk);
    }
    // last core: sum of the projected terms
    const int rh = rho[N - 1], n = (int)dims[N - 1], yc = Y->capr(0, N - 1);
    for (int j = 0; j < m; ++j) {
      GemmDesc d = gd(rh * n, 1, 1, Yc[j], 1, 0, B.ctx->d_one, 1, 1, Y->core(0, N - 1), 1, 1, 1.0, j == 0 ? 0.0 : 1.0);
      d.m0 = rh; d.a_i0 = 1; d.a_i1 = rh; d.c_i0 = 1; d.c_i1 = yc;
      B.gemm({d});
    }
    B.stage(2);
  });
  for (int k = 0; k < N; ++k) Y->h_ot[k] = (k < N - 1) ? 1 : 0;
  for (int k = 0; k <= N; ++k) Y->h_rks[k] = rho[k];
  Y->rks_dirty = false;
  batch_download_many(Y, 0, 1, y, false);
}

// ---------------------------------------------------------------- MPO apply
void mpo_apply_host(ttc_context* c, const ttc_tto* Ah, const ttc_ttv* x, ttc_ttv_out* y) {
  BatchHolder BH;
  ttc_batch* X = BH.add(batch_from_host(c, x, nullptr));
  std::unique_ptr<DevTTO> H(tto_upload(c, Ah));
  const int N = x->N;
  TTC_REQUIRE(H->N == N && H->dims == X->dims, TTC_EDIM, "Incompatible dimensions");
  std::vector<int> cap(N + 1);
  for (int k = 0; k <= N; ++k) cap[k] = H->rks[k] * X->rk(0, k);
  TTC_REQUIRE(cap[0] == 1 && cap[N] == 1, TTC_EDIM, "apply: boundary ranks of the product must be 1");
  ttc_batch* Y = BH.add(batch_create(c, 1, N, X->dims.data(), cap.data()));
  run_once(c, [&](Builder& B) {
    std::vector<ApplyDesc> v;
    for (int k = 0; k < N; ++k) {
      TTC_REQUIRE(X->capr(0, k) == X->rk(0, k), TTC_EINTERNAL, "apply: packed input expected");
      v.push_back({H->core(k), X->core(0, k), Y->core(0, k), H->rks[k], H->rks[k + 1], X->rk(0, k), X->rk(0, k + 1),
                   (int)X->dims[k]});
    }
    B.apply(v);
  });
  for (int k = 0; k <= N; ++k) Y->h_rks[k] = cap[k];
  for (int k = 0; k < N; ++k) Y->h_ot[k] = 0;
  batch_download_many(Y, 0, 1, y, false);
}

// ---------------------------------------------------------------- dot / partial contraction
double dot_host(ttc_context* c, const ttc_ttv* a, const ttc_ttv* b, double* const* W_out, int reverse) {
  BatchHolder BH;
  ttc_batch* A = BH.add(batch_from_host(c, a, nullptr));
  ttc_batch* Bt = BH.add(batch_from_host(c, b, nullptr));
  const int N = a->N;
  TTC_REQUIRE(b->N == N && A->dims == Bt->dims, TTC_EDIM, "TT dimensions are not compatible");
  std::vector<size_t> off(N + 1);
  size_t tot = 0;
  for (int k = 0; k <= N; ++k) { off[k] = tot; tot += (size_t)A->rk(0, k) * Bt->rk(0, k); }
  ensure_stage(c, tot * sizeof(double) + 256);
  double* Wd = (double*)c->d_stage;
  run_once(c, [&](Builder& B) {
    if (reverse) {
      B.copy({cd2(B.ctx->d_one, Wd + off[N], 1, 1, 0, 0, 0, 0)});
      for (int k = N - 1; k >= 0; --k) {
        const size_t mk = B.mark();
        const int ra = A->rk(0, k), ra1 = A->rk(0, k + 1), rb = Bt->rk(0, k), rb1 = Bt->rk(0, k + 1), n = (int)A->dims[k];
        double* T = B.wd((size_t)ra * n * rb1);
        // T[(a,z), be] = sum_al A[a,z,al] W[al,be]
        B.gemm({gd(ra * n, rb1, ra1, A->core(0, k), 1, (long long)ra * n, Wd + off[k + 1], 1, ra1, T, 1, (long long)ra * n)});
        // W_k[a, b] = sum_{z,be} T[a,(z,be)] B[b,(z,be)]
        B.gemm({gd(ra, rb, n * rb1, T, 1, ra, Bt->core(0, k), rb, 1, Wd + off[k], 1, ra)});
        B.release(mk);
      }
    } else {
      B.copy({cd2(B.ctx->d_one, Wd + off[0], 1, 1, 0, 0, 0, 0)});
      for (int k = 0; k < N; ++k) {
        const size_t mk = B.mark();
        const int ra = A->rk(0, k), ra1 = A->rk(0, k + 1), rb = Bt->rk(0, k), rb1 = Bt->rk(0, k + 1), n = (int)A->dims[k];
        double* T = B.wd((size_t)rb * n * ra1);
        // T[be, (z, a')] = sum_al W[al, be] A[al, (z, a')]
        B.gemm({gd(rb, n * ra1, ra, Wd + off[k], ra, 1, A->core(0, k), 1, ra, T, 1, rb)});
        // W_{k+1}[a', b'] = sum_{(be,z)} T[be, z, a'] B[be, z, b']
        GemmDesc d = gd(ra1, rb1, rb * n, T, (long long)rb * n, 1, Bt->core(0, k), 1, (long long)rb * n, Wd + off[k + 1], 1, ra1);
        B.gemm({d});
        B.release(mk);
      }
    }
  });
  std::vector<double> h(tot);
  TTC_CUDA(cudaMemcpy(h.data(), Wd, tot * sizeof(double), cudaMemcpyDeviceToHost));
  if (W_out)
    for (int k = 0; k <= N; ++k)
      std::memcpy(W_out[k], h.data() + off[k], (size_t)A->rk(0, k) * Bt->rk(0, k) * sizeof(double));
  return reverse ? h[off[0]] : h[off[N]];
}

// ---------------------------------------------------------------- dot_operator
// Right environments E_k[c(phi), b(H), a(psi)] from site N down to 1; <psi|H|phi> = E_0.
static void emit_right_env(Builder& B, ttc_batch* PHI, const DevTTO& H, ttc_batch* PSI, std::vector<double*>& E) {
  const int N = PHI->N;
  E.assign(N + 1, nullptr);
  E[N] = B.ctx->d_one;
  for (int k = N - 1; k >= 0; --k) {
    OpEnvStep st{};
    st.A = PHI->core(0, k); st.r = PHI->rk(0, k); st.xc = PHI->capr(0, k); st.r1 = PHI->rk(0, k + 1);
    st.H = H.core(k); st.R = H.rks[k]; st.R1 = H.rks[k + 1];
    st.n = (int)PHI->dims[k];
    st.g = PSI->rk(0, k + 1); st.cdim = PSI->rk(0, k);
    // psi core (c, ze, ga) at c + capc*(ze + n*ga): S(kappa = ze + n*ga, c)
    st.S = PSI->core(0, k); st.s_k = PSI->capr(0, k); st.s_c = 1;
    st.V = E[k + 1];
    st.batch = 1; st.v_b = 0; st.s_b = 0; st.w_b = 0;
    E[k] = B.wd((size_t)st.r * st.R * st.cdim);
    st.W = E[k];
    const size_t mk2 = B.mark();
    emit_op_env(B, {st});
    B.release(mk2);
  }
}

double dot_operator_host(ttc_context* c, const ttc_ttv* psi, const ttc_tto* Hh, const ttc_ttv* phi) {
  BatchHolder BH;
  ttc_batch* PSI = BH.add(batch_from_host(c, psi, nullptr));
  ttc_batch* PHI = BH.add(batch_from_host(c, phi, nullptr));
  std::unique_ptr<DevTTO> H(tto_upload(c, Hh));
  const int N = psi->N;
  TTC_REQUIRE(phi->N == N && H->N == N && PSI->dims == PHI->dims && H->dims == PSI->dims, TTC_EDIM,
              "dot_operator: dimensions differ");
  double* out = nullptr;
  ensure_stage(c, 256);
  out = (double*)c->d_stage;
  run_once(c, [&](Builder& B) {
    std::vector<double*> E;
    emit_right_env(B, PHI, *H, PSI, E);
    B.copy({cd2(E[0], out, 1, 1, 0, 0, 0, 0)});
  });
  double v = 0;
  TTC_CUDA(cudaMemcpy(&v, out, sizeof(double), cudaMemcpyDeviceToHost));
  return v;
}

// ---------------------------------------------------------------- direct sum and scaling
void tt_add_host(ttc_context* c, const ttc_ttv* x, const ttc_ttv* yv, ttc_ttv_out* out) {
  BatchHolder BH;
  ttc_batch* X = BH.add(batch_from_host(c, x, nullptr));
  ttc_batch* Yb = BH.add(batch_from_host(c, yv, nullptr));
  const int N = x->N;
  TTC_REQUIRE(yv->N == N && X->dims == Yb->dims, TTC_EDIM, "Incompatible dimensions");
  std::vector<int> r(N + 1);
  for (int k = 0; k <= N; ++k) r[k] = X->rk(0, k) + Yb->rk(0, k);
  r[0] = 1;
  r[N] = 1;
  ttc_batch* Z = BH.add(batch_create(c, 1, N, X->dims.data(), r.data()));
  run_once(c, [&](Builder& B) {
    emit_zero_tts(B, Z, {0});
    std::vector<CopyDesc> cp;
    for (int k = 0; k < N; ++k) {
      const long long n = X->dims[k], zc = Z->capr(0, k);
      const int xa = X->rk(0, k), xb = X->rk(0, k + 1), ya = Yb->rk(0, k), yb = Yb->rk(0, k + 1);
      // x block at (0, 0); y block at (xa, xb), except on the boundary bonds (src/tt_operations.jl:97-108)
      const long long ro = (k == 0) ? 0 : xa, co = (k == N - 1) ? 0 : xb;
      cp.push_back(cd3(X->core(0, k), Z->core(0, k), xa, n, xb, 1, xa, (long long)xa * n, 1, zc, zc * n));
      if (N == 1) {
        GemmDesc d = gd(n, 1, 1, Yb->core(0, 0), 1, 0, B.ctx->d_one, 1, 1, Z->core(0, 0), 1, 1, 1.0, 1.0);
        B.gemm({d});
      } else {
        cp.push_back(cd3(Yb->core(0, k), Z->core(0, k) + ro + zc * n * co, ya, n, yb, 1, ya, (long long)ya * n, 1, zc, zc * n));
      }
    }
    B.copy(cp);
  });
  for (int k = 0; k <= N; ++k) Z->h_rks[k] = r[k];
  for (int k = 0; k < N; ++k) Z->h_ot[k] = 0;
  batch_download_many(Z, 0, 1, out, false);
}

void tt_scale_host(ttc_context* c, double a, const ttc_ttv* x, ttc_ttv_out* out) {
  validate_ttv(x);
  const int N = x->N;
  if (a == 0.0) {   // zeros_tt with unit ranks (src/tt_operations.jl:433-434)
    std::vector<int> ones(N + 1, 1);
    std::vector<long long> dims(x->dims, x->dims + N);
    BatchHolder BH;
    ttc_batch* Z = BH.add(batch_create(c, 1, N, dims.data(), ones.data()));
    TTC_CUDA(cudaStreamSynchronize(c->stream));
    for (int k = 0; k < N; ++k) Z->h_ot[k] = 0;
    batch_download_many(Z, 0, 1, out, false);
    return;
  }
  int i = -1;
  for (int k = 0; k < N && x->ot; ++k) if (x->ot[k] == 0) { i = k; break; }
  if (!x->ot) i = 0;
  TTC_REQUIRE(i >= 0, TTC_EARG, "scaling needs a core with ot == 0");
  BatchHolder BH;
  ttc_batch* X = BH.add(batch_from_host(c, x, nullptr));
  ttc_batch* Z = BH.add(batch_from_host(c, x, nullptr));
  run_once(c, [&](Builder& B) {
    const long long cnt = (long long)Z->capr(0, i) * Z->dims[i] * Z->capr(0, i + 1);
    B.copy({cd2(X->core(0, i), Z->core(0, i), cnt, 1, 1, 0, 1, 0, a)});
  });
  batch_download_many(Z, 0, 1, out, false);
}

// ---------------------------------------------------------------- orthogonalize(x; i), norm
static void emit_orth_general(Builder& B, ttc_batch* X, ttc_batch* Y, int root, const std::vector<int>& rp) {
  const int N = X->N;
  const int c0 = root - 1;   // 0-based centre
  // left part: cores 0..c0-1 by QR, FR carried
  double* FR = B.ctx->d_one;
  int frr = 1;
  for (int j = 0; j < c0; ++j) {
    const int n = (int)X->dims[j], a = rp[j], an = rp[j + 1], xr0 = X->rk(0, j), xr1 = X->rk(0, j + 1);
    double* C = B.wd((size_t)a * n * xr1);
    double* Q = B.wd((size_t)a * n * an);
    double* R = B.wd((size_t)an * xr1);
    double* Tws = B.wd(qr_tws2(a * n, xr1));
    B.gemm({gd(a, n * xr1, xr0, FR, 1, frr, X->core(0, j), 1, X->capr(0, j), C, 1, a)});
    B.qr({{a * n, xr1, C, a * n, Q, a * n, R, an, Tws}});
    const int yc = Y->capr(0, j);
    B.copy({cd3(Q, Y->core(0, j), a, n, an, 1, a, (long long)a * n, 1, yc, (long long)yc * n)});
    FR = R; frr = an;
  }
  // right part: cores N-1..c0+1 by LQ, FL carried (FL = L, stored as R^T of the QR of the transpose)
  const double* FLR = B.ctx->d_one;   // R factor whose transpose is FL
  int fl_r = 1;                       // R is (fl_r x xr_{j+1})
  for (int j = N - 1; j > c0; --j) {
    const int n = (int)X->dims[j], xr0 = X->rk(0, j), xr1 = X->rk(0, j + 1), bn = rp[j + 1], b = rp[j];
    // C = core_j * FL : (xr0, n, bn) with FL = R^T (xr1 x bn)
    double* Cm = B.wd((size_t)xr0 * n * bn);
    // FL(al, b') = R(b', al): transposed read of the previous R factor (ld fl_r)
    B.gemm({gd(xr0 * n, bn, xr1, X->core(0, j), 1, (long long)X->capr(0, j) * n, FLR, fl_r, 1, Cm, 1, (long long)xr0 * n)});
    // X = (right unfolding of C)^T : (n*bn) x xr0
    double* Xt = B.wd((size_t)n * bn * xr0);
    B.copy({cd2(Cm, Xt, xr0, (long long)n * bn, 1, xr0, (long long)n * bn, 1)});
    double* Q = B.wd((size_t)n * bn * b);
    double* R = B.wd((size_t)b * xr0);
    double* Tws = B.wd(qr_tws2(n * bn, xr0));
    B.qr({{n * bn, xr0, Xt, n * bn, Q, n * bn, R, b, Tws}});
    // core_j = Q^T : (b, n, bn)
    const int yc = Y->capr(0, j);
    B.copy({cd2(Q, Y->core(0, j), (long long)n * bn, b, 1, (long long)n * bn, yc, 1)});
    FLR = R; fl_r = b;
  }
  // centre: FR * core_c * FL
  const int n = (int)X->dims[c0], xr0 = X->rk(0, c0), xr1 = X->rk(0, c0 + 1), a = rp[c0], bn = rp[c0 + 1];
  double* T = B.wd((size_t)a * n * xr1);
  B.gemm({gd(a, n * xr1, xr0, FR, 1, frr, X->core(0, c0), 1, X->capr(0, c0), T, 1, a)});
  const int yc = Y->capr(0, c0);
  B.gemm({gd(a * n, bn, xr1, T, 1, (long long)a * n, FLR, fl_r, 1, Y->core(0, c0), 1, (long long)yc * n)});
}

static std::vector<int> orth_ranks_general(const ttc_batch* X, int root) {
  const int N = X->N;
  std::vector<int> r(N + 1, 1);
  for (int k = 0; k <= N; ++k) r[k] = X->rk(0, k);
  for (int k = 0; k + 1 < root; ++k) r[k + 1] = (int)std::min<long long>(X->dims[k] * r[k], X->rk(0, k + 1));
  for (int k = N - 1; k >= root; --k) r[k] = (int)std::min<long long>(X->dims[k] * r[k + 1], X->rk(0, k));
  return r;
}

void orthogonalize_host(ttc_context* c, const ttc_ttv* x, int root, ttc_ttv_out* y) {
  const int N = x->N;
  TTC_REQUIRE(root >= 1 && root <= N, TTC_EDIM, "Impossible orthogonalization");
  BatchHolder BH;
  ttc_batch* X = BH.add(batch_from_host(c, x, nullptr));
  const std::vector<int> rp = orth_ranks_general(X, root);
  ttc_batch* Y = BH.add(batch_create(c, 1, N, X->dims.data(), rp.data()));
  run_once(c, [&](Builder& B) {
    emit_zero_tts(B, Y, {0});
    emit_orth_general(B, X, Y, root, rp);
  });
  for (int k = 0; k <= N; ++k) Y->h_rks[k] = rp[k];
  for (int k = 0; k < N; ++k) Y->h_ot[k] = (k < root - 1) ? 1 : (k == root - 1 ? 0 : -1);
  batch_download_many(Y, 0, 1, y, false);
}

double norm_host(ttc_context* c, const ttc_ttv* x) {
  validate_ttv(x);
  const int N = x->N;
  int centre = -1, zeros = 0;
  for (int k = 0; k < N; ++k)
    if ((x->ot ? x->ot[k] : 0) == 0) { ++zeros; if (centre < 0) centre = k; }
  BatchHolder BH;
  ttc_batch* X = BH.add(batch_from_host(c, x, nullptr));
  ttc_batch* Src = X;
  int core = centre;
  if (zeros != 1) {
    const std::vector<int> rp = orth_ranks_general(X, N);
    ttc_batch* Y = BH.add(batch_create(c, 1, N, X->dims.data(), rp.data()));
    run_once(c, [&](Builder& B) {
      emit_zero_tts(B, Y, {0});
      emit_orth_general(B, X, Y, N, rp);
    });
    Src = Y;
    core = N - 1;
  }
  ensure_stage(c, 256);
  double* out = (double*)c->d_stage;
  run_once(c, [&](Builder& B) {
    B.sumsq({{Src->core(0, core), (long long)Src->capr(0, core) * Src->dims[core] * Src->capr(0, core + 1), out}});
  });
  double v = 0;
  TTC_CUDA(cudaMemcpy(&v, out, sizeof(double), cudaMemcpyDeviceToHost));
  return std::sqrt(v);
}

// ---------------------------------------------------------------- Rayleigh-quotient gradient
// Environments (bra = ket = x): left L_k[a(bra), b(H), c(ket)] over sites < k and right
// R_k[d, e, f] over sites >= k; norm environments Ln_k[a, c], Rn_k[d, f].  The gradient of
// R(x) = <x|H|x>/<x|x> at core k is (2/<x,x>) (Heff_k x_k - R Neff_k x_k) with
//   (Heff_k x_k)[a, i, d] = sum L_k[a,b,c] H_k[b,i,j,e] x_k[c,j,f] R_{k+1}[d,e,f].
// Left environments are stored only every `ckpt` sites and recomputed segment by segment.
void rayleigh_grad_host(ttc_context* c, const ttc_tto* Hh, const ttc_ttv* x, int ckpt, double* value,
                        double* const* grads, bool f32) {
  BatchHolder BH;
  ttc_batch* X = BH.add(batch_from_host(c, x, nullptr));
  std::unique_ptr<DevTTO> H(tto_upload(c, Hh));
  const int N = x->N;
  TTC_REQUIRE(H->N == N && H->dims == X->dims, TTC_EDIM, "rayleigh_grad: dimensions differ");
  TTC_REQUIRE(H->rks[N] == 1, TTC_EDIM, "rayleigh_grad: last operator rank must be 1");
  if (ckpt <= 0) ckpt = 1;
  // FP32 variant: float copies of the TT and MPO cores (same element offsets), every contraction
  // on the FP32 grouped GEMM, environments and gradient in float, widened for the host
  const size_t esz = f32 ? sizeof(float) : sizeof(double);
  float* Xf = nullptr;
  float* Hf = nullptr;
  std::vector<double*> own;
  struct FreeV { std::vector<double*>& v; ~FreeV() { for (auto* p : v) { region_remove(p); cudaFree(p); } } } fv{own};
  auto dev_alloc = [&](size_t bytes) {
    double* p = nullptr;
    TTC_CUDA(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
    own.push_back(p);
    region_add(p, std::max<size_t>(bytes, 16));
    return p;
  };
  if (f32) {
    size_t ht = 0;
    for (int k = 0; k < N; ++k)
      ht = std::max<size_t>(ht, (size_t)H->off[k] + (size_t)H->rks[k] * H->dims[k] * H->dims[k] * H->rks[k + 1]);
    Xf = reinterpret_cast<float*>(dev_alloc(sizeof(float) * (size_t)X->total));
    Hf = reinterpret_cast<float*>(dev_alloc(sizeof(float) * ht));
    run_once(c, [&](Builder& B) {
      CvtDesc a{}, h{};
      a.src = X->d_cores; a.dst = Xf; a.rows = X->total; a.cols = 1; a.ss_i = 1; a.ds_i = 1; a.alpha = 1.0;
      h.src = H->d; h.dst = Hf; h.rows = (long long)ht; h.cols = 1; h.ss_i = 1; h.ds_i = 1; h.alpha = 1.0;
      B.cvt_f32({a, h});
    });
  }
  auto xcore = [&](int k) -> double* {
    return f32 ? reinterpret_cast<double*>(Xf + X->off[k]) : X->core(0, k);
  };
  auto hcore = [&](int k) -> double* {
    return f32 ? reinterpret_cast<double*>(Hf + H->off[k]) : H->core(k);
  };
  auto GEMM = [&](Builder& B, std::vector<GemmDesc> v) {
    if (f32) B.gemm32(std::move(v));
    else B.gemm(std::move(v));
  };
  // 1.0 into the first element of a buffer of this precision
  auto set_one = [&](Builder& B, double* dst) {
    if (f32) {
      CvtDesc o1{};
      o1.src = B.ctx->d_one; o1.dst = dst; o1.rows = 1; o1.cols = 1; o1.ss_i = 1; o1.ds_i = 1; o1.alpha = 1.0;
      B.cvt_f32({o1});
    } else {
      B.copy({cd2(B.ctx->d_one, dst, 1, 1, 0, 0, 0, 0)});
    }
  };
  auto rk = [&](int k) { return X->rk(0, k); };
  auto Rk = [&](int k) { return H->rks[k]; };
  // device buffers (outside the plan workspace): checkpoints, segment cache, right envs, grads
  std::vector<size_t> hsz(N + 1), nsz(N + 1);
  for (int k = 0; k <= N; ++k) { hsz[k] = (size_t)rk(k) * Rk(k) * rk(k); nsz[k] = (size_t)rk(k) * rk(k); }
  size_t gsz = 0;
  std::vector<size_t> goff(N);
  for (int k = 0; k < N; ++k) { goff[k] = gsz; gsz += (size_t)rk(k) * X->dims[k] * rk(k + 1); }
  double* dG = dev_alloc(esz * gsz);                  // gradient (this precision), offsets goff
  double* dval = dev_alloc(sizeof(double) * 4);       // [<x|H|x>, <x|x>] in FP64
  auto gcore = [&](int k) -> double* {
    return f32 ? reinterpret_cast<double*>(reinterpret_cast<float*>(dG) + goff[k]) : dG + goff[k];
  };
  // pass 1: left environments with checkpoints, value
  std::vector<double*> Lh_ck(N + 1, nullptr), Ln_ck(N + 1, nullptr);
  for (int k = 0; k <= N; k += ckpt) {
    Lh_ck[k] = dev_alloc(esz * hsz[k]);
    Ln_ck[k] = dev_alloc(esz * nsz[k]);
  }
  // left env step k -> k+1 (bra = ket = x):  L'[a',b',c'] = sum L[a,b,c] x[a,i,a'] H[b,i,j,b'] x[c,j,c']
  // computed as the right-env contraction of the mirrored indices: W[c',b',a'] with A = x (ket), S = x (bra).
  auto emit_left_step = [&](Builder& B, int k, const double* Lh, const double* Ln, double* Lh1, double* Ln1) {
    const int r0 = rk(k), r1 = rk(k + 1), R0 = Rk(k), R1 = Rk(k + 1), n = (int)X->dims[k];
    const int xc = X->capr(0, k);
    // T1[(a, b), (j, c')] = sum_c L[a,b,c] x[c, j, c']   (L as ((a,b) x c))
    double* T1 = B.wd((size_t)r0 * R0 * n * r1);
    GEMM(B, {gd(r0 * R0, n * r1, r0, Lh, 1, (long long)r0 * R0, xcore(k), 1, xc, T1, 1, (long long)r0 * R0)});
    double* T2 = B.wd((size_t)r0 * n * r1 * R1);
    // T2[(a, c'), (i, b')] = sum_{(b,j)} T1[a, b, j, c'] H[b, i, j, b']   (stored (a, i, c', b'))
    GemmDesc f{};
    f.m = r0 * r1; f.n = n * R1; f.k = R0 * n; f.batch = 1;
    f.m0 = r0; f.n0 = n; f.k0e = R0;
    f.A = T1; f.a_i0 = 1; f.a_i1 = (long long)r0 * R0 * n; f.a_k0 = r0; f.a_k1 = (long long)r0 * R0;
    f.B = hcore(k); f.b_k0 = 1; f.b_k1 = (long long)R0 * n; f.b_j0 = R0; f.b_j1 = (long long)R0 * n * n;
    // T2[(a, i), (c', b')] layout (a, i, c', b'): a -> 1, c' -> r0*n, i -> r0, b' -> r0*n*r1
    f.C = T2; f.c_i0 = 1; f.c_i1 = (long long)r0 * n; f.c_j0 = r0; f.c_j1 = (long long)r0 * n * r1;
    f.alpha = 1.0; f.beta = 0.0;
    GEMM(B, {f});
    // L'[a', (b', c')] = sum_{(a, i)} x[a, i, a'] T2[(a, i), (c', b')]  -> stored (a', b', c')
    GemmDesc h{};
    h.m = r1; h.n = r1 * R1; h.k = r0 * n; h.batch = 1;
    h.m0 = r1; h.n0 = r1; h.k0e = r0;
    h.A = xcore(k); h.a_i0 = (long long)xc * n; h.a_i1 = 0; h.a_k0 = 1; h.a_k1 = xc;
    h.B = T2; h.b_k0 = 1; h.b_k1 = r0; h.b_j0 = (long long)r0 * n; h.b_j1 = (long long)r0 * n * r1;
    h.C = Lh1; h.c_i0 = 1; h.c_i1 = 0; h.c_j0 = (long long)r1 * R1; h.c_j1 = r1;
    h.alpha = 1.0; h.beta = 0.0;
    GEMM(B, {h});
    // norm env: Ln'[a', c'] = sum x[a,i,a'] (sum_c Ln[a,c] x[c,i,c'])
    double* U = B.wd((size_t)r0 * n * r1);
    GEMM(B, {gd(r0, n * r1, r0, Ln, 1, r0, xcore(k), 1, xc, U, 1, r0)});
    GemmDesc q{};
    q.m = r1; q.n = r1; q.k = r0 * n; q.batch = 1;
    q.m0 = r1; q.n0 = r1; q.k0e = r0;
    q.A = xcore(k); q.a_i0 = (long long)xc * n; q.a_i1 = 0; q.a_k0 = 1; q.a_k1 = xc;
    q.B = U; q.b_k0 = 1; q.b_k1 = r0; q.b_j0 = (long long)r0 * n; q.b_j1 = 0;
    q.C = Ln1; q.c_i0 = 1; q.c_i1 = 0; q.c_j0 = r1; q.c_j1 = 0;
    q.alpha = 1.0; q.beta = 0.0;
    GEMM(B, {q});
  };
  run_once(c, [&](Builder& B) {
    set_one(B, Lh_ck[0]);
    set_one(B, Ln_ck[0]);
    double* curH = Lh_ck[0];
    double* curN = Ln_ck[0];
    for (int k = 0; k < N; ++k) {
      double* nh; double* nn;
      if ((k + 1) % ckpt == 0 || k + 1 == N) {
        if (Lh_ck[k + 1] == nullptr) { nh = B.wd(hsz[k + 1]); nn = B.wd(nsz[k + 1]); }
        else { nh = Lh_ck[k + 1]; nn = Ln_ck[k + 1]; }
      } else {
        nh = B.wd(hsz[k + 1]); nn = B.wd(nsz[k + 1]);
      }
      emit_left_step(B, k, curH, curN, nh, nn);
      curH = nh; curN = nn;
    }
    if (f32) {
      CvtDesc w1{}, w2{};
      w1.src = curH; w1.dst = dval; w1.rows = 1; w1.cols = 1; w1.ss_i = 1; w1.ds_i = 1; w1.alpha = 1.0;
      w2 = w1; w2.src = curN; w2.dst = dval + 1;
      B.widen({w1, w2});
    } else {
      B.copy({cd2(curH, dval, 1, 1, 0, 0, 0, 0), cd2(curN, dval + 1, 1, 1, 0, 0, 0, 0)});
    }
  });
  double hv[2];
  TTC_CUDA(cudaMemcpy(hv, dval, sizeof(hv), cudaMemcpyDeviceToHost));
  const double e = hv[0], nn = hv[1];
  TTC_REQUIRE(nn > 0.0, TTC_EARG, "rayleigh_grad: <x|x> is zero");
  const double Rq = e / nn;
  *value = Rq;
  // pass 2: right-to-left, recomputing each segment's left environments from its checkpoint
  run_once(c, [&](Builder& B) {
    double* Rh = B.wd(1); double* Rn = B.wd(1);
    set_one(B, Rh);
    set_one(B, Rn);
    int seg_lo = -1;
    std::vector<double*> segH(N + 1, nullptr), segN(N + 1, nullptr);
    for (int k = N - 1; k >= 0; --k) {
      if (seg_lo < 0 || k < seg_lo) {   // enter the segment holding k: recompute its left envs
        seg_lo = (k / ckpt) * ckpt;
        std::fill(segH.begin(), segH.end(), nullptr);
        std::fill(segN.begin(), segN.end(), nullptr);
        segH[seg_lo] = Lh_ck[seg_lo]; segN[seg_lo] = Ln_ck[seg_lo];
        for (int q = seg_lo; q < k; ++q) {
          segH[q + 1] = B.wd(hsz[q + 1]); segN[q + 1] = B.wd(nsz[q + 1]);
          emit_left_step(B, q, segH[q], segN[q], segH[q + 1], segN[q + 1]);
        }
      }
      const int r0 = rk(k), r1 = rk(k + 1), R0 = Rk(k), R1 = Rk(k + 1), n = (int)X->dims[k];
      const int xc = X->capr(0, k);
      const double* Lh = segH[k];
      const double* Ln = segN[k];
      double* G = gcore(k);
      // Heff x: U[(c, j), (d, e)] = sum_f x[c,j,f] R[d,e,f]
      double* U = B.wd((size_t)r0 * n * r1 * R1);
      // right environments are stored (ket f, H e, bra d): R[f + r1*e + r1*R1*d]
      GemmDesc u = gd(r0 * n, r1 * R1, r1, xcore(k), 1, (long long)xc * n, Rh, 1, (long long)r1 * R1, U, 1, (long long)r0 * n);
      u.m0 = r0; u.a_i0 = 1; u.a_i1 = xc; u.c_i0 = 1; u.c_i1 = r0;
      u.n0 = r1; u.b_j0 = (long long)r1 * R1; u.b_j1 = r1;
      u.c_j0 = (long long)r0 * n; u.c_j1 = (long long)r0 * n * r1;   // U layout (c, j, d, e)
      GEMM(B, {u});
      // V[(b, c), (i, d)] = sum_{(j, e)} U[c, j, d, e] H[b, i, j, e]   (U layout (c, j, d, e))
      double* V = B.wd((size_t)R0 * r0 * n * r1);
      GemmDesc w{};
      w.m = r0 * r1; w.n = R0 * n; w.k = n * R1; w.batch = 1;
      w.m0 = r0; w.n0 = R0; w.k0e = n;
      w.A = U; w.a_i0 = 1; w.a_i1 = (long long)r0 * n; w.a_k0 = r0; w.a_k1 = (long long)r0 * n * r1;
      w.B = hcore(k); w.b_k0 = (long long)R0 * n; w.b_k1 = (long long)R0 * n * n; w.b_j0 = 1; w.b_j1 = R0;
      // V layout (b, c, i, d): b -> 1, c -> R0, i -> R0*r0, d -> R0*r0*n
      w.C = V; w.c_i0 = R0; w.c_i1 = (long long)R0 * r0 * n; w.c_j0 = 1; w.c_j1 = (long long)R0 * r0;
      w.alpha = 1.0; w.beta = 0.0;
      GEMM(B, {w});
      // G[a, (i, d)] = (2/nn) sum_{(b, c)} L[a, b, c] V[(b, c), (i, d)]
      GEMM(B, {gd(r0, n * r1, R0 * r0, Lh, 1, r0, V, 1, (long long)R0 * r0, G, 1, r0, 2.0 / nn)});
      // Neff x: T[(c, i), d] = sum_f x[c,i,f] Rn[d,f]; G -= (2R/nn) Ln[a,c] T[c,(i,d)]
      double* T = B.wd((size_t)r0 * n * r1);
      GemmDesc t = gd(r0 * n, r1, r1, xcore(k), 1, (long long)xc * n, Rn, r1, 1, T, 1, (long long)r0 * n);
      t.m0 = r0; t.a_i0 = 1; t.a_i1 = xc; t.c_i0 = 1; t.c_i1 = r0;
      GEMM(B, {t});
      GEMM(B, {gd(r0, n * r1, r0, Ln, 1, r0, T, 1, r0, G, 1, r0, -2.0 * Rq / nn, 1.0)});
      // right environments at k: R_k[d0, e0, f0] = sum x[d0,i,d] H[e0,i,j,e] x[f0,j,f] R[d,e,f]
      double* Rh_new = B.wd((size_t)r0 * R0 * r0);
      double* Rn_new = B.wd((size_t)r0 * r0);
      OpEnvStep st{};
      st.A = xcore(k); st.r = r0; st.xc = xc; st.r1 = r1;
      st.H = hcore(k); st.R = R0; st.R1 = R1; st.n = n;
      st.g = r1; st.cdim = r0;
      st.S = xcore(k); st.s_k = xc; st.s_c = 1;
      st.V = Rh; st.W = Rh_new; st.batch = 1; st.v_b = st.s_b = st.w_b = 0;
      // stored (ket, H, bra), the layout the U contraction above reads
      emit_op_env(B, {st}, f32);
      double* Tn = B.wd((size_t)r0 * n * r1);
      GemmDesc a1 = gd(r0 * n, r1, r1, xcore(k), 1, (long long)xc * n, Rn, 1, r1, Tn, 1, (long long)r0 * n);
      a1.m0 = r0; a1.a_i0 = 1; a1.a_i1 = xc; a1.c_i0 = 1; a1.c_i1 = r0;
      GEMM(B, {a1});
      GEMM(B, {gd(r0, r0, n * r1, Tn, 1, r0, xcore(k), xc, 1, Rn_new, 1, r0)});
      Rh = Rh_new; Rn = Rn_new;
    }
  });
  std::vector<double> hg(gsz);
  if (f32) {
    std::vector<float> hf(gsz);
    TTC_CUDA(cudaMemcpy(hf.data(), dG, gsz * sizeof(float), cudaMemcpyDeviceToHost));
    for (size_t e = 0; e < gsz; ++e) hg[e] = hf[e];
  } else {
    TTC_CUDA(cudaMemcpy(hg.data(), dG, gsz * sizeof(double), cudaMemcpyDeviceToHost));
  }
  // internal (a, i, d) -> Julia (i, a, d)
  for (int k = 0; k < N; ++k) {
    const int r0 = rk(k), r1 = rk(k + 1), n = (int)X->dims[k];
    const double* src = hg.data() + goff[k];
    double* dst = grads[k];
    for (int d = 0; d < r1; ++d)
      for (int a = 0; a < r0; ++a)
        for (int i = 0; i < n; ++i) dst[i + (size_t)n * (a + (size_t)r0 * d)] = src[a + (size_t)r0 * (i + (size_t)n * d)];
  }
}

}  // namespace ttc
