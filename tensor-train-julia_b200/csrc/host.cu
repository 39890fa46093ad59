// One-shot host entry points (the methods a Julia ccall binds): they stage the host
// tensors into temporary device batches, run the batch drivers and copy results back.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "api_impl.cuh"

namespace ttc {

static std::vector<long long> dims_of(const ttc_ttv* x) { return std::vector<long long>(x->dims, x->dims + x->N); }

// tt_rounding(x; tol, rmax, direction), src/tt_rounding.jl:146-154.  direction=:right is
// the mirror image of direction=:left: reversing the core order and swapping the two rank
// indices of every core turns right-orthogonalisation (LQ) into left-orthogonalisation (QR)
// and the left-to-right SVD sweep into the right-to-left one, so the same device sweep
// serves both and the result is mirrored back on download.
void tt_rounding_host(ttc_context* c, const ttc_ttv* x, const ttc_round_opts& o, ttc_ttv_out* y) {
  TTC_REQUIRE(o.direction == TTC_DIR_LEFT || o.direction == TTC_DIR_RIGHT, TTC_EARG,
              "Invalid direction. Use direction=:right or direction=:left");
  const bool rev = (o.direction == TTC_DIR_RIGHT);
  validate_ttv(x);
  const int N = x->N;
  // the call's device batches are cached by shape: a repeated call uploads into the same memory
  // and replays its captured plan
  std::string shape = ":" + std::to_string(N) + (rev ? "r" : "l");
  for (int k = 0; k < N; ++k) shape += "," + std::to_string(x->dims[k]);
  for (int k = 0; k <= N; ++k) shape += "," + std::to_string(x->rks[k]);
  ttc_batch* xb = oneshot_batch(c, "round.x" + shape, [&] {
    std::vector<long long> dims(N);
    for (int k = 0; k < N; ++k) dims[k] = x->dims[rev ? N - 1 - k : k];
    std::vector<int> cp(N + 1);
    for (int k = 0; k <= N; ++k) cp[k] = (int)x->rks[rev ? N - k : k];
    return batch_create(c, 1, N, dims.data(), cp.data());
  });
  batch_upload_many(xb, 0, 1, x, rev);
  std::vector<int> cap(N + 1);
  if (is_left_orth(xb, 0)) for (int k = 0; k <= N; ++k) cap[k] = xb->rk(0, k);
  else cap = orth_left_ranks(xb, 0);
  std::string cs = shape;
  for (int v : cap) cs += "," + std::to_string(v);
  ttc_batch* yb = oneshot_batch(c, "round.y" + cs, [&] { return batch_create(c, 1, N, xb->dims.data(), cap.data()); });
  ttc_round_opts lo = o;
  lo.direction = TTC_DIR_LEFT;
  with_svd_retry(c, [&] {
    round_det(c, xb, lo, yb);
    record_stats(c, 3);
    check_device_flags(c);
  });
  batch_download_many(yb, 0, 1, y, rev);
}

// ttrand_rounding and its linear-combination / operator variants (src/tt_randtools.jl:112-354).
// m == 1 and A == null is the single-TT rounding; the others are handled by
// rand_rounding_general (contractions.cu).
void rand_rounding_general(ttc_context* c, int m, const double* alpha, const ttc_tto* A, const ttc_ttv* ys,
                           const int64_t* rks, const ttc_sketch_opts& sk, ttc_ttv_out* y);

void rand_rounding_host(ttc_context* c, int m, const double* alpha, const ttc_tto* A, const ttc_ttv* ys,
                        const ttc_round_opts* after, const int64_t* rks, const ttc_sketch_opts& sk, ttc_ttv_out* y) {
  if (m != 1 || A != nullptr || alpha[0] != 1.0) {
    TTC_REQUIRE(after == nullptr, TTC_EARG, "rounding of combinations returns the sketched TT only");
    rand_rounding_general(c, m, alpha, A, ys, rks, sk, y);
    return;
  }
  BatchHolder H;
  ttc_batch* xb = H.add(batch_from_host(c, ys, nullptr));
  const int N = ys->N;
  const auto r = rks_vec(rks, N);
  const SketchPlan sp = sketch_plan(xb->dims, r, sk.block_rks);
  const std::vector<int> cap = rand_out_ranks(xb->dims, sp);
  ttc_batch* yb = H.add(batch_create(c, 1, N, xb->dims.data(), cap.data()));
  check_precision(sk.precision);
  std::string key;
  const auto raw = upload_host_blocks(c, xb->dims, sp, sk.sketch_blocks, key);
  with_svd_retry(c, [&] {
    round_rand(c, xb, r, sk, after, yb, raw, key);
    record_stats(c, 4);
    check_device_flags(c);
  });
  batch_download_many(yb, 0, 1, y, false);
}

// tt_recursive_sketch (src/sketches.jl:175-305 / :317-461), reverse=true.  W_out[k] receives
// W[k] / sqrt(p_k) as (r_k, s_k) (TT) or (r_k, R_k, s_k) (operator) column-major.
void emit_sketch_op_f64(Builder& B, const DevTTO& H, ttc_batch* x, int t, const SketchPlan& sp,
                        const std::vector<double*>& S, std::vector<double*>& W);
void emit_sketch_op_tc(Builder& B, const DevTTO& H, ttc_batch* x, int t, const SketchPlan& sp,
                       const std::vector<double*>& S, std::vector<double*>& W, bool tf32);

void recursive_sketch_host(ttc_context* c, const ttc_ttv* Ah, const ttc_tto* Hh, const int64_t* rks,
                           const ttc_sketch_opts& sk, double* const* W_out, int64_t* sketch_rks) {
  BatchHolder BH;
  ttc_batch* xb = BH.add(batch_from_host(c, Ah, nullptr));
  const int N = Ah->N;
  const auto r = rks_vec(rks, N);
  TTC_REQUIRE(r[N] == 1, TTC_EDIM, "tt_recursive_sketch: rks[N+1] must be 1 for reverse=true");
  const SketchPlan sp = sketch_plan(xb->dims, r, sk.block_rks);
  if (sk.orthogonal)
    for (int k = 0; k < N; ++k)
      TTC_REQUIRE(sp.b[k] <= xb->dims[k] * sp.b[k + 1], TTC_EARG, "generate_sketch_blocks: right_rank > dim*left_rank");
  std::unique_ptr<DevTTO> H;
  if (Hh) {
    H.reset(tto_upload(c, Hh));
    TTC_REQUIRE(H->N == N && H->dims == xb->dims, TTC_EDIM, "tt_recursive_sketch: operator and TT dims differ");
    TTC_REQUIRE(H->rks[N] == 1, TTC_EDIM, "tt_recursive_sketch: last operator rank must be 1");
  }
  check_precision(sk.precision);
  std::string key;
  const auto raw = upload_host_blocks(c, xb->dims, sp, sk.sketch_blocks, key);
  // output sizes
  std::vector<size_t> osz(N + 1), ooff(N + 1);
  size_t tot = 0;
  for (int k = 0; k <= N; ++k) {
    const size_t rr = (size_t)xb->rk(0, k) * (H ? H->rks[k] : 1);
    osz[k] = rr * sp.s[k];
    ooff[k] = tot;
    tot += osz[k];
  }
  ensure_stage(c, tot * sizeof(double) + 256);
  double* dst = (double*)c->d_stage;
  Plan* p = get_plan(c, "sketch:" + std::string(H ? "op" : "tt") + key + batch_key(xb) + std::to_string((uintptr_t)H.get()) +
                            ":" + std::to_string((uintptr_t)dst) + ":" +
                            std::to_string(sk.seed) + ":" + std::to_string(sk.orthogonal) + std::to_string(sk.precision),
                     [&](Builder& B) {
    B.stage(0);
    std::vector<double*> S;
    emit_sketch_blocks(B, xb->dims, sp, sk, raw, S);
    std::vector<double*> Wk;
    if (H) {
      if (tensor_core_sketch(sk.precision)) emit_sketch_op_tc(B, *H, xb, 0, sp, S, Wk, sk.precision == TTC_PREC_TF32);
      else emit_sketch_op_f64(B, *H, xb, 0, sp, S, Wk);
    } else {
      std::vector<std::vector<double*>> W;
      if (tensor_core_sketch(sk.precision)) emit_sketch_bf16(B, xb, {0}, sp, S, W, sk.precision == TTC_PREC_TF32);
      else emit_sketch_f64(B, xb, {0}, sp, S, W);
      Wk = W[0];
    }
    std::vector<CopyDesc> cp;
    for (int k = 0; k <= N; ++k)
      cp.push_back(cd2(Wk[k], dst + ooff[k], (long long)osz[k], 1, 1, 0, 1, 0, 1.0 / std::sqrt((double)sp.p[k])));
    B.copy(cp);
    B.stage(1);
  });
  run_plan(c, *p);
  TTC_CUDA(cudaStreamSynchronize(c->stream));
  check_device_flags(c);
  for (int k = 0; k <= N; ++k) {
    TTC_CUDA(cudaMemcpy(W_out[k], dst + ooff[k], osz[k] * sizeof(double), cudaMemcpyDeviceToHost));
    sketch_rks[k] = sp.s[k];
  }
}

}  // namespace ttc
