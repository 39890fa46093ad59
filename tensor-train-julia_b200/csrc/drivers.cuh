// Sweep drivers shared by the C ABI (rounding.cu, sketch_bf16.cu, contractions.cu).
#pragma once
#include <string>
#include <vector>

#include "builder.cuh"

namespace ttc {

// Block structure of the reverse recursive sketch (src/sketches.jl:186-198):
// b = block ranks, p = block counts, s = b .* p (the returned sketch_rks).
struct SketchPlan {
  std::vector<int> b, p, s;
};
SketchPlan sketch_plan(const std::vector<long long>& dims, const std::vector<long long>& rks, long long block_rks);

void emit_zero_tts(Builder& B, ttc_batch* y, const std::vector<int>& tts);
void emit_set_ranks(Builder& B, ttc_batch* y, const std::vector<int>& tts, const std::vector<std::vector<int>>& r);
void emit_copy_tts(Builder& B, ttc_batch* x, ttc_batch* y, const std::vector<int>& tts,
                   const std::vector<std::vector<int>>& r);
void emit_orth_left(Builder& B, ttc_batch* x, ttc_batch* y, const std::vector<int>& tts,
                    const std::vector<std::vector<int>>& rp);
void emit_svd_left(Builder& B, ttc_batch* y, const std::vector<int>& tts, const std::vector<std::vector<int>>& rp,
                   double tol, long long rmax);
void emit_zero_check(Builder& B, ttc_batch* y, const std::vector<int>& tts, int core, double tol);
void emit_finalize(Builder& B, ttc_batch* y, const std::vector<int>& tts, const std::vector<std::vector<int>>& rp);
// Shape of the sketch blocks of one site: p blocks of (left, n, right) in the Julia layout.
struct BlockShape {
  int left, n, right, p;
};
void emit_block_draws(Builder& B, const std::vector<BlockShape>& sh, const ttc_sketch_opts& o, std::vector<double*>& raw);
void emit_sketch_blocks(Builder& B, const std::vector<long long>& dims, const SketchPlan& sp, const ttc_sketch_opts& o,
                        const std::vector<const double*>& host_raw, std::vector<double*>& S);
void emit_sketch_f64(Builder& B, ttc_batch* x, const std::vector<int>& tts, const SketchPlan& sp,
                     const std::vector<double*>& S, std::vector<std::vector<double*>>& W);
// Sketch contractions on the tcgen05 tensor cores: BF16 operands, or FP32 operands read as
// TF32 (tf32 = true); FP32 accumulation either way.
void emit_sketch_bf16(Builder& B, ttc_batch* x, const std::vector<int>& tts, const SketchPlan& sp,
                      const std::vector<double*>& S, std::vector<std::vector<double*>>& W, bool tf32 = false);
// Rejects a sketch precision other than TTC_PREC_FP64, TTC_PREC_BF16 and TTC_PREC_TF32.
inline void check_precision(int p) {
  TTC_REQUIRE(p == TTC_PREC_FP64 || p == TTC_PREC_BF16 || p == TTC_PREC_TF32, TTC_EARG,
              "sketch precision must be TTC_PREC_FP64, TTC_PREC_BF16 or TTC_PREC_TF32");
}
inline bool tensor_core_sketch(int p) { return p == TTC_PREC_BF16 || p == TTC_PREC_TF32; }
// `complete`: write the completion columns of rank-deficient range finders (false when a truncated-SVD
// sweep follows in the same plan, which also selects the reduced forms that need only range(Q));
// `eff` (optional) receives the effective ranks the cores are nonzero within.  W may hold null
// pointers when `complete` is false and sketch_compresses() is false.
void emit_rand_sweep(Builder& B, ttc_batch* x, ttc_batch* y, const std::vector<int>& tts, const SketchPlan& sp,
                     const std::vector<std::vector<double*>>& W, const std::vector<std::vector<int>>& rho,
                     bool complete = true, std::vector<std::vector<int>>* eff = nullptr);
bool sketch_compresses(const ttc_batch* x, const std::vector<int>& tts, const SketchPlan& sp);
std::vector<int> orth_left_ranks(const ttc_batch* x, int t);
std::vector<int> rand_out_ranks(const std::vector<long long>& dims, const SketchPlan& sp);
bool is_left_orth(const ttc_batch* x, int t);

void round_det(ttc_context* c, ttc_batch* x, const ttc_round_opts& o, ttc_batch* y);
void round_rand(ttc_context* c, ttc_batch* x, const std::vector<long long>& rks, const ttc_sketch_opts& o,
                const ttc_round_opts* after, ttc_batch* y, const std::vector<const double*>& host_raw,
                const std::string& raw_key);

}  // namespace ttc
