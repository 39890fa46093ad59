// Host-level implementations behind the one-shot C entry points.
#pragma once
#include <functional>
#include <string>
#include <vector>

#include "drivers.cuh"

namespace ttc {

void ensure_stage(ttc_context* c, size_t bytes);
void validate_ttv(const ttc_ttv* x);
// Upload m host TTs into batch slots [first, first+m).  With `reverse`, slot core k holds
// core N-1-k of the host TT with its two rank indices swapped (the mirror-image TT).
void batch_upload_many(ttc_batch* b, int first, int m, const ttc_ttv* xs, bool reverse = false);
void batch_download_many(ttc_batch* b, int first, int m, ttc_ttv_out* ys, bool reverse = false);
ttc_batch* batch_from_host(ttc_context* c, const ttc_ttv* x, const std::vector<int>* cap, bool reverse = false);
void record_stats(ttc_context* c, int nstages);
std::vector<const double*> upload_host_blocks(ttc_context* c, const std::vector<long long>& dims, const SketchPlan& sp,
                                              const double* const* blocks, std::string& key);
std::vector<long long> rks_vec(const int64_t* rks, int N);

// Sets the Jacobi SVD sweep cap of later launches; plans hold the cap, so they are rebuilt.
void set_jacobi_max_sweeps(ttc_context* c, int sweeps);

// Runs a synchronous rounding `run` (which raises the device flags itself); if the Jacobi SVD
// hit its sweep cap (TTC_ENOCONV), runs it once more with four times the cap, as the reference
// retries a failed gesdd with QR iteration (src/tt_rounding.jl:191-195).  `run` must start from
// inputs the first pass did not modify (roundings write a separate output batch).  A second
// failure is reported as TTC_ENOCONV.
template <class F>
void with_svd_retry(ttc_context* c, F&& run) {
  try {
    run();
  } catch (const Error& e) {
    if (e.status != TTC_ENOCONV) throw;
    const int cap0 = c->jacobi_max_sweeps;
    c->stats.svd_retries += 1;
    set_jacobi_max_sweeps(c, cap0 * 4);
    try {
      run();
    } catch (...) {
      set_jacobi_max_sweeps(c, cap0);
      throw;
    }
    set_jacobi_max_sweeps(c, cap0);
  }
}

// A cached device batch of a one-shot entry point: the batch stored under `key`, or a new one
// from `make` (the eight most recently used are kept; older ones are destroyed).
ttc_batch* oneshot_batch(ttc_context* c, const std::string& key, const std::function<ttc_batch*()>& make);
void oneshot_clear(ttc_context* c);

struct BatchHolder {
  std::vector<ttc_batch*> v;
  ~BatchHolder() { for (auto* b : v) batch_destroy(b); }
  ttc_batch* add(ttc_batch* b) { v.push_back(b); return b; }
};

// A TToperator on the device in the internal layout (R_{k-1}, n_out, n_in, R_k), packed.
struct DevTTO {
  int N = 0;
  std::vector<long long> dims;
  std::vector<int> rks;
  std::vector<long long> off;
  double* d = nullptr;
  ~DevTTO();
  double* core(int k) const { return d + off[k]; }
};
DevTTO* tto_upload(ttc_context* c, const ttc_tto* H);

void tt_rounding_host(ttc_context* c, const ttc_ttv* x, const ttc_round_opts& o, ttc_ttv_out* y);
void orthogonalize_host(ttc_context* c, const ttc_ttv* x, int i, ttc_ttv_out* y);
double norm_host(ttc_context* c, const ttc_ttv* x);
void recursive_sketch_host(ttc_context* c, const ttc_ttv* A, const ttc_tto* H, const int64_t* rks,
                           const ttc_sketch_opts& sk, double* const* W_out, int64_t* sketch_rks);
void rand_rounding_host(ttc_context* c, int m, const double* alpha, const ttc_tto* A, const ttc_ttv* ys,
                        const ttc_round_opts* after, const int64_t* rks, const ttc_sketch_opts& sk, ttc_ttv_out* y);
void mpo_apply_host(ttc_context* c, const ttc_tto* A, const ttc_ttv* x, ttc_ttv_out* y);
void hadamard_rounding_host(ttc_context* c, int m, const ttc_ttv* ys, const int64_t* rks, const ttc_sketch_opts& sk,
                            ttc_ttv_out* y);
void stta_host(ttc_context* c, int m, const double* alpha, const ttc_ttv* ys, const int64_t* rks, uint64_t seed_left,
               uint64_t seed_right, int orthogonal, int64_t block_rks, ttc_ttv_out* y);
double dot_host(ttc_context* c, const ttc_ttv* A, const ttc_ttv* B, double* const* W_out, int reverse);
double dot_operator_host(ttc_context* c, const ttc_ttv* psi, const ttc_tto* H, const ttc_ttv* phi);
void tt_add_host(ttc_context* c, const ttc_ttv* x, const ttc_ttv* y, ttc_ttv_out* out);
void tt_scale_host(ttc_context* c, double a, const ttc_ttv* x, ttc_ttv_out* out);
void rayleigh_grad_host(ttc_context* c, const ttc_tto* H, const ttc_ttv* x, int ckpt, double* value,
                        double* const* grads, bool f32 = false);

}  // namespace ttc
