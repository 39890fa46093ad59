// Allocation-free Householder QR of one matrix already in device memory.
//
// Some callers cannot allocate device memory at the moment they need a factorisation: code
// that runs inside a memory pool or arena that owns the whole device budget (a Julia
// CUDA.jl pool, a solver that reserved its memory up front), or code in a context where a
// cudaMalloc would be illegal or would stall other streams.  The context-based entry points
// of this library allocate (workspace, plans, staging buffers), so this one does not: the
// working copy of A, the block-reflector factors, the kernel descriptor and the status word
// live in one file-scope device array, g_qr_scratch, of fixed size (about 4.1 MiB, held by
// every GPU that loads the library until the process exits).
//
// Limits: 1 <= m <= 1536 (the QR kernel's row limit), m * n <= 524288, min(m, n) <= 512.
// Larger problems are rejected with TTC_EDIM before anything is launched.
//
// Every call on a device shares the array and leaves its contents behind; each call
// rewrites the parts it uses (the working copy, the descriptor) and zeroes the status word
// before the factorisation runs.  Calls whose work overlaps on the GPU (different streams,
// or different host threads on the same device) race on the array and must be serialised
// by the caller.  The first call on a device resolves the array's device address
// (cudaGetSymbolAddress) once and caches it; that first call should come before any CUDA
// stream capture is begun on the device.
#include <mutex>

#include "ttcuda.h"
#include "kernels.cuh"

namespace ttc {
void set_noctx_error(const std::string& msg);   // capi.cu: message of ttc_last_error(NULL)
}

namespace {
constexpr long long QRNA_MAX_ELEMS = 1LL << 19;            // m * n of the working copy
constexpr int QRNA_MAX_K = 512;                             // min(m, n)
constexpr long long QRNA_TWS = (QRNA_MAX_K / 16) * 256;     // T factors: 16 x 16 per panel
constexpr long long QRNA_DESC = QRNA_MAX_ELEMS + QRNA_TWS;  // offset of the descriptor (doubles)
constexpr long long QRNA_FLAG = QRNA_DESC + 32;             // offset of the status word (doubles)
constexpr long long QRNA_TOTAL = QRNA_FLAG + 32;
static_assert(sizeof(ttc::QRDesc) <= 32 * sizeof(double), "descriptor slot too small");

static __device__ __align__(256) double g_qr_scratch[QRNA_TOTAL];

constexpr int QRNA_MAX_DEVICES = 64;
std::mutex g_mu;
double* g_addr[QRNA_MAX_DEVICES] = {nullptr};

// Device address of g_qr_scratch on the current device (resolved once per device).
double* scratch_address(int dev) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_qr_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw ttc::Error(TTC_ECUDA, std::string("ttc_qr_noalloc: cudaGetSymbolAddress failed: ") +
                                      cudaGetErrorString(e));
    }
    g_addr[dev] = static_cast<double*>(p);
  }
  return g_addr[dev];
}

// Writes the descriptor (passed by value as a kernel parameter, so no host-to-device copy is
// needed) and zeroes the status word the QR kernel ORs its flags into.
__global__ void qrna_prepare(ttc::QRDesc d, ttc::QRDesc* dst, int* status) {
  if (threadIdx.x == 0) {
    *dst = d;
    *status = 0;
  }
}
}  // namespace

extern "C" int ttc_qr_noalloc(int32_t m, int32_t n, const double* A, int64_t lda, double* Q, int64_t ldq,
                              double* R, int64_t ldr, int32_t* status, void* stream) {
  try {
    const long long K = (m < n) ? m : n;
    if (m < 1 || n < 1 || !A) throw ttc::Error(TTC_EARG, "ttc_qr_noalloc: m, n >= 1 and A are required");
    if (m > ttc::QR_MAX_M || (long long)m * n > QRNA_MAX_ELEMS || K > QRNA_MAX_K)
      throw ttc::Error(TTC_EDIM, "ttc_qr_noalloc: matrix exceeds the fixed scratch (m <= 1536, m*n <= 524288, "
                                 "min(m,n) <= 512)");
    if (lda < m || (Q && ldq < m) || (R && ldr < K))
      throw ttc::Error(TTC_EARG, "ttc_qr_noalloc: leading dimensions too small");
    // the kernel descriptor holds 32-bit leading dimensions
    if (lda > INT32_MAX || (Q && ldq > INT32_MAX) || (R && ldr > INT32_MAX))
      throw ttc::Error(TTC_EARG, "ttc_qr_noalloc: leading dimensions above 2^31 - 1");
    int dev = 0;
    TTC_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= QRNA_MAX_DEVICES) throw ttc::Error(TTC_EARG, "ttc_qr_noalloc: device index out of range");
    double* base = scratch_address(dev);
    double* work = base;
    double* tws = base + QRNA_MAX_ELEMS;
    ttc::QRDesc* ddesc = reinterpret_cast<ttc::QRDesc*>(base + QRNA_DESC);
    int* flag = status ? reinterpret_cast<int*>(status) : reinterpret_cast<int*>(base + QRNA_FLAG);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // working copy (the kernel overwrites its input with the Householder vectors)
    TTC_CUDA(cudaMemcpy2DAsync(work, (size_t)m * sizeof(double), A, (size_t)lda * sizeof(double),
                               (size_t)m * sizeof(double), (size_t)n, cudaMemcpyDeviceToDevice, s));
    ttc::QRDesc d{m, n, work, m, Q, (int)ldq, R, (int)ldr, tws};
    qrna_prepare<<<1, 32, 0, s>>>(d, ddesc, flag);
    TTC_CHECK_LAUNCH();
    ttc::launch_qr(ddesc, 1, m, s, flag);
    return TTC_OK;
  } catch (const ttc::Error& e) {
    ttc::set_noctx_error(e.what());
    return e.status;
  } catch (const std::exception& e) {
    ttc::set_noctx_error(e.what());
    return TTC_EINTERNAL;
  }
}
