// noalloc.cu -- an allocation-free variant of mat_2_norm.
//
// qd_mat_2_norm reduces through per-CTA partial sums kept in the layout's
// work arena, which the library allocates with cudaMalloc.  Some callers must
// not allocate device memory while they run: for example, a host that reserves
// its whole device-memory budget up front and forbids allocation inside its
// flow loop (cudaMalloc can synchronise the device and fail once a caching
// allocator holds the rest of the memory).  qd_mat_2_norm_noalloc serves them:
// the caller passes the operator and a device scalar for the result, and the
// partial sums live in a fixed static device array.
#include <mutex>

#include "dev_common.cuh"

namespace qd {

constexpr int NA_THREADS = 256;
constexpr i64 NA_MIN_CHUNK = 2048;  // entries per partial sum, at least
constexpr i64 NA_MAX_CHUNK = QD_NOALLOC_MAX_ENTRIES / QD_NOALLOC_MAX_PARTIALS;
static_assert(NA_MAX_CHUNK % NA_THREADS == 0, "chunk must be a multiple of the CTA size");

// Partial sums of the reduction.  Static device memory: every GPU that loads
// this library holds these QD_NOALLOC_MAX_PARTIALS doubles (32 KiB) until the
// process exits.  Every call overwrites them, so calls that overlap on the GPU
// (different streams, or several threads) race on this array.
static __device__ __align__(256) double g_noalloc_partials[QD_NOALLOC_MAX_PARTIALS];

// Partial b = sum of squares of entries [b*chunk, (b+1)*chunk) of x (n total).
__global__ void __launch_bounds__(NA_THREADS) k_na_partial(const double* __restrict__ x, i64 n, i64 chunk,
                                                           double* __restrict__ partials) {
  __shared__ double sh[NA_THREADS / 32];
  const i64 base = (i64)blockIdx.x * chunk;
  const i64 end = min(base + chunk, n);
  double s = 0.0;
  for (i64 i = base + threadIdx.x; i < end; i += NA_THREADS) {
    const double v = x[i];
    s += v * v;
  }
  s = block_sum<NA_THREADS>(s, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// out = sqrt(sum of the np partials), summed in a fixed order.
__global__ void __launch_bounds__(NA_THREADS) k_na_final(const double* __restrict__ partials, int np,
                                                         double* __restrict__ out) {
  __shared__ double sh[NA_THREADS / 32];
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += NA_THREADS) s += partials[i];
  s = block_sum<NA_THREADS>(s, sh);
  if (threadIdx.x == 0) *out = sqrt(s);
}

namespace {
// Device address of g_noalloc_partials, looked up once per device.
std::mutex g_na_mutex;
constexpr int NA_MAX_DEVICES = 64;
double* g_na_ptr[NA_MAX_DEVICES] = {nullptr};

int na_run(const qd_layout* L, const double* d_op, double* d_norm, cudaStream_t s) {
  double* partials;
  {
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[L->device]) {
      // In host code g_noalloc_partials names a host-side stand-in, not a
      // device address; the runtime translates it here, on this device.
      void* p = nullptr;
      QD_CUDA(cudaGetSymbolAddress(&p, g_noalloc_partials));
      g_na_ptr[L->device] = (double*)p;
    }
    partials = g_na_ptr[L->device];
  }
  // every stored one- and two-body entry: [o_fhh, neq) of the vectorize array
  const i64 n = L->neq - L->o_fhh;
  i64 np = (n + NA_MIN_CHUNK - 1) / NA_MIN_CHUNK;
  if (np > QD_NOALLOC_MAX_PARTIALS) np = QD_NOALLOC_MAX_PARTIALS;
  i64 chunk = np > 0 ? (n + np - 1) / np : 0;
  chunk = (chunk + NA_THREADS - 1) / NA_THREADS * NA_THREADS;
  if (np > 0) k_na_partial<<<(unsigned)np, NA_THREADS, 0, s>>>(d_op + L->o_fhh, n, chunk, partials);
  k_na_final<<<1, NA_THREADS, 0, s>>>(partials, (int)np, d_norm);
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}
}  // namespace

}  // namespace qd

extern "C" int qd_mat_2_norm_noalloc(const qd_layout* L, const double* d_op, double* d_norm, void* stream) {
  using namespace qd;
  if (!L || !d_op || !d_norm) {
    set_error("qd_mat_2_norm_noalloc: null argument");
    return QD_ERR_ARG;
  }
  const i64 n = L->neq - L->o_fhh;
  if (n > (i64)QD_NOALLOC_MAX_ENTRIES) {
    set_error("qd_mat_2_norm_noalloc: %lld one- and two-body entries exceed the maximum of %lld (%d partial sums "
              "of at most %lld entries)",
              (long long)n, (long long)QD_NOALLOC_MAX_ENTRIES, QD_NOALLOC_MAX_PARTIALS, (long long)NA_MAX_CHUNK);
    return QD_ERR_ARG;
  }
  if (L->device < 0 || L->device >= NA_MAX_DEVICES) {
    set_error("qd_mat_2_norm_noalloc: layout has no CUDA device (host-only layout)");
    return L->device < 0 ? QD_ERR_STATE : QD_ERR_ARG;
  }
  // run on the layout's device and give the caller's current device back
  int prev = -1;
  QD_CUDA(cudaGetDevice(&prev));
  if (prev != L->device) QD_CUDA(cudaSetDevice(L->device));
  const int rc = na_run(L, d_op, d_norm, stream ? (cudaStream_t)stream : L->stream);
  if (prev != L->device) {
    const cudaError_t e = cudaSetDevice(prev);
    if (rc == QD_OK && e != cudaSuccess) return cuda_fail(e, "cudaSetDevice(restore)");
  }
  return rc;
}
