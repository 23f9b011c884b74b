// mlp.cu -- the per-element network of the learned warm start:
//   16 -> 256 -> 256 -> 1, GELU (erf form) after the two hidden layers,
//   FP32 master weights, BF16 copies of the 256 x 256 layer and of the
//   activations that feed it, FP32 accumulation everywhere.
// Training: mean squared error, full backward pass, Adam.  Every kernel is
// written here: the 256-wide products run on the tensor cores
// (mma.sync.m16n8k16 bf16 -> f32, NT layout: both operands K-contiguous),
// the 16-wide first layer, the 1-wide last layer, the batch reductions of the
// gradients (fixed order, deterministic) and Adam on CUDA cores.
//
// Parameters (one FP32 vector, QD_MLP_NPARAM entries): W1 [256][16], b1 [256],
// W2 [256][256], b2 [256], w3 [256], b3 [1]; W[out][in].
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "dev_common.cuh"

typedef __nv_bfloat16 bf16;

namespace qd {
namespace {

constexpr int NI = 16, NH = 256;
constexpr i64 O_W1 = 0, O_B1 = O_W1 + NH * NI, O_W2 = O_B1 + NH, O_B2 = O_W2 + NH * NH, O_W3 = O_B2 + NH,
              O_B3 = O_W3 + NH, NPARAM = O_B3 + 1;
constexpr int RED_CHUNKS = 64;  // row chunks of the batch reductions

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// ---- C[M][N] (+= over split-K slices into partial buffers) = A[M][K] B[N][K]^T
constexpr int GBM = 64, GBN = 64, GBK = 32, GLD = GBK + 8;

__device__ __forceinline__ void mma_bf16(float* d, const unsigned* a, const unsigned* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// K and kchunk multiples of GBK; lda, ldb multiples of 8 (16-byte rows).
// Slice z = blockIdx.z covers k in [z*kchunk, min(K, (z+1)*kchunk)) and
// writes C + z * cstride.
__global__ void __launch_bounds__(128) k_gemm_nt_bf16(const bf16* __restrict__ A, int lda, const bf16* __restrict__ B,
                                                      int ldb, float* __restrict__ C, int ldc, i64 cstride, int M,
                                                      int N, int K, int kchunk) {
  __shared__ __align__(16) bf16 As[GBM][GLD];
  __shared__ __align__(16) bf16 Bs[GBN][GLD];
  const int m0 = blockIdx.y * GBM, n0 = blockIdx.x * GBN;
  const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
  C += (i64)blockIdx.z * cstride;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = warp >> 1, g = lane >> 2, t = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;
  for (int k0 = kb; k0 < ke; k0 += GBK) {
#pragma unroll
    for (int it = 0; it < 2; ++it) {  // 64 rows x 4 vectors of 8 per operand
      const int v = tid + it * 128, r = v >> 2, seg = (v & 3) * 8;
      uint4 va = make_uint4(0, 0, 0, 0), vb = make_uint4(0, 0, 0, 0);
      if (m0 + r < M) va = *reinterpret_cast<const uint4*>(A + (i64)(m0 + r) * lda + k0 + seg);
      if (n0 + r < N) vb = *reinterpret_cast<const uint4*>(B + (i64)(n0 + r) * ldb + k0 + seg);
      *reinterpret_cast<uint4*>(&As[r][seg]) = va;
      *reinterpret_cast<uint4*>(&Bs[r][seg]) = vb;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GBK; kk += 16) {
      unsigned af[2][4], bfr[4][2];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) {
        const int rb = wm * 32 + mi * 16;
        af[mi][0] = *reinterpret_cast<const unsigned*>(&As[rb + g][kk + 2 * t]);
        af[mi][1] = *reinterpret_cast<const unsigned*>(&As[rb + g + 8][kk + 2 * t]);
        af[mi][2] = *reinterpret_cast<const unsigned*>(&As[rb + g][kk + 2 * t + 8]);
        af[mi][3] = *reinterpret_cast<const unsigned*>(&As[rb + g + 8][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int ni = 0; ni < 4; ++ni) {
        const int cb = wn * 32 + ni * 8;
        bfr[ni][0] = *reinterpret_cast<const unsigned*>(&Bs[cb + g][kk + 2 * t]);
        bfr[ni][1] = *reinterpret_cast<const unsigned*>(&Bs[cb + g][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni) mma_bf16(acc[mi][ni], af[mi], bfr[ni]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int ni = 0; ni < 4; ++ni) {
      const int r0 = m0 + wm * 32 + mi * 16 + g, c = n0 + wn * 32 + ni * 8 + 2 * t;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = r0 + 8 * h;
        if (r >= M) continue;
        if (c < N) C[(i64)r * ldc + c] = acc[mi][ni][2 * h];
        if (c + 1 < N) C[(i64)r * ldc + c + 1] = acc[mi][ni][2 * h + 1];
      }
    }
}

// out[i] = sum over the nz slices of part[z][i], fixed order
__global__ void k_sum_slices(const float* __restrict__ part, int nz, i64 n, float* __restrict__ out) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int z = 0; z < nz; ++z) s += part[(i64)z * n + i];
  out[i] = s;
}

// ---- layer 1: Z1 = X W1^T + b1, H1 = GELU(Z1) -> bf16 row-major (and transposed)
__global__ void k_layer1(const float* __restrict__ X, const float* __restrict__ P, float* __restrict__ Z1,
                         bf16* __restrict__ H1, bf16* __restrict__ H1t, i64 n) {
  const i64 i = blockIdx.x;
  const int j = threadIdx.x;  // NH threads
  if (i >= n) return;
  __shared__ float x[NI];
  if (j < NI) x[j] = X[i * NI + j];
  __syncthreads();
  float z = P[O_B1 + j];
  const float* w = P + O_W1 + j * NI;
#pragma unroll
  for (int c = 0; c < NI; ++c) z += x[c] * w[c];
  if (Z1) Z1[i * NH + j] = z;
  const bf16 h = __float2bfloat16_rn(gelu(z));
  H1[i * NH + j] = h;
  if (H1t) H1t[(i64)j * n + i] = h;
}

// ---- layer 2 epilogue and layer 3: Z2 += b2, H2 = GELU(Z2), y = H2 w3 + b3 (warp per row)
__global__ void k_layer23(float* __restrict__ Z2, const float* __restrict__ P, float* __restrict__ y, i64 n) {
  const i64 i = (i64)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  float s = 0.f;
  for (int j = lane; j < NH; j += 32) {
    const float z = Z2[i * NH + j] + P[O_B2 + j];
    Z2[i * NH + j] = z;
    s += gelu(z) * P[O_W3 + j];
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) y[i] = s + P[O_B3];
}

// ---- backward
// dy = 2 (y - t) / n; per-chunk partial sums of (y - t)^2
__global__ void k_loss(const float* __restrict__ y, const float* __restrict__ tg, float* __restrict__ dy, i64 n,
                       float* __restrict__ lpart) {
  __shared__ double sh[8];
  double s = 0.0;
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
    const float d = y[i] - tg[i];
    dy[i] = 2.0f * d / (float)n;
    s += (double)d * d;
  }
  s = block_sum<256>(s, sh);
  if (threadIdx.x == 0) lpart[blockIdx.x] = (float)s;
}

// dZ2 = dy (x) w3 * GELU'(Z2), bf16, row-major and transposed
__global__ void k_dz2(const float* __restrict__ dy, const float* __restrict__ Z2, const float* __restrict__ P,
                      bf16* __restrict__ dZ2, bf16* __restrict__ dZ2t, i64 n) {
  const i64 i = blockIdx.x;
  const int j = threadIdx.x;
  if (i >= n) return;
  const bf16 v = __float2bfloat16_rn(dy[i] * P[O_W3 + j] * gelu_d(Z2[i * NH + j]));
  dZ2[i * NH + j] = v;
  dZ2t[(i64)j * n + i] = v;
}

// per row chunk: db2[j] += dy_i w3_j g'(Z2_ij); dw3[j] += dy_i GELU(Z2_ij); db3 += dy_i
__global__ void k_red23(const float* __restrict__ dy, const float* __restrict__ Z2, const float* __restrict__ P,
                        i64 n, float* __restrict__ part) {
  const int j = threadIdx.x;
  const i64 r0 = n * blockIdx.x / gridDim.x, r1 = n * (blockIdx.x + 1) / gridDim.x;
  float db2 = 0.f, dw3 = 0.f, db3 = 0.f;
  const float w3 = P[O_W3 + j];
  for (i64 i = r0; i < r1; ++i) {
    const float z = Z2[i * NH + j], d = dy[i];
    db2 += d * w3 * gelu_d(z);
    dw3 += d * gelu(z);
    db3 += d;
  }
  float* o = part + (i64)blockIdx.x * (2 * NH + 1);
  o[j] = db2;
  o[NH + j] = dw3;
  if (j == 0) o[2 * NH] = db3;
}

// per row chunk: dZ1 = dH1 * GELU'(Z1); db1[j] += dZ1_ij; dW1[j][c] += dZ1_ij X_ic
__global__ void k_red1(const float* __restrict__ dH1, const float* __restrict__ Z1, const float* __restrict__ X, i64 n,
                       float* __restrict__ part) {
  const int j = threadIdx.x;
  const i64 r0 = n * blockIdx.x / gridDim.x, r1 = n * (blockIdx.x + 1) / gridDim.x;
  float db1 = 0.f, dw[NI];
#pragma unroll
  for (int c = 0; c < NI; ++c) dw[c] = 0.f;
  __shared__ float xs[NI];
  for (i64 i = r0; i < r1; ++i) {
    __syncthreads();
    if (j < NI) xs[j] = X[i * NI + j];
    __syncthreads();
    const float d = dH1[i * NH + j] * gelu_d(Z1[i * NH + j]);
    db1 += d;
#pragma unroll
    for (int c = 0; c < NI; ++c) dw[c] += d * xs[c];
  }
  float* o = part + (i64)blockIdx.x * (NH + NH * NI);
  o[j] = db1;
#pragma unroll
  for (int c = 0; c < NI; ++c) o[NH + j * NI + c] = dw[c];
}

// gradient vector G from the chunk partials (fixed order) and the dW2 product
__global__ void k_grad_collect(const float* __restrict__ p23, const float* __restrict__ p1, int nch,
                               const float* __restrict__ dW2, float* __restrict__ G) {
  const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= NPARAM) return;
  float s = 0.f;
  if (e < O_B1) {  // W1[j][c]
    for (int z = 0; z < nch; ++z) s += p1[(i64)z * (NH + NH * NI) + NH + e];
  } else if (e < O_W2) {  // b1
    for (int z = 0; z < nch; ++z) s += p1[(i64)z * (NH + NH * NI) + (e - O_B1)];
  } else if (e < O_B2) {  // W2[j][l] = dW2[j][l]
    s = dW2[e - O_W2];
  } else if (e < O_W3) {  // b2
    for (int z = 0; z < nch; ++z) s += p23[(i64)z * (2 * NH + 1) + (e - O_B2)];
  } else if (e < O_B3) {  // w3
    for (int z = 0; z < nch; ++z) s += p23[(i64)z * (2 * NH + 1) + NH + (e - O_W3)];
  } else {
    for (int z = 0; z < nch; ++z) s += p23[(i64)z * (2 * NH + 1) + 2 * NH];
  }
  G[e] = s;
}

__global__ void k_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ M,
                       float* __restrict__ V, float lr, float c1, float c2) {
  const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= NPARAM) return;
  const float g = G[e];
  const float m = 0.9f * M[e] + 0.1f * g, v = 0.999f * V[e] + 0.001f * g * g;
  M[e] = m;
  V[e] = v;
  P[e] -= lr * (m / c1) / (sqrtf(v / c2) + 1e-8f);
}

// bf16 copies of W2 (row-major [out][in]) and its transpose
__global__ void k_w2_bf16(const float* __restrict__ P, bf16* __restrict__ W2b, bf16* __restrict__ W2tb) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= NH * NH) return;
  const int j = e / NH, l = e % NH;
  const bf16 v = __float2bfloat16_rn(P[O_W2 + e]);
  W2b[e] = v;
  W2tb[(i64)l * NH + j] = v;
}

}  // namespace
}  // namespace qd

struct qd_mlp {
  int device = 0;
  float *P = nullptr, *M = nullptr, *V = nullptr, *G = nullptr;
  bf16 *W2b = nullptr, *W2tb = nullptr;
  long long step = 0;
  // activations for up to cap rows
  qd::i64 cap = 0;
  float *Z1 = nullptr, *Z2 = nullptr, *y = nullptr, *dy = nullptr, *dH1 = nullptr;
  bf16 *H1 = nullptr, *H1t = nullptr, *dZ2 = nullptr, *dZ2t = nullptr;
  float *p23 = nullptr, *p1 = nullptr, *lpart = nullptr, *dW2 = nullptr, *kpart = nullptr;
  int kslices = 0;
};

using namespace qd;

namespace {
void mlp_free_acts(qd_mlp* m) {
  for (void* p : {(void*)m->Z1, (void*)m->Z2, (void*)m->y, (void*)m->dy, (void*)m->dH1, (void*)m->H1, (void*)m->H1t,
                  (void*)m->dZ2, (void*)m->dZ2t, (void*)m->kpart})
    if (p) cudaFree(p);
  m->Z1 = m->Z2 = m->y = m->dy = m->dH1 = m->kpart = nullptr;
  m->H1 = m->H1t = m->dZ2 = m->dZ2t = nullptr;
  m->cap = 0;
}

int mlp_ensure(qd_mlp* m, i64 n) {
  if (n <= m->cap) return QD_OK;
  mlp_free_acts(m);
  const i64 c = ((n + 1023) / 1024) * 1024;
  QD_CUDA(cudaMalloc(&m->Z1, sizeof(float) * c * NH));
  QD_CUDA(cudaMalloc(&m->Z2, sizeof(float) * c * NH));
  QD_CUDA(cudaMalloc(&m->dH1, sizeof(float) * c * NH));
  QD_CUDA(cudaMalloc(&m->y, sizeof(float) * c));
  QD_CUDA(cudaMalloc(&m->dy, sizeof(float) * c));
  QD_CUDA(cudaMalloc(&m->H1, sizeof(bf16) * c * NH));
  QD_CUDA(cudaMalloc(&m->H1t, sizeof(bf16) * c * NH));
  QD_CUDA(cudaMalloc(&m->dZ2, sizeof(bf16) * c * NH));
  QD_CUDA(cudaMalloc(&m->dZ2t, sizeof(bf16) * c * NH));
  m->kslices = (int)std::max<i64>(1, std::min<i64>(64, c / 512));
  QD_CUDA(cudaMalloc(&m->kpart, sizeof(float) * (size_t)m->kslices * NH * NH));
  m->cap = c;
  return QD_OK;
}

int gemm_nt(const bf16* A, int lda, const bf16* B, int ldb, float* C, int ldc, int M, int N, int K, int slices,
            float* part, cudaStream_t st) {
  if (K % GBK) {
    set_error("mlp: inner dimension %d is not a multiple of %d", K, GBK);
    return QD_ERR_ARG;
  }
  int kchunk = ((K + slices - 1) / slices + GBK - 1) / GBK * GBK;
  slices = (K + kchunk - 1) / kchunk;
  dim3 grid((N + GBN - 1) / GBN, (M + GBM - 1) / GBM, slices);
  if (slices == 1) {
    k_gemm_nt_bf16<<<grid, 128, 0, st>>>(A, lda, B, ldb, C, ldc, 0, M, N, K, kchunk);
  } else {
    k_gemm_nt_bf16<<<grid, 128, 0, st>>>(A, lda, B, ldb, part, ldc, (i64)M * ldc, M, N, K, kchunk);
    const i64 nn = (i64)M * ldc;
    k_sum_slices<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(part, slices, nn, C);
  }
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// forward of rows [0, n) of X into m->y (keeps Z1, H1, H1t, Z2 when train)
int mlp_forward(qd_mlp* m, const float* X, i64 n, bool train, cudaStream_t st) {
  int rc = mlp_ensure(m, n);
  if (rc) return rc;
  k_layer1<<<(unsigned)n, NH, 0, st>>>(X, m->P, train ? m->Z1 : nullptr, m->H1, train ? m->H1t : nullptr, n);
  if ((rc = gemm_nt(m->H1, NH, m->W2b, NH, m->Z2, NH, (int)n, NH, NH, 1, nullptr, st))) return rc;
  k_layer23<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(m->Z2, m->P, m->y, n);
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

// gradient of mean((y - t)^2) into m->G; loss into *loss (host) if given
int mlp_grad(qd_mlp* m, const float* X, const float* T, i64 n, float* loss, cudaStream_t st) {
  if (n <= 0 || n % GBK) {
    set_error("qd_mlp: the batch (%lld rows) must be a positive multiple of %d", (long long)n, GBK);
    return QD_ERR_ARG;
  }
  int rc = mlp_forward(m, X, n, true, st);
  if (rc) return rc;
  k_loss<<<RED_CHUNKS, 256, 0, st>>>(m->y, T, m->dy, n, m->lpart);
  k_dz2<<<(unsigned)n, NH, 0, st>>>(m->dy, m->Z2, m->P, m->dZ2, m->dZ2t, n);
  k_red23<<<RED_CHUNKS, NH, 0, st>>>(m->dy, m->Z2, m->P, n, m->p23);
  // dW2[j][l] = sum_i dZ2[i][j] H1[i][l]: A = dZ2^T (256 x n), B = H1^T (256 x n), K = n
  if ((rc = gemm_nt(m->dZ2t, (int)n, m->H1t, (int)n, m->dW2, NH, NH, NH, (int)n, m->kslices, m->kpart, st)))
    return rc;
  // dH1 = dZ2 W2: A = dZ2 (n x 256), B = W2^T (256 x 256)
  if ((rc = gemm_nt(m->dZ2, NH, m->W2tb, NH, m->dH1, NH, (int)n, NH, NH, 1, nullptr, st))) return rc;
  k_red1<<<RED_CHUNKS, NH, 0, st>>>(m->dH1, m->Z1, X, n, m->p1);
  k_grad_collect<<<(unsigned)((NPARAM + 255) / 256), 256, 0, st>>>(m->p23, m->p1, RED_CHUNKS, m->dW2, m->G);
  QD_CUDA(cudaGetLastError());
  if (loss) {
    float lp[RED_CHUNKS];
    QD_CUDA(cudaMemcpyAsync(lp, m->lpart, sizeof(lp), cudaMemcpyDeviceToHost, st));
    QD_CUDA(cudaStreamSynchronize(st));
    double s = 0.0;
    for (int z = 0; z < RED_CHUNKS; ++z) s += lp[z];
    *loss = (float)(s / (double)n);
  }
  return QD_OK;
}
}  // namespace

extern "C" {

int qd_mlp_create(int device, uint64_t seed, qd_mlp** out) {
  if (!out) {
    set_error("qd_mlp_create: null output");
    return QD_ERR_ARG;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_error("qd_mlp_create: no CUDA device");
    return QD_ERR_NODEVICE;
  }
  qd_mlp* m = new qd_mlp();
  if (device < 0)
    cudaGetDevice(&m->device);
  else
    m->device = device;
  QD_CUDA(cudaSetDevice(m->device));
  // He-style initialisation, fixed seed
  std::vector<float> p(NPARAM, 0.f);
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  for (i64 e = O_W1; e < O_B1; ++e) p[e] = nd(rng) * std::sqrt(2.0f / NI);
  for (i64 e = O_W2; e < O_B2; ++e) p[e] = nd(rng) * std::sqrt(2.0f / NH);
  for (i64 e = O_W3; e < O_B3; ++e) p[e] = nd(rng) * std::sqrt(1.0f / NH);
  int rc = QD_OK;
  auto al = [&](void** ptr, size_t b) {
    if (!rc && cudaMalloc(ptr, b) != cudaSuccess) rc = cuda_fail(cudaErrorMemoryAllocation, "qd_mlp_create");
  };
  al((void**)&m->P, sizeof(float) * NPARAM);
  al((void**)&m->M, sizeof(float) * NPARAM);
  al((void**)&m->V, sizeof(float) * NPARAM);
  al((void**)&m->G, sizeof(float) * NPARAM);
  al((void**)&m->W2b, sizeof(bf16) * NH * NH);
  al((void**)&m->W2tb, sizeof(bf16) * NH * NH);
  al((void**)&m->p23, sizeof(float) * RED_CHUNKS * (2 * NH + 1));
  al((void**)&m->p1, sizeof(float) * RED_CHUNKS * (NH + NH * NI));
  al((void**)&m->lpart, sizeof(float) * RED_CHUNKS);
  al((void**)&m->dW2, sizeof(float) * NH * NH);
  if (rc) {
    delete m;
    return rc;
  }
  QD_CUDA(cudaMemcpy(m->P, p.data(), sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
  QD_CUDA(cudaMemset(m->M, 0, sizeof(float) * NPARAM));
  QD_CUDA(cudaMemset(m->V, 0, sizeof(float) * NPARAM));
  k_w2_bf16<<<NH * NH / 256, 256>>>(m->P, m->W2b, m->W2tb);
  QD_CUDA(cudaDeviceSynchronize());
  *out = m;
  return QD_OK;
}

int qd_mlp_destroy(qd_mlp* m) {
  if (!m) return QD_OK;
  cudaSetDevice(m->device);
  cudaDeviceSynchronize();
  mlp_free_acts(m);
  for (void* p : {(void*)m->P, (void*)m->M, (void*)m->V, (void*)m->G, (void*)m->W2b, (void*)m->W2tb, (void*)m->p23,
                  (void*)m->p1, (void*)m->lpart, (void*)m->dW2})
    if (p) cudaFree(p);
  (void)cudaGetLastError();
  delete m;
  return QD_OK;
}

int qd_mlp_get_params(const qd_mlp* m, float* host, int64_t n) {
  if (!m || !host || n != NPARAM) {
    set_error("qd_mlp_get_params: need %lld floats", (long long)NPARAM);
    return QD_ERR_ARG;
  }
  QD_CUDA(cudaSetDevice(m->device));
  QD_CUDA(cudaMemcpy(host, m->P, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
  return QD_OK;
}

int qd_mlp_set_params(qd_mlp* m, const float* host, int64_t n) {
  if (!m || !host || n != NPARAM) {
    set_error("qd_mlp_set_params: need %lld floats", (long long)NPARAM);
    return QD_ERR_ARG;
  }
  QD_CUDA(cudaSetDevice(m->device));
  QD_CUDA(cudaMemcpy(m->P, host, sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
  QD_CUDA(cudaMemset(m->M, 0, sizeof(float) * NPARAM));
  QD_CUDA(cudaMemset(m->V, 0, sizeof(float) * NPARAM));
  m->step = 0;
  k_w2_bf16<<<NH * NH / 256, 256>>>(m->P, m->W2b, m->W2tb);
  QD_CUDA(cudaDeviceSynchronize());
  return QD_OK;
}

int qd_mlp_forward(qd_mlp* m, const float* d_X, float* d_y, int64_t n, void* stream) {
  if (!m || (n > 0 && (!d_X || !d_y)) || n < 0) {
    set_error("qd_mlp_forward: bad argument");
    return QD_ERR_ARG;
  }
  QD_CUDA(cudaSetDevice(m->device));
  cudaStream_t st = (cudaStream_t)stream;
  const i64 chunk = 1 << 18;  // bounded activation workspace
  for (i64 r = 0; r < n; r += chunk) {
    const i64 k = std::min<i64>(chunk, n - r);
    int rc = mlp_forward(m, d_X + r * NI, k, false, st);
    if (rc) return rc;
    QD_CUDA(cudaMemcpyAsync(d_y + r, m->y, sizeof(float) * k, cudaMemcpyDeviceToDevice, st));
  }
  return QD_OK;
}

int qd_mlp_grad(qd_mlp* m, const float* d_X, const float* d_T, int64_t n, float* d_grad, float* loss, void* stream) {
  if (!m || !d_X || !d_T || !d_grad) {
    set_error("qd_mlp_grad: null argument");
    return QD_ERR_ARG;
  }
  QD_CUDA(cudaSetDevice(m->device));
  cudaStream_t st = (cudaStream_t)stream;
  int rc = mlp_grad(m, d_X, d_T, n, loss, st);
  if (rc) return rc;
  QD_CUDA(cudaMemcpyAsync(d_grad, m->G, sizeof(float) * NPARAM, cudaMemcpyDeviceToDevice, st));
  QD_CUDA(cudaStreamSynchronize(st));
  return QD_OK;
}

int qd_mlp_train_step(qd_mlp* m, const float* d_X, const float* d_T, int64_t n, float lr, float* loss,
                      void* stream) {
  if (!m || !d_X || !d_T) {
    set_error("qd_mlp_train_step: null argument");
    return QD_ERR_ARG;
  }
  QD_CUDA(cudaSetDevice(m->device));
  cudaStream_t st = (cudaStream_t)stream;
  int rc = mlp_grad(m, d_X, d_T, n, loss, st);
  if (rc) return rc;
  m->step += 1;
  const float c1 = 1.0f - std::pow(0.9f, (float)m->step), c2 = 1.0f - std::pow(0.999f, (float)m->step);
  k_adam<<<(unsigned)((NPARAM + 255) / 256), 256, 0, st>>>(m->P, m->G, m->M, m->V, lr, c1, c2);
  k_w2_bf16<<<NH * NH / 256, 256, 0, st>>>(m->P, m->W2b, m->W2tb);
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

}  // extern "C"
