// split_gemm.cu -- split-precision FP64 products on the tcgen05 tensor cores.
//
// The FP64 block contractions (src/commutators.f90 matrix_mult222 and
// construct_cc_ints, which call dgemm) can run in split form: each operand is
// written as a short sum of BF16 "slices" whose products are exact in the
// tensor cores' FP32 accumulators (an Ozaki-style error-free splitting:
// Ozaki, Ogita, Oishi, Rump, Numer. Algorithms 59 (2012) 95), and the slice
// products are summed in FP64.
//
// Splitting.  A row i of op(A) (a column of op(B)) gets the exponent e_i with
// max_k |x(i,k)| < 2^e_i; r = x / 2^e_i in (-1, 1) (exact), and
//   d_1 = rint(128 r), r <- 128 r - d_1;  d_s = rint(128 r), ...   (exact)
// so x = 2^e_i sum_{s=1..S} d_s 2^-7s + O(2^(e_i - 7S - 1)), |d_1| <= 128,
// |d_s| <= 64 for s >= 2: every digit is an integer that BF16 holds exactly.
//
// Products.  C(m,n) = 2^(e_m + f_n) sum_{s+t <= S+1} 2^-7(s+t) sum_k a_s b_t.
// The slice pairs of one diagonal d = s + t share a TMEM accumulator (FP32);
// its partial sums are integers whose magnitude over a K chunk of KC terms
// is at most KC * bound(d) (bound = 2^14 for d <= 3, 2^12 (d+1) above), so
// with KC * bound < 2^24 every FP32 sum is exact.  After each chunk the
// diagonals are read from TMEM (tcgen05.ld) and added in FP64 with their
// scale 2^(e_m + f_n - 7d).  The only rounding is the truncation of the
// slice series and the FP64 summation.
//
// Kernel.  Persistent CTAs (one per SM) walk the 128 x 64 output tiles.  Per
// 64-wide K step a producer warp bulk-copies the S slices of the A tile
// (128 x 64) and of the B tile (64 x 64), stored pre-swizzled, into one of
// NST shared-memory stages; an MMA warp issues tcgen05.mma (kind::f16,
// BF16 x BF16 -> FP32, M=128, N=64, K=16) for every slice pair of the
// triangle into TMEM (S diagonals x 64 columns, two buffers when they fit)
// and commits to mbarriers; four epilogue warps read each finished chunk
// with tcgen05.ld and accumulate it in FP64 while the next chunk runs.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "dev_common.cuh"

namespace qd {

constexpr int SG_BM = 128, SG_BN = 64, SG_BK = 64;
constexpr int SG_MAXS = 8;
constexpr size_t SG_ATILE = (size_t)SG_BM * SG_BK * 2;  // bytes per A slice tile
constexpr size_t SG_BTILE = (size_t)SG_BN * SG_BK * 2;  // bytes per B slice tile
constexpr long long SG_SPIN = 1LL << 22;                // mbarrier polls before giving up

// Operand role: the slices of one op(A) (rows i = m) or op(B) (rows i = n),
// K-major, in a shared workspace: slice s of row i at
// slbase[S * unit + (s * rpad + i) * kpad + k] (unit = the sum of rpad * kpad
// over the roles before it); e_i at exbase[ex_off + i].  The slicer reads the role
// from source buffer src: x(i,k) = src[off + i * si + k * sk].
struct SRole {
  i64 unit;
  int ex_off, rpad, kpad, R, K, src;
  i64 off, si, sk;
};
struct SSeg {  // acc += c * hv0^pa * hv1^pb * op(A) op(B)
  int ra, rb, K;
  signed char pa, pb, pad0, pad1;
  double c;
};
struct SProb {
  int M, N, ldc, seg0, nseg, mode, outbuf, pad;  // mode: 0 SET, 1 ACC, 2 C = V + beta C
  i64 offC;
  double beta;
};
struct STask {
  int prob;
  short ti, tj;
};
struct SPtrs {
  const double* p[8];
};
constexpr int SG_NBUF = 8;

// K chunk over which every diagonal's FP32 sums stay exact
__host__ __device__ inline int split_kchunk(int S) {
  long long worst = 1LL << 14;
  for (int d = 4; d <= S + 1; ++d) worst = std::max(worst, (long long)4096 * (d + 1));
  long long kc = ((1LL << 24) - 1) / worst;
  kc = (kc / SG_BK) * SG_BK;
  return (int)std::max<long long>(SG_BK, std::min<long long>(kc, 1024));
}

__host__ __device__ inline int split_tmem_cols(int S) {
  int need = S * SG_BN, c = 32;
  while (c < need) c <<= 1;
  return c;
}

// ---------------------------------------------------------------------------
// slicing: role (x(i,k) = X[i*si + k*sk]) -> exponents and S slices
// ---------------------------------------------------------------------------
// Slices are stored pre-tiled: per role and slice, 128-row x 64-K tiles of
// 16 KB, row-tile major, each tile already in the K-major 128-byte-swizzled
// shared-memory layout (row r at r*128 bytes, 16-byte chunk c at
// (c ^ (r & 7))*16), so one bulk copy moves a whole tile (or a 64-row half).
__device__ __forceinline__ i64 tiled_off(int i, int k, int kpad) {
  const int r = i & 127, kk = k & 63;
  return ((i64)(i >> 7) * (kpad >> 6) + (k >> 6)) * 8192 + r * 64 + ((((kk >> 3) ^ (r & 7)) << 3) | (kk & 7));
}

// One CTA (256 threads) per (role, block of 32 rows): the rows' maxima, then
// per 64-wide K tile a coalesced load into shared memory (along the index that
// is contiguous in the source) and the slices, 8 digits of a row per 16-byte
// store.  Rows beyond R and K beyond the role's K get zero slices.
constexpr int SL_ROWS = 32, SL_THREADS = 256;
__global__ void __launch_bounds__(SL_THREADS) k_split_slice(const SRole* __restrict__ roles,
                                                            const i64* __restrict__ blkstart, int nroles, SPtrs src,
                                                            int S, __nv_bfloat16* __restrict__ slbase,
                                                            int* __restrict__ exbase) {
  __shared__ double T[SL_ROWS][65];
  __shared__ double red[SL_THREADS / 32][SL_ROWS];
  __shared__ int ex[SL_ROWS];
  const int r = find_seg(blkstart, nroles, blockIdx.x);
  const SRole ro = roles[r];
  const int i0 = (int)(blockIdx.x - blkstart[r]) * SL_ROWS;
  const double* X = src.p[ro.src] + ro.off;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const bool rowc = ro.si == 1;  // consecutive rows are adjacent in memory
  // maxima
  double mx = 0.0;
  if (rowc) {  // lane = row, warps stride over k
    const int i = i0 + lane;
    if (i < ro.R)
      for (int k = w; k < ro.K; k += SL_THREADS / 32) mx = fmax(mx, fabs(X[i + (i64)k * ro.sk]));
    red[w][lane] = mx;
  } else {  // warp per row, lanes over k
    for (int rr = w; rr < SL_ROWS; rr += SL_THREADS / 32) {
      const int i = i0 + rr;
      double m2 = 0.0;
      if (i < ro.R)
        for (int k = lane; k < ro.K; k += 32) m2 = fmax(m2, fabs(X[(i64)i * ro.si + (i64)k * ro.sk]));
      for (int o = 16; o; o >>= 1) m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
      if (lane == 0) red[0][rr] = m2;
    }
  }
  __syncthreads();
  if (t < SL_ROWS) {
    double m2 = red[0][t];
    if (rowc)
      for (int g = 1; g < SL_THREADS / 32; ++g) m2 = fmax(m2, red[g][t]);
    const int e = m2 > 0.0 ? ilogb(m2) + 1 : 0;
    ex[t] = e;
    exbase[ro.ex_off + i0 + t] = e;
  }
  __syncthreads();
  __nv_bfloat16* out = slbase + (i64)S * ro.unit;
  const i64 sstride = (i64)ro.rpad * ro.kpad;
  for (int k0 = 0; k0 < ro.kpad; k0 += 64) {
    // tile x(i0 + rr, k0 + c), rr < 32, c < 64
    for (int e = t; e < SL_ROWS * 64; e += SL_THREADS) {
      const int rr = rowc ? (e & 31) : (e >> 6), c = rowc ? (e >> 5) : (e & 63);
      const int i = i0 + rr, k = k0 + c;
      T[rr][c] = (i < ro.R && k < ro.K) ? X[(i64)i * ro.si + (i64)k * ro.sk] : 0.0;
    }
    __syncthreads();
    {  // thread = (row rr, 8-wide chunk cc)
      const int rr = t >> 3, cc = t & 7;
      const int e = ex[rr];
      double x[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) x[q] = scalbn(T[rr][cc * 8 + q], -e);
      const i64 o = tiled_off(i0 + rr, k0 + cc * 8, ro.kpad);  // 8 consecutive k share one 16-byte chunk
      for (int sl = 0; sl < S; ++sl) {
        __align__(16) __nv_bfloat16 d8[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const double tq = x[q] * 128.0;
          const double dq = rint(tq);
          x[q] = tq - dq;
          d8[q] = __float2bfloat16_rn((float)dq);
        }
        *reinterpret_cast<uint4*>(out + sl * sstride + o) = *reinterpret_cast<const uint4*>(d8);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// tcgen05 helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// K-major, 128-byte swizzle, 8-row atoms 1024 bytes apart (SBO), LBO 16 bytes
__device__ __forceinline__ uint64_t umma_desc(unsigned saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)64 << 32) | ((uint64_t)1 << 46) |
         ((uint64_t)2 << 61);
}
// kind::f16: D f32 (bits 4-5 = 1), A bf16 (7-9 = 1), B bf16 (10-12 = 1),
// both K-major, N >> 3 at 17, M >> 4 at 24
constexpr uint32_t SG_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(SG_BN >> 3) << 17) |
                              ((uint32_t)(SG_BM >> 4) << 24);

__device__ __forceinline__ void umma_bf16(unsigned dtmem, uint64_t ad, uint64_t bd, unsigned accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "l"(ad), "l"(bd), "r"(SG_IDESC), "r"(accum));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
// wait for the phase with parity `ph`; false if it did not complete in time
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned ph) {
  for (long long it = 0; it < SG_SPIN; ++it) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(ph)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(unsigned taddr, float* v) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void mbar_init_n(uint64_t* bar, unsigned n) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(n) : "memory");
}
__device__ __forceinline__ void mbar_expect(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// ---------------------------------------------------------------------------
// the grouped split GEMM: warp-specialised pipeline
// ---------------------------------------------------------------------------
// warps 0-3: epilogue (TMEM lanes 32w.., FP64 accumulation, output);
// warp 4: producer (bulk copies of the slice tiles into NST stages);
// warp 5: MMA issuer (tcgen05.mma into NB TMEM accumulator buffers).
// Barriers: full/empty per stage, accf/acce per accumulator buffer; every
// wait is bounded and a timeout sets `fail` (all roles then stop).
constexpr int SG_WARPS = 6, SG_THREADS_P = SG_WARPS * 32, SG_MAXST = 4;

template <int S>
__global__ void __launch_bounds__(SG_THREADS_P, 1)
    k_split_gemm(const STask* __restrict__ tasks, int ntask, const SProb* __restrict__ probs,
                 const SSeg* __restrict__ segs, const SRole* __restrict__ roles, int NST, int NB,
                 const __nv_bfloat16* __restrict__ slbase, const int* __restrict__ exbase, SPtrs outs, double hv0,
                 double hv1, int* __restrict__ err) {
  extern __shared__ uint8_t smraw[];
  __shared__ uint64_t full[SG_MAXST], empty[SG_MAXST], accf[2], acce[2];
  __shared__ unsigned tslot;
  __shared__ double fsc[SG_BN];  // 2^(column exponent) of the current segment
  __shared__ volatile int fail;
  const unsigned sbase = (smem_u32(smraw) + 1023u) & ~1023u;
  const unsigned stage_bytes = (unsigned)(S * (SG_ATILE + SG_BTILE));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ncols = split_tmem_cols(NB * S);
  const int kcs = split_kchunk(S) / SG_BK;  // K steps per exact chunk

  if (threadIdx.x == 0) {
    for (int i = 0; i < NST; ++i) {
      mbar_init_n(&full[i], 1);
      mbar_init_n(&empty[i], 1);
    }
    for (int i = 0; i < NB; ++i) {
      mbar_init_n(&accf[i], 1);
      mbar_init_n(&acce[i], 128);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fail = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tbase = tslot;

  if (warp == 4) {
    // ---- producer
    if (lane == 0) {
      int it = 0;
      for (int tk = blockIdx.x; tk < ntask && !fail; tk += gridDim.x) {
      const STask t = tasks[tk];
      const SProb P = probs[t.prob];
      const int col0 = t.tj * SG_BN;
      for (int sg = 0; sg < P.nseg && !fail; ++sg) {
        const SSeg G = segs[P.seg0 + sg];
        const SRole RA = roles[G.ra], RB = roles[G.rb];
        const int ksteps = (G.K + SG_BK - 1) / SG_BK;
        const __nv_bfloat16* a0 = slbase + (i64)S * RA.unit + (i64)t.ti * (RA.kpad >> 6) * 8192;
        const __nv_bfloat16* b0 =
            slbase + (i64)S * RB.unit + (i64)(col0 >> 7) * (RB.kpad >> 6) * 8192 + ((col0 >> 6) & 1) * 4096;
        const i64 sa = (i64)RA.rpad * RA.kpad, sb = (i64)RB.rpad * RB.kpad;
        for (int ks = 0; ks < ksteps; ++ks, ++it) {
          const int st = it % NST;
          if (!mbar_wait(&empty[st], ((it / NST) & 1) ^ 1)) {
            fail = 1;
            break;
          }
          mbar_expect(&full[st], stage_bytes);
          const unsigned sA = sbase + st * stage_bytes, sB = sA + S * (unsigned)SG_ATILE;
          for (int s = 0; s < S; ++s) {
            bulk_g2s(sA + s * (unsigned)SG_ATILE, a0 + s * sa + (i64)ks * 8192, (unsigned)SG_ATILE, &full[st]);
            bulk_g2s(sB + s * (unsigned)SG_BTILE, b0 + s * sb + (i64)ks * 8192, (unsigned)SG_BTILE, &full[st]);
          }
        }
      }
      }
    }
  } else if (warp == 5) {
    // ---- MMA issuer
    if (lane == 0) {
      int it = 0, ch = 0;
      for (int tk = blockIdx.x; tk < ntask && !fail; tk += gridDim.x) {
      const SProb P = probs[tasks[tk].prob];
      for (int sg = 0; sg < P.nseg && !fail; ++sg) {
        const int ksteps = (segs[P.seg0 + sg].K + SG_BK - 1) / SG_BK;
        for (int c0 = 0; c0 < ksteps && !fail; c0 += kcs, ++ch) {
          const int b = ch % NB;
          if (!mbar_wait(&acce[b], ((ch / NB) & 1) ^ 1)) {
            fail = 1;
            break;
          }
          tc_fence_after();
          const unsigned dbase = tbase + b * S * SG_BN;
          const int c1 = min(ksteps, c0 + kcs);
          for (int ks = c0; ks < c1; ++ks, ++it) {
            const int st = it % NST;
            if (!mbar_wait(&full[st], (it / NST) & 1)) {
              fail = 1;
              break;
            }
            tc_fence_after();
            const unsigned sA = sbase + st * stage_bytes, sB = sA + S * (unsigned)SG_ATILE;
            // descriptors advance by (byte offset >> 4) within the stage
            const uint64_t dA = umma_desc(sA), dB = umma_desc(sB);
            const unsigned first = ks == c0 ? 0u : 1u;
#pragma unroll
            for (int k16 = 0; k16 < SG_BK / 16; ++k16)
#pragma unroll
              for (int s = 0; s < S; ++s)
#pragma unroll
                for (int u = 0; u + s < S; ++u)  // slice pair (s+1, u+1), diagonal s+u+2
                  umma_bf16(dbase + (s + u) * SG_BN, dA + ((s * (unsigned)SG_ATILE + k16 * 32) >> 4),
                            dB + ((u * (unsigned)SG_BTILE + k16 * 32) >> 4),
                            (k16 | s) ? 1u : first);  // each diagonal starts at (k16, s) = (0, 0)
            umma_commit(&empty[st]);  // the stage is free once these MMAs complete
          }
          umma_commit(&accf[b]);  // the chunk's diagonals are complete
        }
      }
      }
    }
  } else {
    // ---- epilogue: thread = output row m (TMEM lane)
    int ch = 0;
    for (int tk = blockIdx.x; tk < ntask; tk += gridDim.x) {
    const STask t = tasks[tk];
    const SProb P = probs[t.prob];
    const int row0 = t.ti * SG_BM, col0 = t.tj * SG_BN;
    const int m = row0 + threadIdx.x;
    double acc[SG_BN];
#pragma unroll
    for (int j = 0; j < SG_BN; ++j) acc[j] = 0.0;
    // the four epilogue warps run every segment (their named barriers must
    // match); after a failed wait they skip the waits and reads
    for (int sg = 0; sg < P.nseg; ++sg) {
      const SSeg G = segs[P.seg0 + sg];
      const SRole RA = roles[G.ra], RB = roles[G.rb];
      const double alpha = G.c * (G.pa ? hv0 : 1.0) * (G.pb ? hv1 : 1.0);
      const int em = m < P.M ? exbase[RA.ex_off + m] : 0;
      asm volatile("bar.sync 1, 128;" ::: "memory");  // fsc of the previous segment is no longer read
      if (threadIdx.x < SG_BN)
        fsc[threadIdx.x] = ldexp(1.0, (col0 + threadIdx.x < P.N) ? exbase[RB.ex_off + col0 + threadIdx.x] : 0);
      asm volatile("bar.sync 1, 128;" ::: "memory");
      const int ksteps = (G.K + SG_BK - 1) / SG_BK;
      for (int c0 = 0; c0 < ksteps; c0 += kcs, ++ch) {
        const int b = ch % NB;
        if (fail) continue;
        if (!mbar_wait(&accf[b], (ch / NB) & 1)) {
          fail = 1;
          continue;
        }
        tc_fence_after();
        const unsigned dbase = tbase + ((unsigned)(warp * 32) << 16) + b * S * SG_BN;
        for (int d = 0; d < S; ++d) {
          const double rs = ldexp(alpha, em - 7 * (d + 2));
#pragma unroll
          for (int q = 0; q < SG_BN / 16; ++q) {
            float v[16];
            tmem_ld16(dbase + d * SG_BN + q * 16, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[q * 16 + j] = fma((double)v[j] * rs, fsc[q * 16 + j], acc[q * 16 + j]);
          }
        }
        tc_fence_before();
        mbar_arrive(&acce[b]);
      }
    }
    if (!fail && m < P.M) {
      double* out = const_cast<double*>(outs.p[P.outbuf]) + P.offC + m;
      const int nn = min(SG_BN, P.N - col0);
#pragma unroll
      for (int j = 0; j < SG_BN; ++j) {
        if (j >= nn) break;
        double* p = out + (i64)(col0 + j) * P.ldc;
        if (P.mode == 0)
          *p = acc[j];
        else if (P.mode == 1)
          *p += acc[j];
        else
          *p = acc[j] + (P.beta == 0.0 ? 0.0 : P.beta * *p);
      }
    }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (fail && threadIdx.x == 0) atomicExch(err, 1);
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(ncols) : "memory");
  }
}

// pipeline shape for S slices: stages of S A tiles and S B tiles (24 KB per
// slice) within 192 KB; two TMEM accumulator sets when they fit 512 columns
int split_stages(int S) { return std::max(1, std::min(SG_MAXST, (192 * 1024) / (S * (int)(SG_ATILE + SG_BTILE)))); }
int split_nbuf(int S) { return 2 * S * SG_BN <= 512 ? 2 : 1; }
size_t split_gemm_smem(int S) { return (size_t)split_stages(S) * S * (SG_ATILE + SG_BTILE) + 1024; }

// pair modes: C = (C +) V + sigma V^T from the product V (M x M scratch)
struct SPair {
  int M, ldc, outbuf, acc;
  i64 offV, offC;
  double sc;
  int spa, spb;
};
struct SPairTask {
  int pair;
  short ti, tj;
};
__global__ void k_split_pair(const SPairTask* __restrict__ tasks, const SPair* __restrict__ pairs,
                             const double* __restrict__ V, SPtrs outs, double hv0, double hv1) {
  __shared__ double t[32][33];
  const SPairTask tk = tasks[blockIdx.x];
  const SPair P = pairs[tk.pair];
  const double sigma = P.sc * (P.spa ? hv0 : 1.0) * (P.spb ? hv1 : 1.0);
  const double* v = V + P.offV;
  double* C = const_cast<double*>(outs.p[P.outbuf]) + P.offC;
  const int r0 = tk.ti * 32, c0 = tk.tj * 32, M = P.M;
  for (int e = threadIdx.x; e < 1024; e += blockDim.x) {  // t[i][j] = V(c0+i, r0+j)
    const int i = e & 31, j = e >> 5;
    t[i][j] = (c0 + i < M && r0 + j < M) ? v[(c0 + i) + (i64)(r0 + j) * M] : 0.0;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < 1024; e += blockDim.x) {
    const int a = e & 31, b = e >> 5, r = r0 + a, c = c0 + b;
    if (r < M && c < M) {
      const double val = v[r + (i64)c * M] + sigma * t[b][a];
      double* p = C + r + (i64)c * P.ldc;
      *p = P.acc ? *p + val : val;
    }
  }
}

__global__ void k_scale2d(double* __restrict__ C, int ldc, int M, i64 n, double beta) {
  const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) C[(e % M) + (e / M) * ldc] *= beta;
}

// ---------------------------------------------------------------------------
// host side: split plans of the grouped GEMM programs
// ---------------------------------------------------------------------------
namespace {

struct SplitPlan {
  std::vector<SRole> roles;
  i64 units = 0, exn = 0, vsize = 0, rows = 0;
  SRole* d_roles = nullptr;
  i64* d_rowstart = nullptr;
  SSeg* d_segs = nullptr;
  SProb* d_probs = nullptr;
  STask* d_tasks = nullptr;
  SPair* d_pairs = nullptr;
  SPairTask* d_ptasks = nullptr;
  int ntask = 0, nptask = 0;
};

struct SplitState {
  std::map<std::tuple<const void*, unsigned, unsigned>, SplitPlan> plans;
  __nv_bfloat16* sl = nullptr;
  size_t sl_n = 0;
  int* ex = nullptr;
  size_t ex_n = 0;
  double* V = nullptr;
  size_t v_n = 0;
  int* err = nullptr;
};

template <class T>
int upload(const std::vector<T>& h, T** d) {
  QD_CUDA(cudaMalloc((void**)d, std::max<size_t>(1, h.size()) * sizeof(T)));
  if (!h.empty()) QD_CUDA(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return QD_OK;
}

bool seg_live(const GSeg& s, unsigned mA, unsigned mB) {
  auto dead = [&](int src, int dep) {
    if (dep < 0) return false;
    unsigned m = src == 0 ? mA : (src == 1 ? mB : 0u);
    return ((m >> dep) & 1u) != 0;
  };
  return s.K > 0 && !dead(s.srcA, s.depA) && !dead(s.srcB, s.depB);
}

constexpr int SG_VBUF = 7;  // output slot of the pair-mode scratch

int build_plan(const GemmProgram& G, unsigned mA, unsigned mB, SplitPlan& sp) {
  std::map<std::tuple<int, i64, i64, i64, int, int>, int> rk;
  auto role = [&](int src, i64 off, i64 si, i64 sk, int R, int K) {
    auto key = std::make_tuple(src, off, si, sk, R, K);
    auto it = rk.find(key);
    if (it != rk.end()) return it->second;
    SRole r;
    r.R = R;
    r.K = K;
    r.rpad = (R + SG_BM - 1) / SG_BM * SG_BM;
    r.kpad = std::max(SG_BK, (K + SG_BK - 1) / SG_BK * SG_BK);
    r.unit = sp.units;
    r.ex_off = (int)sp.exn;
    r.src = src;
    r.off = off;
    r.si = si;
    r.sk = sk;
    sp.units += (i64)r.rpad * r.kpad;
    sp.exn += r.rpad;
    sp.roles.push_back(r);
    rk[key] = (int)sp.roles.size() - 1;
    return (int)sp.roles.size() - 1;
  };
  std::vector<SSeg> segs;
  std::vector<SProb> probs;
  std::vector<SPair> pairs;
  std::vector<std::pair<double, STask>> tv;
  for (const GProb& g : G.probs) {
    const bool pair = g.mode == GM_ACC_PAIR || g.mode == GM_SET_PAIR;
    const bool set = g.mode == GM_SET || g.mode == GM_SET_PAIR;
    SProb p;
    std::memset(&p, 0, sizeof(p));
    p.M = g.M;
    p.N = g.N;
    p.seg0 = (int)segs.size();
    double cost = 1.0;
    for (int k = 0; k < g.nseg; ++k) {
      const GSeg& s = G.segs[g.seg0 + k];
      if (!seg_live(s, mA, mB)) continue;
      SSeg q;
      std::memset(&q, 0, sizeof(q));
      q.ra = role(s.srcA, s.offA, s.tA ? s.lda : 1, s.tA ? 1 : s.lda, g.M, s.K);
      q.rb = role(s.srcB, s.offB, s.tB ? 1 : s.ldb, s.tB ? s.ldb : 1, g.N, s.K);
      q.K = s.K;
      q.c = s.c;
      q.pa = s.pa;
      q.pb = s.pb;
      segs.push_back(q);
      cost += (s.K + SG_BK - 1) / SG_BK;
    }
    p.nseg = (int)segs.size() - p.seg0;
    if (p.nseg == 0 && !set) continue;
    if (pair) {
      SPair pr;
      std::memset(&pr, 0, sizeof(pr));
      pr.M = g.M;
      pr.ldc = g.ldc;
      pr.outbuf = g.outbuf;
      pr.acc = g.mode == GM_ACC_PAIR;
      pr.offV = sp.vsize;
      pr.offC = g.offC;
      pr.sc = g.sc;
      pr.spa = g.spa;
      pr.spb = g.spb;
      pairs.push_back(pr);
      p.mode = 0;
      p.outbuf = SG_VBUF;
      p.offC = sp.vsize;
      p.ldc = g.M;
      sp.vsize += (i64)g.M * g.M;
    } else {
      p.mode = set ? 0 : 1;
      p.outbuf = g.outbuf;
      p.offC = g.offC;
      p.ldc = g.ldc;
    }
    probs.push_back(p);
    const int tm = (g.M + SG_BM - 1) / SG_BM, tn = (g.N + SG_BN - 1) / SG_BN;
    for (int i = 0; i < tm; ++i)
      for (int j = 0; j < tn; ++j) tv.push_back({cost, STask{(int)probs.size() - 1, (short)i, (short)j}});
  }
  std::stable_sort(tv.begin(), tv.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  std::vector<STask> tasks(tv.size());
  for (size_t i = 0; i < tv.size(); ++i) tasks[i] = tv[i].second;
  std::vector<SPairTask> pt;
  for (size_t k = 0; k < pairs.size(); ++k) {
    const int t = (pairs[k].M + 31) / 32;
    for (int i = 0; i < t; ++i)
      for (int j = 0; j < t; ++j) pt.push_back(SPairTask{(int)k, (short)i, (short)j});
  }
  std::vector<i64> rowstart(sp.roles.size() + 1, 0);  // slicer blocks of SL_ROWS rows per role
  for (size_t r = 0; r < sp.roles.size(); ++r) rowstart[r + 1] = rowstart[r] + sp.roles[r].rpad / SL_ROWS;
  sp.rows = rowstart.back();
  int rc;
  if ((rc = upload(sp.roles, &sp.d_roles)) || (rc = upload(rowstart, &sp.d_rowstart)) ||
      (rc = upload(segs, &sp.d_segs)) || (rc = upload(probs, &sp.d_probs)) || (rc = upload(tasks, &sp.d_tasks)) ||
      (rc = upload(pairs, &sp.d_pairs)) || (rc = upload(pt, &sp.d_ptasks)))
    return rc;
  sp.ntask = (int)tasks.size();
  sp.nptask = (int)pt.size();
  return QD_OK;
}

void free_plan(SplitPlan& sp) {
  for (void* p : {(void*)sp.d_roles, (void*)sp.d_rowstart, (void*)sp.d_segs, (void*)sp.d_probs, (void*)sp.d_tasks,
                  (void*)sp.d_pairs, (void*)sp.d_ptasks})
    if (p) cudaFree(p);
}

// slices, products and pair combines of one plan on `st`; workspaces grown on demand
int run_plan(SplitState& ss, const SplitPlan& sp, int S, SPtrs bufs, double hv0, double hv1, cudaStream_t st,
             i64* ws_bytes) {
  auto grow = [&](auto*& ptr, size_t& have, size_t need, size_t elem) -> int {
    if (need <= have) return QD_OK;
    if (ptr) {
      QD_CUDA(cudaStreamSynchronize(st));
      QD_CUDA(cudaFree(ptr));
    }
    ptr = nullptr;
    QD_CUDA(cudaMalloc((void**)&ptr, need * elem));
    if (ws_bytes) *ws_bytes += (i64)((need - have) * elem);
    have = need;
    return QD_OK;
  };
  int rc;
  if ((rc = grow(ss.sl, ss.sl_n, (size_t)S * sp.units, 2)) || (rc = grow(ss.ex, ss.ex_n, (size_t)sp.exn, 4)) ||
      (rc = grow(ss.V, ss.v_n, (size_t)std::max<i64>(1, sp.vsize), 8)))
    return rc;
  if (!ss.err) {
    QD_CUDA(cudaMalloc((void**)&ss.err, sizeof(int)));
    QD_CUDA(cudaMemsetAsync(ss.err, 0, sizeof(int), st));
  }
  if (sp.rows > 0)
    k_split_slice<<<(unsigned)sp.rows, SL_THREADS, 0, st>>>(sp.d_roles, sp.d_rowstart, (int)sp.roles.size(), bufs,
                                                            S, ss.sl, ss.ex);
  SPtrs outs = bufs;
  outs.p[SG_VBUF] = ss.V;
  if (sp.ntask > 0) {
    const size_t smem = split_gemm_smem(S);
    int dev = 0, nsm = 148;
    QD_CUDA(cudaGetDevice(&dev));
    QD_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int grid = std::min(sp.ntask, nsm);  // one CTA per SM (the stages fill shared memory)
    switch (S) {
#define QD_SPLIT_LAUNCH(SS)                                                                                       \
  case SS:                                                                                                        \
    QD_CUDA(cudaFuncSetAttribute(k_split_gemm<SS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));      \
    k_split_gemm<SS><<<grid, SG_THREADS_P, smem, st>>>(sp.d_tasks, sp.ntask, sp.d_probs, sp.d_segs, sp.d_roles,  \
                                                       split_stages(SS), split_nbuf(SS), ss.sl, ss.ex, outs, hv0, \
                                                       hv1, ss.err);                                              \
    break;
      QD_SPLIT_LAUNCH(1) QD_SPLIT_LAUNCH(2) QD_SPLIT_LAUNCH(3) QD_SPLIT_LAUNCH(4)
      QD_SPLIT_LAUNCH(5) QD_SPLIT_LAUNCH(6) QD_SPLIT_LAUNCH(7) QD_SPLIT_LAUNCH(8)
#undef QD_SPLIT_LAUNCH
      default:
        set_error("split product: slices must be 1..8");
        return QD_ERR_ARG;
    }
  }
  if (sp.nptask > 0) k_split_pair<<<sp.nptask, 256, 0, st>>>(sp.d_ptasks, sp.d_pairs, ss.V, outs, hv0, hv1);
  QD_CUDA(cudaGetLastError());
  return QD_OK;
}

int check_err(SplitState& ss, cudaStream_t st) {
  if (!ss.err) return QD_OK;
  int h = 0;
  QD_CUDA(cudaMemcpyAsync(&h, ss.err, sizeof(int), cudaMemcpyDeviceToHost, st));
  QD_CUDA(cudaStreamSynchronize(st));
  if (h) {
    set_error("split product: tensor-core wait timed out");
    return QD_ERR_CUDA;
  }
  return QD_OK;
}

void free_state(SplitState* ss) {
  if (!ss) return;
  for (auto& kv : ss->plans) free_plan(kv.second);
  for (void* p : {(void*)ss->sl, (void*)ss->ex, (void*)ss->V, (void*)ss->err})
    if (p) cudaFree(p);
  delete ss;
}

}  // namespace

// the commutator's GEMM programs in the split form (L->split_slices slices)
int run_program_split(qd_layout* L, GemmProgram& P, const double* const* bufs, double hv0, double hv1, unsigned maskA,
                      unsigned maskB) {
  SplitState*& ss = reinterpret_cast<SplitState*&>(L->split);
  if (!ss) ss = new SplitState();
  auto key = std::make_tuple((const void*)&P, maskA, maskB);
  auto it = ss->plans.find(key);
  if (it == ss->plans.end()) {
    SplitPlan sp;
    int rc = build_plan(P, maskA, maskB, sp);
    if (rc) {
      free_plan(sp);
      return rc;
    }
    it = ss->plans.emplace(key, sp).first;
  }
  SPtrs b;
  for (int i = 0; i < SG_NBUF; ++i) b.p[i] = i < 7 ? bufs[i] : nullptr;
  int rc = run_plan(*ss, it->second, L->split_slices, b, hv0, hv1, L->stream, &L->ws_bytes);
  L->nlaunch += 3;
  return rc;
}

void split_free(qd_layout* L) {
  free_state(reinterpret_cast<SplitState*>(L->split));
  L->split = nullptr;
}

}  // namespace qd

using namespace qd;

extern "C" {

// ---------------------------------------------------------------------------
// C ABI: one split-precision product with dgemm's argument meaning
// ---------------------------------------------------------------------------
int qd_gemm_split(int device, void* stream, char transa, char transb, int M, int N, int K, double alpha,
                  const double* A, int lda, const double* B, int ldb, double beta, double* C, int ldc, int slices) {
  const bool ta = transa == 'T' || transa == 't', tb = transb == 'T' || transb == 't';
  if (!(ta || transa == 'N' || transa == 'n') || !(tb || transb == 'N' || transb == 'n') || M < 0 || N < 0 ||
      K < 0 || slices < 1 || slices > SG_MAXS || (M > 0 && N > 0 && (!C || ldc < M)) ||
      (M > 0 && K > 0 && (!A || lda < (ta ? K : M))) || (N > 0 && K > 0 && (!B || ldb < (tb ? N : K)))) {
    set_error("qd_gemm_split: bad argument");
    return QD_ERR_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("qd_gemm_split: no CUDA device");
    return QD_ERR_NODEVICE;
  }
  QD_CUDA(cudaSetDevice(device));
  cudaStream_t st = (cudaStream_t)stream;
  if (M == 0 || N == 0) return QD_OK;
  // a one-problem program: buffers 0 = A, 1 = B, 4 = C
  GemmProgram G;
  GProb g;
  std::memset(&g, 0, sizeof(g));
  g.M = M;
  g.N = N;
  g.ldc = ldc;
  g.mode = GM_ACC;
  g.outbuf = 4;
  g.nseg = K > 0 ? 1 : 0;
  G.probs.push_back(g);
  if (K > 0) {
    GSeg s;
    std::memset(&s, 0, sizeof(s));
    s.lda = lda;
    s.ldb = ldb;
    s.K = K;
    s.srcA = 0;
    s.srcB = 1;
    s.tA = ta;
    s.tB = tb;
    s.depA = s.depB = -1;
    s.c = alpha;
    G.segs.push_back(s);
  }
  // C = V + beta C: scale C first (beta = 0 overwrites, as dgemm), then accumulate
  if (beta == 0.0) {
    QD_CUDA(cudaMemset2DAsync(C, sizeof(double) * ldc, 0, sizeof(double) * M, N, st));
  } else if (beta != 1.0) {
    const i64 n = (i64)M * N;
    k_scale2d<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(C, ldc, M, n, beta);
  }
  SplitState ss;
  SplitPlan sp;
  int rc = build_plan(G, 0u, 0u, sp);
  if (!rc) {
    SPtrs b;
    for (int i = 0; i < SG_NBUF; ++i) b.p[i] = nullptr;
    b.p[0] = A;
    b.p[1] = B;
    b.p[4] = C;
    rc = run_plan(ss, sp, slices, b, 1.0, 1.0, st, nullptr);
    if (!rc) rc = check_err(ss, st);
  }
  cudaStreamSynchronize(st);
  free_plan(sp);
  for (void* p : {(void*)ss.sl, (void*)ss.ex, (void*)ss.V, (void*)ss.err})
    if (p) cudaFree(p);
  return rc;
}

}  // extern "C"
