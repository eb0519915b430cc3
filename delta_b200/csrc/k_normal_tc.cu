// Normal equations of the kernel fit on the 5th-generation tensor cores
// (reference src/solve.cpp:70-145, the X^T W X rank updates), "mixed" precision.
//
// The Kronecker-packed contraction
//     G[u][v] = sum_i U[i][u] V[i][v],   U[i][u] = b_a b_b (u = {a,b}, b = [bn_i, 1]),
//                                        V[i][v] = w_i d_m d_m' (v = {m,m'}),
// is a (Mu x N) x (N x Nv) product with the N stamp rows as the reduction
// dimension. Each CTA owns one 128 x BN output tile and one contiguous row
// range (split K). Per 64-row chunk the CTA stages the rows in shared memory,
// generates U and V for its tile in FP32, splits every value into
// x = hi + lo (two bf16), writes both into the UMMA K-major canonical layout,
// and one elected thread issues tcgen05.mma (kind::f16, bf16 x bf16 -> FP32)
// for hi*hi + hi*lo + lo*hi into the TMEM accumulator (BF16x3: about 16
// significant bits per product, FP32 accumulation). Two shared-memory stages
// let the tensor core consume chunk c while the threads generate chunk c+1;
// tcgen05.commit on an mbarrier releases a stage. Every kDrainChunks chunks
// the CTA waits for its MMAs, reads the accumulator with tcgen05.ld and adds
// it into its FP64 partial in global memory, and the next chunk starts a fresh
// accumulation: each FP32 accumulation chain is at most 12 kDrainChunks MMAs
// long, where a whole split (80+ chunks) would lose about 1e-4 of the sums
// to FP32 accumulation rounding. The host-side caller reduces the splits in a
// fixed order in FP64 and an FP64 refinement step follows the solve.
//
// Every mbarrier wait is bounded: on expiry the kernel sets the loop-limit
// status bit, waits (bounded) for its own MMAs, frees its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "dev_common.cuh"
#include "fit_internal.h"

namespace dgpu {
namespace {

constexpr int kBM = 128;       // u rows per tile (UMMA M)
constexpr int kKC = 64;        // stamp rows per chunk (4 UMMA K-steps of 16)
constexpr int kThreads = 512;
constexpr int kRS = kKC + 4;  // staged row-value stride (floats): rows contiguous, banks staggered
constexpr long long kSpinCap = 1ll << 22;
constexpr int kDrainChunks = 4;  // chunks per FP32 accumulation chain

struct TcArgs {
  int64_t N;
  int nc, k, SS;
  FitRows R;
  const uint8_t* accepted;
  const int2* upairs;
  int Mu;
  const int2* vpairs;
  int Nv;
  int BN;  // N tile, multiple of 16, <= 256
  int tmem_cols;
  int64_t rows_per_split;
  double* gpart;  // per split: tiles x BN x kBM, (tile, column, row) order
  unsigned* status;
  int bulk;  // row arrays 16-byte aligned: full chunks arrive by cp.async.bulk
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor, no swizzle (K-major "interleaved" canonical
// layout): start address, leading byte offset (between the two K-adjacent
// 8x16-byte core matrices), stride byte offset (between 8-row groups),
// descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  return d;
}

// kind::f16 instruction descriptor: FP32 accumulate, bf16 A and B, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Bounded wait for the phase of `bar` with the given parity; false on expiry.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  const uint32_t a = smem_addr(bar);
  for (long long it = 0; it < kSpinCap; ++it) {
    uint32_t done = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 1-D bulk async copy global -> this CTA's shared memory, completing on `bar`
// (no multicast). dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// kind::tf32 instruction descriptor: FP32 accumulate, TF32 A and B, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(M >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Byte offset of element (row, kk) of a rows x kKC bf16 tile in the K-major
// canonical layout: 8x8 core matrices of 128 contiguous bytes, the kKC/8 core
// matrices of one 8-row group adjacent (LBO = 128 B), groups kKC*16 B apart (SBO).
__device__ __forceinline__ uint32_t canon_off(int row, int kg) {
  return static_cast<uint32_t>(((row >> 3) * (kKC / 8) + kg) * 128 + (row & 7) * 16);
}

// x = hi + lo, both bf16 (hi = rn(x), lo = rn(x - hi)), eight values per
// call as packed pairs; one 16-byte store per half.
__device__ __forceinline__ void split_store(unsigned char* hi_base, unsigned char* lo_base, uint32_t off,
                                            const float (&v)[8]) {
  __align__(16) __nv_bfloat162 h[4];
  __align__(16) __nv_bfloat162 l[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    h[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
    const float2 hf = __bfloat1622float2(h[j]);
    l[j] = __floats2bfloat162_rn(v[2 * j] - hf.x, v[2 * j + 1] - hf.y);
  }
  *reinterpret_cast<uint4*>(hi_base + off) = *reinterpret_cast<const uint4*>(h);
  *reinterpret_cast<uint4*>(lo_base + off) = *reinterpret_cast<const uint4*>(l);
}

// TF32 operands: 4-byte elements, so a core matrix (8 rows x 16 bytes) holds 4
// K values; 8 values round to nearest (ties away) with cvt.rna.tf32.f32 and
// go out as two 16-byte stores into K-adjacent core matrices (128 bytes apart).
__device__ __forceinline__ uint32_t canon_off_tf32(int row, int kg8) {
  return static_cast<uint32_t>(((row >> 3) * (kKC / 4) + 2 * kg8) * 128 + (row & 7) * 16);
}

__device__ __forceinline__ void tf32_store(unsigned char* base, uint32_t off, const float (&v)[8]) {
  __align__(16) uint32_t t[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t[j]) : "f"(v[j]));
  *reinterpret_cast<uint4*>(base + off) = *reinterpret_cast<const uint4*>(t);
  *reinterpret_cast<uint4*>(base + off + 128) = *reinterpret_cast<const uint4*>(t + 4);
}

// kTf32: one TF32 product per K-step (kind::tf32, 8 K values per MMA) in place
// of the three BF16 products; the two stage buffers of 32-bit operands take
// the place of the four bf16 hi / lo buffers (same bytes).
template <bool kTf32>
__global__ void __launch_bounds__(kThreads, 1) k_normal_tc(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x;
  const int BN = a.BN;
  const int nf = a.nc + 1;
  const int u0 = blockIdx.x * kBM, v0 = blockIdx.y * BN;
  const int64_t rbeg = static_cast<int64_t>(blockIdx.z) * a.rows_per_split;
  const int64_t rend = min(a.N, rbeg + a.rows_per_split);
  const int nchunks = rend > rbeg ? static_cast<int>((rend - rbeg + kKC - 1) / kKC) : 0;

  // Shared memory carve-up (all operand buffers 1024-byte aligned).
  const uint32_t a_bytes = kBM * kKC * 2, b_bytes = static_cast<uint32_t>(BN) * kKC * 2;
  // stage st: A hi at st*a_bytes, A lo at (2+st)*a_bytes; B hi / lo likewise after the A buffers
  unsigned char* b_base = smem + 4 * a_bytes;
  // Staged chunk, value-major: bnT[q][r] = b_q of row r (b_nc = 1),
  // dT[m][r] = d_m, wdT[m][r] = w_r d_m (w_r = 0 for inactive rows).
  float* bnT = reinterpret_cast<float*>(b_base + 4 * b_bytes);  // nf x kRS
  float* dT = bnT + nf * kRS;                                    // k x kRS
  float* wdT = dT + a.k * kRS;                                   // k x kRS
  float* w_s = wdT + a.k * kRS;                                  // kKC row weights
  int2* up_s = reinterpret_cast<int2*>(w_s + kKC);               // kBM
  int2* vp_s = up_s + kBM;                                       // BN
  uint64_t* mbar = reinterpret_cast<uint64_t*>(vp_s + BN + (BN & 1));  // [0,1] MMA stages, [2,3] row loads
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 4);
  // Raw rows of a chunk as stored in global memory, two buffers (16-byte aligned).
  const uint32_t raw_bn = kKC * a.nc * 8, raw_d = kKC * a.k * 8, raw_w = kKC * 8, raw_v = kKC;
  const uint32_t raw_bytes = raw_bn + raw_d + raw_w + raw_v;
  unsigned char* raw_base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(tmem_slot + 4) + 15) & ~static_cast<uintptr_t>(15));
  __shared__ int s_fail;

  for (int m = tid; m < kBM; m += blockDim.x) up_s[m] = (u0 + m < a.Mu) ? a.upairs[u0 + m] : make_int2(-1, -1);
  for (int n = tid; n < BN; n += blockDim.x) vp_s[n] = (v0 + n < a.Nv) ? a.vpairs[v0 + n] : make_int2(-1, -1);
  if (tid == 0) {
    s_fail = 0;
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    mbar_init(&mbar[2], 1);
    mbar_init(&mbar[3], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(a.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = kTf32 ? umma_idesc_tf32(kBM, BN) : umma_idesc_bf16(kBM, BN);
  constexpr uint32_t kLBO = 128, kSBO = kTf32 ? (kKC / 4) * 128 : (kKC / 8) * 128;

  // Chunk c of this split is bulk-loaded when it is full and the rows are aligned.
  auto chunk_rows = [&](int c) {
    const int64_t left = rend - (rbeg + static_cast<int64_t>(c) * kKC);
    return static_cast<int>(left < kKC ? left : kKC);
  };
  auto issue_rows = [&](int c) {  // by one thread
    const int64_t r0 = rbeg + static_cast<int64_t>(c) * kKC;
    unsigned char* dst = raw_base + (c & 1) * raw_bytes;
    uint64_t* bar = &mbar[2 + (c & 1)];
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar, raw_bytes);
    bulk_g2s(dst, a.R.bn + r0 * a.nc, raw_bn, bar);
    bulk_g2s(dst + raw_bn, a.R.d + r0 * a.k, raw_d, bar);
    bulk_g2s(dst + raw_bn + raw_d, a.R.w + r0, raw_w, bar);
    bulk_g2s(dst + raw_bn + raw_d + raw_w, a.R.valid + r0, raw_v, bar);
  };
  int ld_hi = -1, ld_done = -1;  // highest chunk whose rows were bulk-requested / waited (uniform)
  if (nchunks > 0 && a.bulk && chunk_rows(0) == kKC) {
    ld_hi = 0;
    if (tid == 0) issue_rows(0);
  }

  // Accumulator -> FP64 partial of this split: warp w reads TMEM lanes
  // 32 (w % 4) .. +31 (tile rows); the warp groups split the column blocks of
  // 16. The partial is column-major within the tile, so each column of a
  // warp's 32 rows is one contiguous 256-byte access. The first drain stores,
  // later ones add; padding rows and columns hold zeros.
  const int warp = tid >> 5, lane = tid & 31;
  const int quarter = warp & 3, grp = warp >> 2, ngrp = (blockDim.x >> 5) / 4;
  double* out = a.gpart +
                (static_cast<size_t>(blockIdx.z) * gridDim.x * gridDim.y + blockIdx.x * gridDim.y + blockIdx.y) *
                    static_cast<size_t>(BN) * kBM +
                quarter * 32 + lane;
  auto drain = [&](bool first, bool valid) {
    for (int cb = grp; cb < BN / 16; cb += ngrp) {
      uint32_t r[16];
      if (valid) {
        tmem_ld16(tmem + (static_cast<uint32_t>(quarter * 32) << 16) + static_cast<uint32_t>(cb * 16), r);
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) r[j] = 0u;
      }
      double* o = out + static_cast<size_t>(cb) * 16 * kBM;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const double x = static_cast<double>(__uint_as_float(r[j]));
        o[j * kBM] = first ? x : o[j * kBM] + x;
      }
    }
  };

  int issued = 0;  // chunks whose MMAs were issued (uniform over the CTA)
  for (int c = 0; c < nchunks; ++c) {
    const int st = c & 1;
    unsigned char* ahi = smem + (kTf32 ? 2 * st : st) * a_bytes;
    unsigned char* alo = smem + (2 + st) * a_bytes;
    unsigned char* bhi = b_base + (kTf32 ? 2 * st : st) * b_bytes;
    unsigned char* blo = b_base + (2 + st) * b_bytes;
    const int64_t r0 = rbeg + static_cast<int64_t>(c) * kKC;
    const int rows = chunk_rows(c);
    const bool bulk_c = a.bulk && rows == kKC;
    // Next chunk's rows fly in while this one is generated (its buffer was
    // last read two chunks ago, before the last barrier).
    if (c + 1 < nchunks && a.bulk && chunk_rows(c + 1) == kKC) {
      ld_hi = c + 1;
      if (tid == 0) issue_rows(c + 1);
    }
    const unsigned char* raw = raw_base + st * raw_bytes;
    if (bulk_c) {
      if (mbar_wait(&mbar[2 + st], static_cast<unsigned>(c >> 1) & 1u))
        ld_done = c;
      else
        s_fail = 1;
      __syncthreads();
      if (s_fail) break;
    }
    const double* rbn = reinterpret_cast<const double*>(raw);
    const double* rd = reinterpret_cast<const double*>(raw + raw_bn);
    const double* rw = reinterpret_cast<const double*>(raw + raw_bn + raw_d);
    const uint8_t* rv = raw + raw_bn + raw_d + raw_w;
    // Stage the chunk's rows as FP32, value-major (the previous chunk's
    // generation finished at the last barrier). Row weights first (0 for
    // inactive rows); then thread (value q = lane, rows 4 g .. 4 g + 3)
    // converts four rows of one value and stores them as one float4. Rows of
    // weight 0 stage zeros: an inactive row may hold a non-finite value (a
    // masked pixel), and 0 x NaN would reach the sums through the tensor core.
    for (int r = tid; r < kKC; r += blockDim.x) {
      const int64_t row = r0 + r;
      float wr = 0.0f;
      if (r < rows && (bulk_c ? rv[r] : a.R.valid[row]) && a.accepted[row / a.SS])
        wr = static_cast<float>(bulk_c ? rw[r] : a.R.w[row]);
      w_s[r] = wr;
    }
    __syncthreads();
    {
      const int lane = tid & 31, qmax = nf > a.k ? nf : a.k;
      for (int g = tid >> 5; g < kKC / 4; g += blockDim.x >> 5) {
        for (int q = lane; q < qmax; q += 32) {
          float bv[4], dv[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int r = 4 * g + i;
            const int64_t row = r0 + r;
            const bool in = r < rows && w_s[r] != 0.0f;
            bv[i] = 0.0f;
            dv[i] = 0.0f;
            if (in && q < nf)
              bv[i] = q < a.nc ? static_cast<float>(bulk_c ? rbn[r * a.nc + q] : a.R.bn[row * a.nc + q]) : 1.0f;
            if (in && q < a.k) dv[i] = static_cast<float>(bulk_c ? rd[r * a.k + q] : a.R.d[row * a.k + q]);
          }
          if (q < nf) *reinterpret_cast<float4*>(bnT + q * kRS + 4 * g) = make_float4(bv[0], bv[1], bv[2], bv[3]);
          if (q < a.k) {
            const float4 w4 = *reinterpret_cast<const float4*>(w_s + 4 * g);
            *reinterpret_cast<float4*>(dT + q * kRS + 4 * g) = make_float4(dv[0], dv[1], dv[2], dv[3]);
            *reinterpret_cast<float4*>(wdT + q * kRS + 4 * g) =
                make_float4(w4.x * dv[0], w4.y * dv[1], w4.z * dv[2], w4.w * dv[3]);
          }
        }
      }
    }
    // The MMAs of chunk c-2 read this stage: wait for their commit.
    if (c >= 2 && !mbar_wait(&mbar[st], static_cast<unsigned>((c - 2) >> 1) & 1u)) s_fail = 1;
    __syncthreads();
    if (s_fail) break;
    // A = U tile (kBM x kKC), 8 consecutive rows (one 16-byte store) per item;
    // consecutive threads take consecutive tile rows (conflict-free stores).
    for (int item = tid; item < kBM * (kKC / 8); item += blockDim.x) {
      const int m = (item & 7) + ((item >> 3) / (kKC / 8)) * 8;
      const int kg = (item >> 3) % (kKC / 8);
      const int2 p = up_s[m];
      float v[8];
      if (p.x >= 0) {
        const float4* x = reinterpret_cast<const float4*>(bnT + p.x * kRS + kg * 8);
        const float4* y = reinterpret_cast<const float4*>(bnT + p.y * kRS + kg * 8);
        const float4 x0 = x[0], x1 = x[1], y0 = y[0], y1 = y[1];
        v[0] = x0.x * y0.x; v[1] = x0.y * y0.y; v[2] = x0.z * y0.z; v[3] = x0.w * y0.w;
        v[4] = x1.x * y1.x; v[5] = x1.y * y1.y; v[6] = x1.z * y1.z; v[7] = x1.w * y1.w;
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = 0.0f;
      }
      if (kTf32)
        tf32_store(ahi, canon_off_tf32(m, kg), v);
      else
        split_store(ahi, alo, canon_off(m, kg), v);
    }
    // B = V tile (BN x kKC): (w d_m) d_m'.
    for (int item = tid; item < BN * (kKC / 8); item += blockDim.x) {
      const int n = (item & 7) + ((item >> 3) / (kKC / 8)) * 8;
      const int kg = (item >> 3) % (kKC / 8);
      const int2 q = vp_s[n];
      float v[8];
      if (q.x >= 0) {
        const float4* x = reinterpret_cast<const float4*>(wdT + q.x * kRS + kg * 8);
        const float4* y = reinterpret_cast<const float4*>(dT + q.y * kRS + kg * 8);
        const float4 x0 = x[0], x1 = x[1], y0 = y[0], y1 = y[1];
        v[0] = x0.x * y0.x; v[1] = x0.y * y0.y; v[2] = x0.z * y0.z; v[3] = x0.w * y0.w;
        v[4] = x1.x * y1.x; v[5] = x1.y * y1.y; v[6] = x1.z * y1.z; v[7] = x1.w * y1.w;
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = 0.0f;
      }
      if (kTf32)
        tf32_store(bhi, canon_off_tf32(n, kg), v);
      else
        split_store(bhi, blo, canon_off(n, kg), v);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t ah = smem_addr(ahi), al = smem_addr(alo);
      const uint32_t bh = smem_addr(bhi), bl = smem_addr(blo);
      if (kTf32) {
        // K-steps of 8 TF32 values: 32 bytes per row, two core matrices.
#pragma unroll
        for (int s = 0; s < kKC / 8; ++s) {
          const uint32_t ko = static_cast<uint32_t>(s) * 256;
          const uint32_t acc0 = (c % kDrainChunks != 0 || s > 0) ? 1u : 0u;
          umma_tf32(tmem, umma_desc(ah + ko, kLBO, kSBO), umma_desc(bh + ko, kLBO, kSBO), idesc, acc0);
        }
      } else {
#pragma unroll
        for (int s = 0; s < kKC / 16; ++s) {
          const uint32_t ko = static_cast<uint32_t>(s) * 256;  // two core matrices per K-step of 16
          const uint32_t acc0 = (c % kDrainChunks != 0 || s > 0) ? 1u : 0u;
          umma_bf16(tmem, umma_desc(ah + ko, kLBO, kSBO), umma_desc(bh + ko, kLBO, kSBO), idesc, acc0);
          umma_bf16(tmem, umma_desc(ah + ko, kLBO, kSBO), umma_desc(bl + ko, kLBO, kSBO), idesc, 1u);
          umma_bf16(tmem, umma_desc(al + ko, kLBO, kSBO), umma_desc(bh + ko, kLBO, kSBO), idesc, 1u);
        }
      }
      umma_commit(&mbar[st]);
    }
    issued = c + 1;
    if (issued % kDrainChunks == 0 && issued < nchunks) {
      // Chunk c's commit covers every MMA of this chain; the next chunk's
      // MMAs overwrite the accumulator only after the barrier below.
      if (!mbar_wait(&mbar[st], static_cast<unsigned>(c >> 1) & 1u)) s_fail = 1;
      __syncthreads();
      if (s_fail) break;
      tc_fence_after();
      drain(issued == kDrainChunks, true);
      tc_fence_before();
      __syncthreads();
    }
  }

  // Drain: wait for the most recent commit of each stage (the ones not waited
  // in the loop); together they cover every MMA issued.
  bool ok = !s_fail;
  for (int c = max(0, issued - 2); c < issued; ++c)
    if (!mbar_wait(&mbar[c & 1], static_cast<unsigned>(c >> 1) & 1u)) ok = false;
  // Row loads still in flight (only after an early exit): wait for them too.
  for (int c = ld_done + 1; c <= ld_hi; ++c)
    if (!mbar_wait(&mbar[2 + (c & 1)], static_cast<unsigned>(c >> 1) & 1u)) ok = false;
  __syncthreads();
  if (!ok && tid == 0) atomicOr(a.status, kStatusLoopLimit);
  tc_fence_after();

  // Epilogue: the last chain (stores when it is the only one; zeros after a
  // failure, which the status bit reports).
  if (issued > 0 && ok)
    drain(issued <= kDrainChunks, true);
  else
    drain(true, false);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tmem_cols) : "memory");
  }
}

}  // namespace

size_t normal_tc_smem(int nc, int k, int BN) {
  const size_t a_bytes = static_cast<size_t>(kBM) * kKC * 2, b_bytes = static_cast<size_t>(BN) * kKC * 2;
  size_t s = 4 * a_bytes + 4 * b_bytes;
  s += sizeof(float) * (static_cast<size_t>(kRS) * ((nc + 1) + 2 * static_cast<size_t>(k)) + kKC);
  s += sizeof(int2) * (kBM + BN + (BN & 1));
  s = (s + 7) / 8 * 8 + 4 * sizeof(uint64_t) + 16;
  s += 16 + 2 * (static_cast<size_t>(kKC) * (nc + k + 1) * 8 + kKC);  // aligned raw row buffers
  return s;
}

namespace {

// G[u][v] = sum over the splits z (in order) of the tiled partials.
__global__ void k_reduce_tiles(int nsplit, size_t split_len, int BN, int tiles_n, int Mu, int Nv,
                               const double* __restrict__ gpart, double* __restrict__ g) {
  for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < split_len;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int m = static_cast<int>(i % kBM);
    const size_t cv = i / kBM;
    const int col = static_cast<int>(cv % BN);
    const int tile = static_cast<int>(cv / BN);
    const int u = (tile / tiles_n) * kBM + m, v = (tile % tiles_n) * BN + col;
    if (u >= Mu || v >= Nv) continue;
    double s = 0.0;
    for (int z = 0; z < nsplit; ++z) s += gpart[static_cast<size_t>(z) * split_len + i];
    g[static_cast<size_t>(u) * Nv + v] = s;
  }
}

}  // namespace

// G of the tensor-core paths (row-major Mu x Nv, FP64): BF16x3 ("mixed") or TF32.
void launch_normal_tc(Context& c, int64_t N, int nc, int k, int SS, const FitRows& R, const uint8_t* accepted,
                      const int2* upairs, int Mu, const int2* vpairs, int Nv, Slot gpart_slot, double* g, bool tf32) {
  // Widest N tile (<= 256) whose staging fits; wide fits (many components and
  // knots) trade a narrower B tile for more column tiles.
  int tiles_n = (Nv + 255) / 256, BN = 0;
  size_t smem = 0;
  for (;; ++tiles_n) {
    BN = ((Nv + tiles_n - 1) / tiles_n + 15) / 16 * 16;
    smem = normal_tc_smem(nc, k, BN);
    if (smem <= 227 * 1024 || BN <= 16) break;
  }
  const int tiles_m = (Mu + kBM - 1) / kBM;
  const int tmem_cols = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
  if (smem > 227 * 1024) fail(DGPU_ERR_INVALID, "fit_kernel: mixed-precision tile does not fit in shared memory");
  const int64_t chunks = (N + kKC - 1) / kKC;
  const int64_t want = std::max<int64_t>(1, 148 / std::max(1, tiles_m * tiles_n));
  int64_t rps = ((chunks + want - 1) / want) * kKC;
  rps = std::max<int64_t>(rps, kKC);
  const int nsplit = static_cast<int>(std::max<int64_t>(1, (N + rps - 1) / rps));
  const size_t split_len = static_cast<size_t>(tiles_m) * tiles_n * BN * kBM;
  double* gpart = static_cast<double*>(c.slot(gpart_slot, sizeof(double) * nsplit * split_len));
  TcArgs a;
  a.N = N;
  a.nc = nc;
  a.k = k;
  a.SS = SS;
  a.R = R;
  a.accepted = accepted;
  a.upairs = upairs;
  a.Mu = Mu;
  a.vpairs = vpairs;
  a.Nv = Nv;
  a.BN = BN;
  a.tmem_cols = tmem_cols;
  a.rows_per_split = rps;
  a.gpart = gpart;
  a.status = c.d_status;
  auto al16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
  a.bulk = al16(R.bn) && al16(R.d) && al16(R.w) && al16(R.valid) && (static_cast<size_t>(kKC) * nc * 8) % 16 == 0 &&
           (static_cast<size_t>(kKC) * k * 8) % 16 == 0;
  if (tf32) {
    ensure_dynamic_smem(reinterpret_cast<const void*>(k_normal_tc<true>), smem);
    k_normal_tc<true><<<dim3(tiles_m, tiles_n, nsplit), kThreads, smem, c.stream>>>(a);
  } else {
    ensure_dynamic_smem(reinterpret_cast<const void*>(k_normal_tc<false>), smem);
    k_normal_tc<false><<<dim3(tiles_m, tiles_n, nsplit), kThreads, smem, c.stream>>>(a);
  }
  DGPU_LAUNCH("k_normal_tc");
  const int rb = static_cast<int>(std::min<size_t>(148 * 4, (split_len + 255) / 256));
  k_reduce_tiles<<<rb, 256, 0, c.stream>>>(nsplit, split_len, BN, tiles_n, Mu, Nv, gpart, g);
  DGPU_LAUNCH("k_reduce_tiles");
}

}  // namespace dgpu
