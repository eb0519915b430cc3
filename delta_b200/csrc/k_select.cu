// Radix-select sample medians (select_internal.h): one compaction launch, then
// per 8-bit digit a grid-wide histogram whose last block picks the digit
// holding the rank. No host synchronisation: the count, the rank and the key
// prefix stay on the device.
#include <cuda_runtime.h>

#include <algorithm>

#include "dev_common.cuh"
#include "select_internal.h"

namespace dgpu {

// One reservation per block and sweep (a block-wide count of its finite,
// unmasked samples, then one atomicAdd): a reservation per warp put up to
// 8192 atomics on the one counter. The keys' order within the sample is free:
// only their multiset decides the median.
__global__ void __launch_bounds__(256) k_sample_keys(int64_t n, int64_t step, const float* __restrict__ v,
                                                     const uint8_t* __restrict__ mask, uint32_t* __restrict__ keys,
                                                     RadixSelect* st) {
  __shared__ unsigned warp_n[8];
  __shared__ unsigned block_base;
  const int64_t ns = (n + step - 1) / step;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t j0 = static_cast<int64_t>(blockIdx.x) * blockDim.x; j0 < ns;
       j0 += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t j = j0 + threadIdx.x;
    bool ok = false;
    float x = 0.0f;
    if (j < ns) {
      const int64_t i = j * step;
      x = v[i];
      ok = isfinite(x) && (mask == nullptr || mask[i] == 0);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, ok);
    if (lane == 0) warp_n[warp] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned tot = 0;
      for (int w = 0; w < 8; ++w) {
        const unsigned c = warp_n[w];
        warp_n[w] = tot;
        tot += c;
      }
      block_base = tot ? atomicAdd(&st->count, tot) : 0u;
    }
    __syncthreads();
    if (ok) keys[block_base + warp_n[warp] + __popc(bal & ((1u << lane) - 1))] = float_key(x);
    __syncthreads();  // warp_n and block_base are rewritten by the next sweep
  }
}

__global__ void k_select_init(RadixSelect* st) {
  st->rank = st->count / 2;
  st->prefix = 0;
  st->arrived = 0;
  for (int i = threadIdx.x; i < 256; i += blockDim.x) st->hist[i] = 0;
}

// One warp of the last block to finish a histogram pass: each lane sums 8
// bins, a warp prefix sum finds the lane whose bins hold the rank, that lane
// walks its 8, and the histogram is cleared for the next pass.
__device__ void select_pick_warp(RadixSelect* st, int shift, float* result, int last) {
  const int lane = threadIdx.x & 31;
  unsigned h[8];
  unsigned local = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    h[j] = __ldcg(&st->hist[lane * 8 + j]);  // every block's atomics, past the fence
    local += h[j];
  }
  unsigned incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  const unsigned excl = incl - local;
  const unsigned rank = st->rank;
  // The lane holding the rank (the last lane when the rank is past every bin,
  // which leaves digit 255 as a sequential scan would).
  const bool here = (rank >= excl && rank < incl) || (lane == 31 && rank >= incl);
  const unsigned who = __ballot_sync(0xffffffffu, here);
  __syncwarp();
  if (lane == __ffs(who) - 1) {
    unsigned cum = excl;
    int digit = lane * 8 + 7;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (rank < cum + h[j]) {
        digit = lane * 8 + j;
        break;
      }
      cum += h[j];
    }
    st->rank = rank - cum;
    st->prefix |= static_cast<unsigned>(digit) << shift;
    if (last) *result = st->count ? key_float(st->prefix) : 0.0f;
  }
#pragma unroll
  for (int j = 0; j < 8; ++j) st->hist[lane * 8 + j] = 0;
  if (lane == 0) st->arrived = 0;
}

// One radix pass: per-block histograms added into st->hist; the last block to
// arrive (after a fence, so it sees every block's additions) picks the digit.
__global__ void k_select_hist(const uint32_t* __restrict__ keys, RadixSelect* st, int shift, float* result, int last) {
  __shared__ unsigned hist[256];
  __shared__ bool is_last;
  for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  const unsigned count = st->count, prefix = st->prefix;
  const unsigned himask = shift >= 24 ? 0u : (0xffffffffu << (shift + 8));
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const uint32_t k = keys[i];
    if ((k & himask) == (prefix & himask)) atomicAdd(&hist[(k >> shift) & 0xffu], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (hist[i]) atomicAdd(&st->hist[i], hist[i]);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) is_last = atomicAdd(&st->arrived, 1u) == gridDim.x - 1;
  __syncthreads();
  if (is_last && threadIdx.x < 32) {
    __threadfence();
    select_pick_warp(st, shift, result, last);
  }
}

void launch_sample_keys(cudaStream_t s, int64_t n, int64_t step, const float* v, const uint8_t* mask, uint32_t* keys,
                        RadixSelect* st) {
  const int64_t ns = (n + step - 1) / step;
  const int blocks = static_cast<int>(std::min<int64_t>((std::max<int64_t>(ns, 1) + 255) / 256, 148 * 8));
  k_sample_keys<<<blocks, 256, 0, s>>>(n, step, v, mask, keys, st);
  DGPU_LAUNCH("k_sample_keys");
}

void launch_select_upper_median(cudaStream_t s, RadixSelect* st, const uint32_t* keys, int64_t cap, float* out) {
  k_select_init<<<1, 256, 0, s>>>(st);
  DGPU_LAUNCH("k_select_init");
  const int hb = static_cast<int>(std::min<int64_t>((std::max<int64_t>(cap, 1) + 1023) / 1024, 148 * 2));
  for (int pass = 0; pass < 4; ++pass) {
    k_select_hist<<<hb, 256, 0, s>>>(keys, st, 24 - 8 * pass, out, pass == 3);
    DGPU_LAUNCH("k_select_hist");
  }
}

}  // namespace dgpu
