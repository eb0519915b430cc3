// Exact sample medians on the device by radix select: the sample is compacted
// into monotone uint32 keys (float_key), then four 8-bit histogram passes find
// the element of rank count / 2 -- the value std::nth_element(count / 2)
// returns. Shared by the subtraction's fill values (src/subtract.cpp:20-51,
// 915-945) and stamp selection's background and MAD (src/detect.cpp:100-112).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace dgpu {

struct RadixSelect {
  unsigned count;   // keys in the sample
  unsigned rank;    // remaining rank within the current prefix bucket
  unsigned prefix;  // key bits fixed so far
  unsigned arrived;  // blocks done with the current histogram pass
  unsigned hist[256];
};

// Appends the keys of the finite values v[j * step] whose mask byte is 0 (any
// value when mask is null) to keys, counting them in st->count, which the
// caller has zeroed. keys must hold ceil(n / step) entries.
void launch_sample_keys(cudaStream_t s, int64_t n, int64_t step, const float* v, const uint8_t* mask, uint32_t* keys,
                        RadixSelect* st);

// *out = the key of rank st->count / 2 among keys[0 .. st->count) as a float
// (0 for an empty sample); cap bounds st->count. Leaves st->count as it was.
void launch_select_upper_median(cudaStream_t s, RadixSelect* st, const uint32_t* keys, int64_t cap, float* out);

}  // namespace dgpu
