// Onesweep radix sort entry points (see sort.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace mrb {

// Scratch bytes for sorting up to maxCount pairs of keyBytes-wide keys.
size_t radix_sort_temp_bytes(uint32_t maxCount, int keyBytes, int beginBit, int endBit);

// Stable sort of (keys, vals) on bits [beginBit, endBit).  The count is read
// from dCount on the device when it is non-null (maxCount bounds it), else
// maxCount is the count.  valsAreIota: vals are generated as 0..n-1 on the
// first pass instead of being read.  Returns 0, or -1 with set_error().
template <class K>
int radix_sort_pairs(K* keys, uint32_t* vals, const uint32_t* dCount, uint32_t maxCount,
                     int beginBit, int endBit, bool desc, void* temp, size_t tempBytes,
                     cudaStream_t stream, bool valsAreIota);

// Device word set to 1 when a look-back wait gave up (never expected).
uint32_t* radix_sort_error_flag(void* temp, uint32_t maxCount);

}  // namespace mrb
