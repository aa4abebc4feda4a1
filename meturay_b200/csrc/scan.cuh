// Device-wide exclusive prefix sum (see scan.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace mrb {
size_t exclusive_scan_temp_bytes(uint32_t n);
// out[0..n]: out[i] = sum(in[0..i)), out[n] = total.  out needs n + 1 words.
int exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, void* temp,
                       cudaStream_t stream);
}  // namespace mrb
