// Test stand-in for the product-sampler harness (psamp_harness.cu): the
// medium types that ProductSampler.cuh names, with nothing behind them (the
// stand-in surface ignores media).
#pragma once
#include <cstdint>

class GPUMediumI {};

class GPUMediumVacuum : public GPUMediumI {
  public:
    __host__ __device__ explicit GPUMediumVacuum(uint32_t) {}
};
