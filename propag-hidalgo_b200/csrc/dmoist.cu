// Hourly dead fuel moisture per cell (the dmoist model,
// crates/dmoist/src/lib.rs:55-715) from per-cell weather rasters, ahead of
// the fire-behaviour pass.
//
// One thread per cell.  The 1-h moisture of an hour needs only that hour's
// weather; the 10-h class interpolates the 1-h values of the requested hour
// and of hours 6 and 15, and the 100-h class does the same on the 10-h
// values (lib.rs:109-127) -- so a cell reads the weather of three hours, not
// 24.  The model's look-up tables are copied to shared memory per block
// (per-lane indices would serialise constant-memory reads).  Float
// operations follow the reference's order; this file is compiled without
// FMA contraction, explicit __fmaf_rn where the portable arctangent uses
// fused multiply-adds, so results equal the CPU restatement bit for bit.
#include <cuda_runtime.h>

#include <cstdint>

#include "dmoist_device.cuh"

namespace propag {

__global__ void __launch_bounds__(256) dmoist_kernel(DmoistIn in, uint64_t n, int hour, int month,
                                                     float scale, float *__restrict__ d1,
                                                     float *__restrict__ d10,
                                                     float *__restrict__ d100) {
  __shared__ DmoistTables T;
  load_dmoist_tables(T);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    float m1, m10, m100;
    dmoist_cell(T, in, n, i, hour, month, __ldg(in.fuel + i), __ldg(in.slope + i), __ldg(in.aspect + i),
                m1, m10, m100);
    d1[i] = m1 * scale;
    d10[i] = m10 * scale;
    d100[i] = m100 * scale;
  }
}

cudaError_t launch_dmoist(uint64_t n, int hour, int month, const float *t, const float *rh,
                          const float *cc, const float *pp, const float *slope, const float *aspect,
                          const uint8_t *fuel, float scale, float *d1, float *d10, float *d100,
                          int sm_count, cudaStream_t stream) {
  DmoistIn in{t, rh, cc, pp, slope, aspect, fuel};
  uint64_t blocks = (n + 255) / 256;
  const uint64_t cap = (uint64_t)sm_count * 8;
  if (blocks > cap) blocks = cap;
  if (blocks == 0) blocks = 1;
  dmoist_kernel<<<(unsigned)blocks, 256, 0, stream>>>(in, n, hour, month, scale, d1, d10, d100);
  return cudaGetLastError();
}

}  // namespace propag
