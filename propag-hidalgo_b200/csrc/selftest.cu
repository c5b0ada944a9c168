// Element-wise views of the propagation's device arithmetic, for the tests
// that check it: time_from in either arithmetic, and tables of the two CUDA
// functions the reference's time_from calls (crates/propag/src/propag.cu:
// 269-294), so that a CPU restatement can use the device's own values.
#include <cuda_runtime.h>

#include <cstdint>

#include "propag_device.cuh"

namespace propag {

__global__ void time_from_kernel(bool refm, uint64_t n, const int32_t *fx, const int32_t *fy,
                                 const float *ftime, const int32_t *tx, const int32_t *ty,
                                 const float *smax, const float *azmax, const float *ecc,
                                 float gdx, float gdy, bool north_up, float *out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Fire f{smax[i], azmax[i], ecc[i]};
  out[i] = time_from(fx[i], fy[i], ftime[i], tx[i], ty[i], f, gdx, gdy, north_up, refm);
}

// out[i] = __cosf(x) for the float x whose bits are first + i.
__global__ void cosf_table_kernel(uint32_t first, uint64_t n, float *out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = __cosf(__uint_as_float(first + (uint32_t)i));
}

// out[(a + ma) + (b + mb) (2 ma + 1)] = atan2f(a, b) for integers |a| <= ma,
// |b| <= mb (rows b0 .. b0 + nb - 1 of the table).
__global__ void atan2f_table_kernel(int32_t ma, int32_t mb, int32_t b0, int32_t nb, float *out) {
  const int64_t w = 2 * (int64_t)ma + 1;
  const int64_t n = w * nb;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = (int32_t)(i % w) - ma;
    const int32_t b = b0 + (int32_t)(i / w) - mb;
    out[i] = atan2f((float)a, (float)b);
  }
}

cudaError_t launch_time_from(bool refm, uint64_t n, const int32_t *fx, const int32_t *fy,
                             const float *ftime, const int32_t *tx, const int32_t *ty,
                             const float *smax, const float *azmax, const float *ecc, float gdx,
                             float gdy, bool north_up, float *out, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  time_from_kernel<<<blocks, 256, 0, stream>>>(refm, n, fx, fy, ftime, tx, ty, smax, azmax, ecc,
                                               gdx, gdy, north_up, out);
  return cudaGetLastError();
}

cudaError_t launch_cosf_table(uint32_t first, uint64_t n, float *out, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  cosf_table_kernel<<<148 * 8, 256, 0, stream>>>(first, n, out);
  return cudaGetLastError();
}

cudaError_t launch_atan2f_table(int32_t ma, int32_t mb, int32_t b0, int32_t nb, float *out,
                                cudaStream_t stream) {
  if (nb <= 0) return cudaSuccess;
  atan2f_table_kernel<<<148 * 8, 256, 0, stream>>>(ma, mb, b0, nb, out);
  return cudaGetLastError();
}

}  // namespace propag
