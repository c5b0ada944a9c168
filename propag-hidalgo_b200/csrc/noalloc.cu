// Fixed device scratch for the allocation-free propagation entry point
// (propag_run_device_static in api.cpp).
//
// The scratch is one file-scope device array, reserved by the CUDA driver
// when this module is loaded; nothing is allocated per call.  Its layout:
//
//   [0, 256)        JobDev of the running job
//   [256, 512)      SlotDev (counters and list overflow: tiles run in shared memory)
//   [512, 768)      StatsDev
//   [768, 1024)     job queue counter
//   [1024, 1280)    slot counters
//   [2048, ...)     five per-cell arrays of kStaticMaxCells uint32 (references
//                   and the four referrer-box corners), then the boundary
//                   bitmap (kStaticMaxCells / 32 words), then the overflow of
//                   the shared-memory work and update lists
//                   (kStaticOvfSlots u16 entries, then kStaticOvfSlots Updates)
//
// The per-cell arrays are initialised by the boundary/initial-state pass of
// every call; the statistics, queue and counters are cleared by
// stage_static_kernel at the start of every call; list overflow entries are
// written before they are read within a sweep.  Nothing needs to be zero
// across calls.
#include <cuda_runtime.h>

#include "engine.cuh"
#include "noalloc.hpp"

namespace propag {

static_assert(sizeof(JobDev) <= 256, "JobDev exceeds its scratch slot");
static_assert(sizeof(SlotDev) <= 256, "SlotDev exceeds its scratch slot");
static_assert(sizeof(StatsDev) <= 256, "StatsDev exceeds its scratch slot");
static_assert(kStaticMaxCells % 32 == 0, "bitmap words");
static_assert(sizeof(Update) == 16, "overflow update entries are 16 bytes");
static_assert(kStaticOvfUpdOff % 16 == 0, "overflow updates are 16-byte aligned");

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

cudaError_t static_scratch_address(void **ptr) {
  return cudaGetSymbolAddress(ptr, g_static_scratch);
}

// Writes the job and slot descriptors into the scratch and clears the
// statistics, the job queue and the slot counters.
__global__ void stage_static_kernel(JobDev *dj, JobDev j, SlotDev *ds, SlotDev s, StatsDev *st,
                                    uint32_t *queue) {
  if (threadIdx.x == 0) {
    *dj = j;
    *ds = s;
    *st = StatsDev{};
    *queue = 0u;
  }
  if (threadIdx.x < kStaticCtrWords) s.ctr[threadIdx.x] = 0u;
}

cudaError_t launch_stage_static(JobDev *dj, const JobDev &j, SlotDev *ds, const SlotDev &s,
                                StatsDev *st, uint32_t *queue, cudaStream_t stream) {
  stage_static_kernel<<<1, 32, 0, stream>>>(dj, j, ds, s, st, queue);
  return cudaGetLastError();
}

}  // namespace propag
