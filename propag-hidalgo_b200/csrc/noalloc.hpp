// Layout of the fixed device scratch of the allocation-free propagation
// entry point (noalloc.cu).
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace propag {

struct JobDev;
struct SlotDev;
struct StatsDev;

// Largest grid the fixed scratch holds: 1024 x 1024 cells (20 B per cell of
// references and referrer boxes, plus one boundary bit).
constexpr uint64_t kStaticMaxCells = 1ull << 20;
constexpr size_t kStaticJobOff = 0;
constexpr size_t kStaticSlotOff = 256;
constexpr size_t kStaticStatsOff = 512;
constexpr size_t kStaticQueueOff = 768;
constexpr size_t kStaticCtrOff = 1024;
constexpr int kStaticCtrWords = 16;
constexpr size_t kStaticCellsOff = 2048;
constexpr size_t kStaticArrayBytes = kStaticMaxCells * 4;
constexpr size_t kStaticBndOff = kStaticCellsOff + 5 * kStaticArrayBytes;
// Overflow of the shared-memory work and update lists: cluster size x cell
// slots per CTA entries (16 CTAs x 17 408 slots covers every tile whose
// shared-memory footprint fits the 200 KB budget).
constexpr size_t kStaticOvfSlots = 16 * 17408;
constexpr size_t kStaticOvfListOff = kStaticBndOff + kStaticMaxCells / 8;
constexpr size_t kStaticOvfUpdOff = kStaticOvfListOff + kStaticOvfSlots * 2;
constexpr size_t kStaticScratchBytes = kStaticOvfUpdOff + kStaticOvfSlots * 16;

// Device address of the scratch on the current device (cudaGetSymbolAddress).
cudaError_t static_scratch_address(void **ptr);

cudaError_t launch_stage_static(JobDev *dj, const JobDev &j, SlotDev *ds, const SlotDev &s,
                                StatsDev *st, uint32_t *queue, cudaStream_t stream);

}  // namespace propag
