// Test infrastructure: runs CUDA kernel source on the host, so that the CPU
// tests can execute the device code of kernels without a GPU.
//
// The threads of a block are coroutines (ucontext) on one OS thread, run
// round-robin; blocks run one after another.  A thread runs until it reaches
// a barrier (__syncthreads, or a warp vote or shuffle, each treated as a
// barrier of the whole block) or returns; a round ends when every thread has
// done so, so no thread passes barrier k before all threads have reached it.
// That is exact for kernels whose threads all meet the same barriers in the
// same order -- the only kind emulated here.  __shared__ variables become
// statics (one block runs at a time); atomics are plain read-modify-writes
// (one thread runs at a time).  Only the built-ins the emulated kernels use
// are provided.  Include this before the kernel source and launch with
// emul::launch(grid, block, kernel, args...).
#pragma once

#include <ucontext.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <vector>

struct EmulDim3 {
  unsigned x, y, z;
};
inline EmulDim3 threadIdx, blockIdx, blockDim, gridDim;

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __launch_bounds__(...)
#define __restrict__ __restrict
#define __shared__ static

namespace emul {

struct Fiber {
  ucontext_t ctx;
  std::vector<char> stack;
  bool done = false;
};

inline ucontext_t scheduler;
inline std::vector<Fiber> fibers;
inline unsigned current = 0;
inline std::function<void()> body;
inline uint32_t warp_vote[32];
inline uint32_t slots[1024];

// Back to the scheduler until the next round.
inline void barrier() { swapcontext(&fibers[current].ctx, &scheduler); }

inline void entry() {
  body();
  fibers[current].done = true;
}

// kernel<<<grid, block>>>(args...), synchronously.  block: a multiple of 32, <= 1024.
template <typename K, typename... A>
void launch(unsigned grid, unsigned block, K kernel, A... args) {
  if (block == 0 || block > 1024 || block % 32) {
    std::fprintf(stderr, "emul::launch: unsupported block size %u\n", block);
    std::abort();
  }
  gridDim = {grid, 1, 1};
  blockDim = {block, 1, 1};
  body = [&] { kernel(args...); };
  if (fibers.size() < block) fibers.resize(block);
  for (unsigned b = 0; b < grid; ++b) {
    blockIdx = {b, 0, 0};
    for (unsigned t = 0; t < block; ++t) {
      Fiber &f = fibers[t];
      f.done = false;
      if (f.stack.size() < 128 * 1024) f.stack.resize(128 * 1024);
      getcontext(&f.ctx);
      f.ctx.uc_stack.ss_sp = f.stack.data();
      f.ctx.uc_stack.ss_size = f.stack.size();
      f.ctx.uc_link = &scheduler;
      makecontext(&f.ctx, entry, 0);
    }
    for (bool running = true; running;) {
      running = false;
      unsigned finished = 0;
      for (unsigned t = 0; t < block; ++t) {
        if (fibers[t].done) {
          ++finished;
          continue;
        }
        current = t;
        threadIdx = {t, 0, 0};
        swapcontext(&scheduler, &fibers[t].ctx);
        if (!fibers[t].done) running = true;
        else ++finished;
      }
      if (running && finished) {  // some threads returned while others wait at a barrier
        std::fprintf(stderr, "emul::launch: threads of a block met different barriers\n");
        std::abort();
      }
    }
  }
}

}  // namespace emul

template <class T>
inline T min(T a, T b) {
  return b < a ? b : a;
}
inline int __popc(uint32_t x) { return __builtin_popcount(x); }
#define __syncthreads() emul::barrier()

inline uint32_t __ballot_sync(uint32_t, bool p) {
  const unsigned lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  if (lane == 0) emul::warp_vote[warp] = 0;
  emul::barrier();
  if (p) emul::warp_vote[warp] |= 1u << lane;
  emul::barrier();
  const uint32_t r = emul::warp_vote[warp];
  emul::barrier();  // every lane has read the vote before the next one clears it
  return r;
}
inline uint32_t __shfl_xor_sync(uint32_t, uint32_t v, int lane_mask) {
  emul::slots[threadIdx.x] = v;
  emul::barrier();
  const uint32_t r = emul::slots[(threadIdx.x & ~31u) | ((threadIdx.x % 32) ^ (unsigned)lane_mask)];
  emul::barrier();
  return r;
}
inline int32_t atomicMax(int32_t *p, int32_t v) {
  const int32_t old = *p;
  if (v > old) *p = v;
  return old;
}
inline uint32_t atomicXor(uint32_t *p, uint32_t v) {
  const uint32_t old = *p;
  *p = old ^ v;
  return old;
}
