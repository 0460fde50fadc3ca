// simt_host.hpp -- run CUDA-style kernels on host cores (test infrastructure).
//
// This header is part of the ORACLE, not of the product.  It lets the
// reference's own CUDA kernel sources (glide/cuda/*.cu, compiled unmodified as
// host C++) execute on the CPU so that the restated oracle and the golden
// fixtures can be pinned against the reference itself.
//
// Model: every CUDA thread of a block is a cooperative fiber with its own
// stack.  Fibers of one block run on one OS thread; __syncthreads() yields to
// a per-block scheduler which releases the barrier once every live fiber has
// reached it (fibers that returned early count as departed, which is how the
// reference's early returns before __syncthreads behave on the GPU).  Blocks
// are distributed over OS threads with OpenMP.  __shared__ storage maps to
// function-local `static thread_local` objects: one copy per OS thread, shared
// by the fibers of the block that thread is running.  Global atomics are
// compare-and-swap loops so concurrent blocks stay correct.
#pragma once

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <vector>

namespace simt {

struct uint3_ { unsigned x, y, z; };

struct Fiber {
    void* sp = nullptr;
    int state = 0;  // 0 ready, 1 at barrier, 2 done
    uint3_ tid{0, 0, 0};
};

struct BlockRun {
    std::vector<Fiber> fibers;
    void* sched_sp = nullptr;
    int cur = -1;
    const std::function<void()>* body = nullptr;
    uint3_ bid{0, 0, 0};
    uint3_ bdim{1, 1, 1};
    uint3_ gdim{1, 1, 1};
};

extern "C" void simt_switch(void** save_sp, void* load_sp);

inline BlockRun*& current_block() {
    static thread_local BlockRun* run = nullptr;
    return run;
}

inline const uint3_& tidx() { BlockRun* r = current_block(); return r->fibers[r->cur].tid; }
inline const uint3_& bidx() { return current_block()->bid; }
inline const uint3_& bdimv() { return current_block()->bdim; }
inline const uint3_& gdimv() { return current_block()->gdim; }

void barrier();
void launch(uint3_ grid, uint3_ block, const std::function<void()>& body);

template <class T>
inline T atomic_add(T* addr, T val) {
    T expected;
    __atomic_load(addr, &expected, __ATOMIC_RELAXED);
    T desired;
    do {
        desired = expected + val;
    } while (!__atomic_compare_exchange(addr, &expected, &desired, true,
                                        __ATOMIC_RELAXED, __ATOMIC_RELAXED));
    return expected;
}

}  // namespace simt

// ---- CUDA spellings used by the kernels --------------------------------
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __shared__ static thread_local
#define threadIdx (::simt::tidx())
#define blockIdx (::simt::bidx())
#define blockDim (::simt::bdimv())
#define gridDim (::simt::gdimv())
#define __syncthreads() ::simt::barrier()

using std::max;
using std::min;

inline float atomicAdd(float* a, float v) { return simt::atomic_add(a, v); }
inline double atomicAdd(double* a, double v) { return simt::atomic_add(a, v); }

// Fast-math intrinsics map to the correctly rounded host functions.  Overloads
// for double exist so that a build with `float` redefined as `double` keeps
// every operation in double precision.
inline float __powf(float a, float b) { return std::pow(a, b); }
inline double __powf(double a, double b) { return std::pow(a, b); }
inline float __expf(float a) { return std::exp(a); }
inline double __expf(double a) { return std::exp(a); }
inline float __logf(float a) { return std::log(a); }
inline double __logf(double a) { return std::log(a); }
inline float __fmaf_rn(float a, float b, float c) { return std::fma(a, b, c); }
inline double __fmaf_rn(double a, double b, double c) { return std::fma(a, b, c); }
