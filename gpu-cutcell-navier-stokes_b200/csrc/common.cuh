// Shared device utilities: status codes, bounded grid barrier, deterministic
// block / grid reductions, storage-type conversions.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/cutcell_b200.h"

#ifndef CUTCELL_BLOCK
#define CUTCELL_BLOCK 256
#endif
#define CUTCELL_WARPS (CUTCELL_BLOCK / 32)

// Grid barrier wait limit in SM clock cycles (about one second at 2 GHz).  A
// barrier that runs out sets CUTCELL_E_BARRIER and every block leaves its loop.
#define CUTCELL_BARRIER_CYCLES 2000000000LL

struct GridSync {
    unsigned* count;  // arrival word (own 128-byte line); its top bit flips once per barrier
    unsigned* gen;    // unused (kept for layout compatibility)
    int* err;         // error word (own 128-byte line)
    unsigned nblocks;
};

__device__ __forceinline__ int grid_error(const GridSync& gs) {
    return *((volatile int*)gs.err);
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned atom_add_release_u32(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Grid barrier for a cooperative (co-resident) grid: every block adds to one
// arrival word, block 0 adds 2^31 - (nblocks - 1) so the word's top bit flips
// exactly when the last block arrives; waiters poll the word with acquire
// loads.  No reset is needed between barriers.  Every wait is bounded: after
// CUTCELL_BARRIER_CYCLES the error word is set and all blocks leave their loops.
// Ordering: the block barrier makes the block's writes precede thread 0's
// release add (release is cumulative); the acquire load that sees the flip
// and the closing block barrier make every other block's writes visible to
// all threads, without full fences on either side.
__device__ __forceinline__ bool grid_sync(const GridSync& gs) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned add = (blockIdx.x == 0) ? (0x80000000u - (gs.nblocks - 1u)) : 1u;
        const unsigned old = atom_add_release_u32(gs.count, add);
        long long t0 = clock64();
        unsigned spins = 0;
        while (((old ^ ld_acquire_u32(gs.count)) & 0x80000000u) == 0u) {
            if ((++spins & 1023u) == 0u) {
                if (clock64() - t0 > CUTCELL_BARRIER_CYCLES) {
                    atomicExch(gs.err, CUTCELL_E_BARRIER);
                    break;
                }
                if (*((volatile int*)gs.err) != 0) break;
            }
        }
    }
    __syncthreads();
    return grid_error(gs) == 0;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum (fixed tree); result broadcast to all threads.
// ``sh`` needs CUTCELL_WARPS doubles.
__device__ __forceinline__ double block_sum(double v, double* sh) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = (threadIdx.x < CUTCELL_WARPS) ? sh[threadIdx.x] : 0.0;
    if (w == 0) t = warp_sum(t);
    if (threadIdx.x == 0) sh[0] = t;
    __syncthreads();
    double r = sh[0];
    __syncthreads();
    return r;
}

// Sum of nblocks partials written at part[0..nblocks-1], in a fixed order so
// every block obtains the bit-identical value.
__device__ __forceinline__ double grid_reduce(const double* part, int nblocks, double* sh) {
    double s = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) s += ((volatile const double*)part)[i];
    return block_sum(s, sh);
}

// p_new = D^-1 r + beta p_old with one fixed rounding sequence, so a value
// formed on the fly is bit-identical to the stored one.
__device__ __forceinline__ double p_next(double dinv, double r, double beta, double pold) {
    return __fma_rn(beta, pold, __dmul_rn(dinv, r));
}

template <typename T> struct Conv;
// ld: read-only global load; sld: shared-memory load, both widened to acc
template <> struct Conv<double> {
    typedef double acc;
    __device__ __forceinline__ static double ld(const double* p) { return __ldg(p); }
    __device__ __forceinline__ static double sld(const double* p) { return *p; }
};
template <> struct Conv<float> {
    typedef float acc;
    __device__ __forceinline__ static float ld(const float* p) { return __ldg(p); }
    __device__ __forceinline__ static float sld(const float* p) { return *p; }
};
template <> struct Conv<__nv_bfloat16> {
    typedef float acc;
    __device__ __forceinline__ static float ld(const __nv_bfloat16* p) { return __bfloat162float(*p); }
    __device__ __forceinline__ static float sld(const __nv_bfloat16* p) { return __bfloat162float(*p); }
};

// Optional self-checks (build with -DCUTCELL_DEBUG_CHECKS): a failed check
// records (code, info) in two debug words and the guarded access is skipped.
#ifdef CUTCELL_DEBUG_CHECKS
__device__ __forceinline__ bool dbg_ok(bool cond, unsigned code, unsigned info, unsigned* words) {
    if (!cond && words) {
        if (atomicCAS(words, 0u, code) == 0u) atomicExch(words + 1, info);
    }
    return cond;
}
#define CUTCELL_OK_IF(cond, code, info, words) dbg_ok((cond), (code), (unsigned)(info), (words))
#else
#define CUTCELL_OK_IF(cond, code, info, words) true
#endif
#define CUTCELL_ALIGNED(p, a) ((((uintptr_t)(p)) % (a)) == 0)

static inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }
