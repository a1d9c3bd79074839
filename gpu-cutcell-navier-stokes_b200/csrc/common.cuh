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

// Grid barrier wait limit.  Waits are measured on the device's global timer
// (wall-clock nanoseconds, unaffected by SM clocks or by a block being
// descheduled), and the limit is a runtime value carried in GridSync: the
// library default is 10 s, changed by cutcell_set_wait_limit or by the
// environment variable CUTCELL_WAIT_LIMIT_S read at the first launch.  A
// barrier that runs out sets CUTCELL_E_BARRIER and every block leaves its loop.
#define CUTCELL_DEFAULT_WAIT_LIMIT_S 10.0

// Host side: the current limit in nanoseconds (defined in cutcell.cu).
unsigned long long cutcell_internal_wait_limit_ns();

struct GridSync {
    unsigned* count;  // arrival word (own 128-byte line); its top bit flips once per barrier
    unsigned long long limit_ns;  // bounded-wait limit (global-timer nanoseconds)
    int* err;         // error word (own 128-byte line)
    unsigned nblocks;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

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
// gs.limit_ns of global time the error word is set and all blocks leave their loops.
// Ordering: the block barrier makes the block's writes precede thread 0's
// release add (release is cumulative); the acquire load that sees the flip
// and the closing block barrier make every other block's writes visible to
// all threads, without full fences on either side.
__device__ __forceinline__ bool grid_sync(const GridSync& gs) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned add = (blockIdx.x == 0) ? (0x80000000u - (gs.nblocks - 1u)) : 1u;
        const unsigned old = atom_add_release_u32(gs.count, add);
        const unsigned long long t0 = global_ns();
        unsigned spins = 0;
        while (((old ^ ld_acquire_u32(gs.count)) & 0x80000000u) == 0u) {
            if ((++spins & 1023u) == 0u) {
                if (global_ns() - t0 > gs.limit_ns) {
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

// z = z0 + zx[0] + ... + zx[nx - 1], added in that order: the two-level form
// keeps each patch tiling's correction in its own vector (every tiling writes
// every reduced DOF, so they cannot share one within a phase)
#define ZSUM_MAX 3
struct ZSum {
    const double* z0;
    const double* zx[ZSUM_MAX];
    int nx;
    __device__ __forceinline__ double at(int j) const {
        double s = __ldcg(z0 + j);
        for (int i = 0; i < nx; ++i) s = __dadd_rn(s, __ldcg(zx[i] + j));
        return s;
    }
};

// p_new = z + beta p_old with z a ZSum, one fixed rounding sequence
__device__ __forceinline__ double p_next_sum(const ZSum& z, int j, double beta, double pold) {
    return __fma_rn(beta, pold, z.at(j));
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

// Two-plane BF16 storage of the BF16 operator form: a value v is kept as
// hi = bf16(v) and lo = bf16(v - hi), 4 bytes, read back as float(hi) +
// float(lo) (about 16 significant bits) and accumulated in FP32.  One BF16
// plane alone (8 bits) perturbs the weak-penalty cut blocks, whose Nitsche
// penalty entries are two orders of magnitude above their stiffness entries,
// by more than the smallest eigenvalues of the Jacobi-scaled system, and the
// refinement then stagnates.
struct __align__(4) bf16x2_t {
    __nv_bfloat16 hi, lo;
};
template <> struct Conv<bf16x2_t> {
    typedef float acc;
    __device__ __forceinline__ static float unpack(unsigned u) {
        return __uint_as_float(u << 16) + __uint_as_float(u & 0xffff0000u);
    }
    __device__ __forceinline__ static float ld(const bf16x2_t* p) {
        return unpack(__ldg(reinterpret_cast<const unsigned*>(p)));
    }
    __device__ __forceinline__ static float sld(const bf16x2_t* p) {
        return unpack(*reinterpret_cast<const unsigned*>(p));
    }
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
