// team.cuh -- execution teams, device arena and warp helpers.
//
// Every solver phase is written once against a Team:
//   BlockTeam : the threads of one CTA (small instances, one instance per CTA
//               in a batch); sync() is __syncthreads().
//   GridTeam  : every thread of a cooperative grid (one large instance);
//               sync() is a grid-wide barrier.
//   ClusterTeam: the CTAs of one thread-block cluster (mid-size instances,
//               several at once); sync() is the hardware cluster barrier.
//               The hardware schedules a cluster's CTAs together, so its
//               members may wait on one another like a grid's.
// Work decomposition inside a phase uses only rank()/size() (grid-stride) or
// block()/nblocks() (one contiguous chunk per CTA, for order-preserving scans,
// compactions and sorts), so the same code is correct for every team and its
// results do not depend on the team size.
#pragma once
#include <cooperative_groups.h>
#include <cstdint>

namespace rama {
namespace cg = cooperative_groups;

struct BlockTeam {
    __device__ __forceinline__ int rank() const { return threadIdx.x; }
    __device__ __forceinline__ int size() const { return blockDim.x; }
    __device__ __forceinline__ int block() const { return 0; }
    __device__ __forceinline__ int nblocks() const { return 1; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    __device__ __forceinline__ bool leader() const { return threadIdx.x == 0; }
};

struct ClusterTeam {
    __device__ __forceinline__ int rank() const { return (int)cg::this_cluster().block_rank() * blockDim.x + threadIdx.x; }
    __device__ __forceinline__ int size() const { return (int)cg::this_cluster().num_blocks() * blockDim.x; }
    __device__ __forceinline__ int block() const { return (int)cg::this_cluster().block_rank(); }
    __device__ __forceinline__ int nblocks() const { return (int)cg::this_cluster().num_blocks(); }
    __device__ __forceinline__ void sync() const { cg::this_cluster().sync(); }
    __device__ __forceinline__ bool leader() const { return cg::this_cluster().block_rank() == 0 && threadIdx.x == 0; }
};

struct GridTeam {
    __device__ __forceinline__ int rank() const { return blockIdx.x * blockDim.x + threadIdx.x; }
    __device__ __forceinline__ int size() const { return gridDim.x * blockDim.x; }
    __device__ __forceinline__ int block() const { return blockIdx.x; }
    __device__ __forceinline__ int nblocks() const { return gridDim.x; }
    __device__ __forceinline__ void sync() const { cg::this_grid().sync(); }
    __device__ __forceinline__ bool leader() const { return blockIdx.x == 0 && threadIdx.x == 0; }
};

// Loads of values written by other threads before the last team sync.
template <class T>
__device__ __forceinline__ T uread(const T *p)
{
    return *(const volatile T *)p;
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ int warp_in_block() { return threadIdx.x >> 5; }
__device__ __forceinline__ unsigned lanemask_lt() { return (1u << lane_id()) - 1u; }

template <class Team>
__device__ __forceinline__ int team_warp(const Team &t)
{
    return t.rank() >> 5;
}
template <class Team>
__device__ __forceinline__ int team_nwarps(const Team &t)
{
    return t.size() >> 5;
}

// Status bits written into the instance's error word.
enum : int32_t {
    ERR_NONE = 0,
    ERR_INVALID_ARG = 1,
    ERR_ARENA = 2,       // device arena exhausted
    ERR_ITER_LIMIT = 4,  // a bounded device loop gave up
    ERR_BAD_CONTRACTION = 8,
};

// Device arena: every thread of a team holds an identical copy and performs
// identical (team-uniform) allocations, so no synchronisation is needed to
// allocate.  Temporaries grow upward from `lo`; the current graph lives at the
// top end, [top, cap).  An allocation that does not fit flags ERR_ARENA and
// returns a dummy pointer into the (always allocated) guard area; callers
// check `ok()` (team-uniformly) before touching the memory.
struct Arena {
    char *base;
    uint64_t lo;   // first free byte above the temporaries
    uint64_t top;  // first byte of the graph slot
    uint64_t cap;  // usable bytes (a guard area of 256 B follows)
    uint64_t peak;
    uint64_t want;  // workspace bytes the largest refused allocation needed (0: none refused)
    int failed;

    __device__ __forceinline__ bool ok() const { return !failed; }
    template <class T>
    __device__ __forceinline__ T *take(uint64_t n)
    {
        uint64_t a = (lo + 255) & ~uint64_t(255);
        uint64_t e = a + n * sizeof(T);
        if (failed || e > top) {
            // the temporaries up to e, the graph slot above them and the guard
            const uint64_t need = e + (cap - top) + 512;
            if (!failed && need > want) want = need;
            failed = 1;
            return reinterpret_cast<T *>(base + cap);  // guard area
        }
        lo = e;
        if (lo > peak) peak = lo;
        return reinterpret_cast<T *>(base + a);
    }
    __device__ __forceinline__ uint64_t mark() const { return lo; }
    __device__ __forceinline__ void release(uint64_t m) { lo = m; }
};

// A float -> uint32 map that preserves order (for packed min/max keys).
__device__ __forceinline__ uint32_t float_ordered(float f)
{
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ int bits_for(uint64_t maxval)
{
    return maxval == 0 ? 0 : 64 - __clzll((long long)maxval);
}

}  // namespace rama
