// kernels.cuh -- launch descriptors and declarations of the solver kernels.
//
// Each kernel lives in a translation unit of its own (k_*.cu), so the units
// compile in parallel and each kernel is still optimised as a whole; capi.cu
// holds the host side and launches them through these declarations.
#pragma once
#include "../../include/rama_b200.h"
#include "solver.cuh"

namespace rama {

constexpr int THREADS = 512;
constexpr int SMEM = sort_smem_bytes(THREADS) + 1024;
static_assert(THREADS / 32 * 1024 + BUCKET_MAX * 12 <= sort_smem_bytes(THREADS),
              "the CTA bucket sort's staging area fits");
// the smaller CTA of k_solve_cta_small (the autotuner chooses between the two
// for CTA-team solves); its shared memory also holds a CTA bucket sort of
// BUCKET_MAX items
constexpr int THREADS_SMALL = 256;
constexpr int SMEM_SMALL = (sort_smem_bytes(THREADS_SMALL) > THREADS_SMALL / 32 * 1024 + BUCKET_MAX * 12
                                ? sort_smem_bytes(THREADS_SMALL)
                                : THREADS_SMALL / 32 * 1024 + BUCKET_MAX * 12) +
                           1024;

// persistent CTAs, one instance each (k_solve_cta)
struct CtaLaunch {
    Instance *inst;
    const int32_t *order;
    int32_t count;
    int32_t *queue;
};

// clusters draw instances first; queue entries [0, ncluster) are solved by a
// whole cluster, the rest by single CTAs (k_solve_mixed)
struct MixedLaunch {
    Instance *inst;
    const int32_t *order;
    int32_t count;
    int32_t ncluster;
    int32_t *queue;
};

// one instance on the cooperative grid (k_solve_grid)
struct GridLaunch {
    Instance *inst;
    char *ws;
    uint64_t ws_bytes;
};

// MULTICUT text -> triples on the cooperative grid (k_parse_grid)
struct ParseLaunch {
    const char *text;
    int64_t len;
    int32_t *i, *j;
    float *c;
    int64_t cap;
    int64_t *out;  // count, -1 bad first line, -2 workspace exhausted
    char *ws;
    uint64_t ws_bytes;
};

// device-side maximum node id of an edge list (k_max_id), and the objective
struct MaxIdLaunch {
    const int32_t *i, *j;
    int64_t n;
    int32_t *out;  // [0] max id (-1 if empty), [1] 1 if any id is negative
};

__device__ __forceinline__ Scratch make_scratch(char *base, uint64_t bytes) { return scratch_over(base, bytes); }

// persistent CTAs: each pulls instances from the queue (largest first) and
// solves them alone (BlockTeam)
__device__ __forceinline__ void solve_queue_by_cta(const CtaLaunch &L, char *sm, int *next)
{
    BlockTeam t;
    for (int guard = 0; guard < (1 << 30); ++guard) {
        if (threadIdx.x == 0) *next = atomicAdd(L.queue, 1);
        __syncthreads();
        const int k = *next;
        __syncthreads();
        if (k >= L.count) break;
        Instance *io = &L.inst[L.order[k]];
        Scratch sc = make_scratch(io->ws, io->ws_bytes);
        solve_instance(t, sm, sc, io);
        __syncthreads();
    }
}

}  // namespace rama

__global__ void __launch_bounds__(rama::THREADS, 2) k_solve_cta(rama::CtaLaunch L);
__global__ void __launch_bounds__(rama::THREADS_SMALL, 3) k_solve_cta_small(rama::CtaLaunch L);
__global__ void __launch_bounds__(rama::THREADS, 2) k_solve_mixed(rama::MixedLaunch L);
__global__ void __launch_bounds__(rama::THREADS, 2) k_solve_grid(rama::GridLaunch L);
__global__ void __launch_bounds__(rama::THREADS, 2) k_parse_grid(rama::ParseLaunch L);
__global__ void __launch_bounds__(rama::THREADS, 2) k_step_cta(rama_step_args *a, char *ws, uint64_t bytes);
__global__ void __launch_bounds__(rama::THREADS, 2) k_step_grid(rama_step_args *a, char *ws, uint64_t bytes);
__global__ void __launch_bounds__(rama::THREADS, 2) k_objective(const int32_t *I, const int32_t *J, const float *C,
                                                                int64_t n, const int32_t *lab, double *out, char *ws,
                                                                uint64_t bytes);
__global__ void __launch_bounds__(256) k_max_id(rama::MaxIdLaunch L);
