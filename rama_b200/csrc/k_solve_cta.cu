// k_solve_cta.cu -- persistent CTAs; each pulls instances from a queue
// (largest first) and solves them alone (BlockTeam).  Used for batches
// without cluster instances and for small single instances.
#include "kernels.cuh"

using namespace rama;

__global__ void __launch_bounds__(THREADS, 2) k_solve_cta(CtaLaunch L)
{
    extern __shared__ __align__(16) char sm[];
    __shared__ int next;
    BlockTeam t;
    for (int guard = 0; guard < (1 << 30); ++guard) {
        if (threadIdx.x == 0) next = atomicAdd(L.queue, 1);
        __syncthreads();
        const int k = next;
        __syncthreads();
        if (k >= L.count) break;
        Instance *io = &L.inst[L.order[k]];
        Scratch sc = make_scratch(io->ws, io->ws_bytes);
        solve_instance(t, sm, sc, io);
        __syncthreads();
    }
}
