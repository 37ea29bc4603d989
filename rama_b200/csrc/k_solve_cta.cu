// k_solve_cta.cu -- persistent CTAs of 512 threads; each pulls instances
// from a queue (largest first) and solves them alone (BlockTeam).  Used for
// batches without cluster instances and for small single instances.
#include "kernels.cuh"

using namespace rama;

__global__ void __launch_bounds__(THREADS, 2) k_solve_cta(CtaLaunch L)
{
    extern __shared__ __align__(16) char sm[];
    __shared__ int next;
    solve_queue_by_cta(L, sm, &next);
}
