// k_solve_cta_small.cu -- the same persistent CTAs with 256 threads, three
// per SM: more instances in flight at once, fewer threads on each (the
// autotuner measures which of the two a device's batches prefer).
#include "kernels.cuh"

using namespace rama;

__global__ void __launch_bounds__(THREADS_SMALL, 3) k_solve_cta_small(CtaLaunch L)
{
    extern __shared__ __align__(16) char sm[];
    __shared__ int next;
    solve_queue_by_cta(L, sm, &next);
}
