// k_step_cta.cu -- one solver step on one CTA (rama_step with team 1).
#include "step.cuh"

using namespace rama;

__global__ void __launch_bounds__(THREADS, 2) k_step_cta(rama_step_args *a, char *ws, uint64_t bytes)
{
    extern __shared__ __align__(16) char sm[];
    BlockTeam t;
    run_step(t, sm, make_scratch(ws, bytes), a);
}
