// k_step_grid.cu -- one solver step on the cooperative grid (rama_step with
// team 2).
#include "step.cuh"

using namespace rama;

__global__ void __launch_bounds__(THREADS, 2) k_step_grid(rama_step_args *a, char *ws, uint64_t bytes)
{
    extern __shared__ __align__(16) char sm[];
    GridTeam t;
    run_step(t, sm, make_scratch(ws, bytes), a);
}
