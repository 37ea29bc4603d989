// k_solve_grid.cu -- one cooperative launch; the whole GPU solves one
// instance (GridTeam).
#include "kernels.cuh"

using namespace rama;

__global__ void __launch_bounds__(THREADS, 2) k_solve_grid(GridLaunch L)
{
    extern __shared__ __align__(16) char sm[];
    GridTeam t;
    Scratch sc = make_scratch(L.ws, L.ws_bytes);
    solve_instance(t, sm, sc, L.inst);
}
