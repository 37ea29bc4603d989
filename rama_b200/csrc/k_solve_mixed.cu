// k_solve_mixed.cu -- a batch with instances for clusters: clusters draw from
// the queue, which holds the cluster instances first (largest first); once a
// cluster draws an instance that is not for a cluster, its CTAs go on alone,
// one instance each, like k_solve_cta.  Single mid-size solves run here too
// (one cluster instance).
#include "kernels.cuh"

using namespace rama;

__global__ void __launch_bounds__(THREADS, 2) k_solve_mixed(MixedLaunch L)
{
    extern __shared__ __align__(16) char sm[];
    __shared__ int next;
    cg::cluster_group cl = cg::this_cluster();
    ClusterTeam ct;
    BlockTeam bt;
    int mine = -1;  // an instance this CTA drew for itself
    for (int guard = 0; guard < (1 << 30); ++guard) {
        if (cl.block_rank() == 0 && threadIdx.x == 0) next = atomicAdd(L.queue, 1);
        cl.sync();
        const int k = *cl.map_shared_rank(&next, 0);
        cl.sync();  // no CTA reads another's shared memory after this point
        if (k >= L.count) return;
        if (k >= L.ncluster) {
            if (cl.block_rank() == 0) mine = k;
            break;
        }
        Instance *io = &L.inst[L.order[k]];
        solve_instance(ct, sm, make_scratch(io->ws, io->ws_bytes), io);
        cl.sync();
    }
    for (int guard = 0; guard < (1 << 30); ++guard) {
        int k = mine;
        mine = -1;
        if (k < 0) {
            if (threadIdx.x == 0) next = atomicAdd(L.queue, 1);
            __syncthreads();
            k = next;
            __syncthreads();
        }
        if (k >= L.count) break;
        Instance *io = &L.inst[L.order[k]];
        solve_instance(bt, sm, make_scratch(io->ws, io->ws_bytes), io);
        __syncthreads();
    }
}
