// capi.cu -- the host side of librama_b200.so: the C ABI of
// include/rama_b200.h (handles, workspaces, launches, batches, statistics).
//
// The kernels live in their own translation units (kernels.cuh):
//   k_solve_grid  : one cooperative launch; the whole GPU solves one instance.
//   k_solve_mixed : clusters of CTAs for the largest instances of a batch (and
//                   single mid-size solves), then one CTA per instance.
//   k_solve_cta   : persistent CTAs, one instance each.
//   k_step_*, k_objective, k_parse_grid, k_max_id: steps and helpers.
// Every solve takes its scratch memory from a workspace the handle owns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/rama_b200.h"
#include "kernels.cuh"

using namespace rama;

namespace {

// Launch parameters a handle starts with (rama_tuning; the autotuner of
// rama_b200/autotune.py replaces them with measured choices).  None of them
// changes a result: every team computes the same solve.
constexpr int DEFAULT_CLUSTER_CTAS = 8;            // CTAs of a cluster team (the portable maximum)
constexpr int64_t DEFAULT_SINGLE_CLUSTER_MIN = 4000;  // a single solve from this size on runs on a cluster
constexpr int64_t DEFAULT_SINGLE_GRID_MIN = 100000;   // ... and from this size on on the whole GPU
constexpr int64_t DEFAULT_BATCH_CLUSTER_MIN = 20000;  // smaller batch instances always run on one CTA
constexpr float DEFAULT_BATCH_CLUSTER_SHARE = 1.5f;   // ... larger ones on a cluster above this many
                                                      // times the batch's edges per CTA

thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

#define CU(call)                                                                               \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return fail(RAMA_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

int status_from_bits(int32_t s)
{
    if (s == 0) return RAMA_OK;
    if (s & ERR_INVALID_ARG) return RAMA_ERR_INVALID_ARG;
    if (s & ERR_ARENA) return RAMA_ERR_OOM;
    if (s & ERR_BAD_CONTRACTION) return RAMA_ERR_BAD_CONTRACTION;
    if (s & ERR_ITER_LIMIT) return RAMA_ERR_ITER_LIMIT;
    return RAMA_ERR_CUDA;
}

Options to_opts(const rama_options *o)
{
    Options r;
    r.max_cycle_length_lb = o->max_cycle_length_lb;
    r.num_dual_itr_lb = o->num_dual_itr_lb;
    r.max_cycle_length_primal = o->max_cycle_length_primal;
    r.num_dual_itr_primal = o->num_dual_itr_primal;
    r.num_outer_itr_dual = o->num_outer_itr_dual;
    r.mean_multiplier_mm = o->mean_multiplier_mm;
    r.matching_thresh_crossover_ratio = o->matching_thresh_crossover_ratio;
    r.tri_memory_factor = o->tri_memory_factor;
    r.only_compute_lb = o->only_compute_lb;
    r.max_time_sec = o->max_time_sec;
    r.dump_timeline = o->dump_timeline;
    r.verbose = o->verbose;
    r.sanitize_graph = o->sanitize_graph;
    r.woc_pentagons = o->woc_pentagons;
    return r;
}

}  // namespace

// error text for the entry points of other translation units (noalloc.cu)
void rama_set_last_error(const std::string &msg) { g_err = msg; }

struct rama_context {
    int device = 0;
    int sms = 0;
    int grid_ctas = 0;  // co-resident CTAs of k_solve_grid
    int step_ctas = 0;  // ... of k_step_grid
    int obj_ctas = 0;   // ... of k_objective
    int cta_per_sm = 0;
    int cta_small_per_sm = 0;  // co-resident CTAs of k_solve_cta_small per SM
    int grid_per_sm_max = 0;  // occupancy maximum of k_solve_grid per SM
    int cluster_cap[17] = {};  // co-resident clusters of k_solve_mixed by cluster size (0: not known yet)
    rama_tuning tune{};
    int parse_ctas = 0;   // co-resident CTAs of k_parse_grid
    char *p_text = nullptr;  // device copy of text for rama_parse_multicut_host
    int64_t p_cap = 0;
    char *ws = nullptr;
    uint64_t ws_bytes = 0;
    uint64_t ws_fixed = 0;  // user-requested size (0 = automatic)
    Instance *d_inst = nullptr;
    int32_t inst_cap = 0;
    int32_t *d_queue = nullptr;
    int32_t *d_order = nullptr;
    rama_step_args *d_step = nullptr;
    double *d_scalar = nullptr;
    int32_t *d_timeline = nullptr;
    int64_t tl_cap = 0;
    int64_t *d_prof = nullptr;
    std::vector<int32_t> timeline;
    int32_t tl_rounds = 0;
    int64_t tl_labels = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    rama_stats stats{};
    // device staging of rama_solve_host (grown on demand, reused)
    int32_t *io_i = nullptr, *io_j = nullptr, *io_l = nullptr;
    float *io_c = nullptr;
    cudaStream_t io_stream = nullptr;  // rama_solve_host's copies and solve
    int64_t io_edges = 0, io_labels = 0;
    // asynchronous batch in flight
    bool b_active = false;
    int32_t b_count = 0;
    cudaStream_t b_stream = nullptr;
    Instance *b_host = nullptr;  // pinned: instance descriptors in, results out
    int32_t b_host_cap = 0;
    std::vector<Instance> b_in;
    std::vector<char> b_cluster;  // instance k is solved by a cluster team
    std::vector<int32_t> b_order;
    cudaEvent_t ev_done = nullptr;
};

namespace {

int ensure_ws(rama_context *h, uint64_t need)
{
    if (h->ws && h->ws_bytes >= need) return RAMA_OK;
    if (h->ws) {
        cudaFree(h->ws);
        h->ws = nullptr;
        h->ws_bytes = 0;
    }
    size_t fr = 0, tot = 0;
    CU(cudaMemGetInfo(&fr, &tot));
    uint64_t limit = (uint64_t)((double)fr * 0.92);
    uint64_t bytes = std::min<uint64_t>(need, limit);
    bytes = (bytes + 255) & ~uint64_t(255);
    if (bytes < (4u << 20)) bytes = 4u << 20;
    if (cudaMalloc(&h->ws, bytes) != cudaSuccess) {
        cudaGetLastError();
        h->ws = nullptr;
        return fail(RAMA_ERR_OOM, "cannot allocate the solver workspace");
    }
    h->ws_bytes = bytes;
    return RAMA_OK;
}

int ensure_inst(rama_context *h, int32_t count)
{
    if (h->inst_cap >= count) return RAMA_OK;
    if (h->d_inst) cudaFree(h->d_inst);
    if (h->d_order) cudaFree(h->d_order);
    h->d_inst = nullptr;
    h->d_order = nullptr;
    CU(cudaMalloc(&h->d_inst, sizeof(Instance) * (size_t)count));
    CU(cudaMalloc(&h->d_order, sizeof(int32_t) * (size_t)count));
    h->inst_cap = count;
    return RAMA_OK;
}

// Workspace bytes per edge: about 1 KiB covers a solve whose triangle budget
// is at most twice the repulsive edges; each further unit of the budget
// factor adds triangles at roughly 256 bytes each (sorts, message-passing
// state).  A solve that still runs short reports the size it needed and is
// run again with it.
uint64_t ws_per_edge(float tri_factor)
{
    const double extra = tri_factor > 2.0f ? 256.0 * ((double)tri_factor - 2.0) : 0.0;
    return 1024ull + (uint64_t)extra;
}
uint64_t ws_estimate(int64_t n_edges, float tri_factor = 2.0f)
{
    return (uint64_t)n_edges * ws_per_edge(tri_factor) + (64ull << 20);
}
uint64_t align4k(uint64_t b) { return (b + 4095) & ~uint64_t(4095); }
// workspace slice of one instance of a batch
uint64_t ws_slice(int64_t n_edges, float tri_factor = 2.0f)
{
    return align4k((uint64_t)n_edges * ws_per_edge(tri_factor) + (1ull << 20));
}

// Launches the solve of the instances already in h->d_inst (queue order in
// h->d_order).  team 2: one instance on the cooperative grid; otherwise the
// first `ncluster` queue entries go to cluster teams and the rest to CTAs.
// co-resident clusters of k_solve_mixed for a cluster size (0 if none fits)
int cluster_capacity(rama_context *h, int size)
{
    if (size < 1 || size > 16) return 0;
    if (!h->cluster_cap[size]) {
        if (size > 8 && cudaFuncSetAttribute((const void *)k_solve_mixed,
                                             cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
            cudaGetLastError();
            h->cluster_cap[size] = -1;
            return 0;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(size);
        cfg.blockDim = dim3(THREADS);
        cfg.dynamicSmemBytes = SMEM;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = size;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int ncl = 0;
        if (cudaOccupancyMaxActiveClusters(&ncl, (void *)k_solve_mixed, &cfg) != cudaSuccess) {
            cudaGetLastError();
            ncl = 0;
        }
        h->cluster_cap[size] = ncl > 0 ? ncl : -1;
    }
    return h->cluster_cap[size] > 0 ? h->cluster_cap[size] : 0;
}

int launch_solve(rama_context *h, int32_t count, int team, cudaStream_t st, int32_t ncluster = 0,
                 int64_t grid_edges = 0)
{
    if (team == 2) {
        GridLaunch L{h->d_inst, h->ws, h->ws_bytes};
        void *args[] = {&L};
        const int per_sm = grid_edges < h->tune.grid_small_max ? h->tune.grid_small_ctas_per_sm
                                                                : h->tune.grid_ctas_per_sm;
        CU(cudaLaunchCooperativeKernel((void *)k_solve_grid, dim3(per_sm * h->sms), dim3(THREADS), args, SMEM, st));
    } else if (ncluster > 0) {
        const int csz = h->tune.cluster_ctas;
        const int64_t want = (int64_t)ncluster * csz + (count - ncluster);
        const int64_t cap = (int64_t)std::max(1, cluster_capacity(h, csz)) * csz;
        const int64_t ctas = (std::min(want, cap) + csz - 1) / csz * csz;
        CU(cudaMemsetAsync(h->d_queue, 0, sizeof(int32_t), st));
        MixedLaunch L{h->d_inst, h->d_order, count, ncluster, h->d_queue};
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)ctas);
        cfg.blockDim = dim3(THREADS);
        cfg.dynamicSmemBytes = SMEM;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = csz;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CU(cudaLaunchKernelEx(&cfg, k_solve_mixed, L));
    } else {
        CU(cudaMemsetAsync(h->d_queue, 0, sizeof(int32_t), st));
        CtaLaunch L{h->d_inst, h->d_order, count, h->d_queue};
        if (h->tune.cta_threads == THREADS_SMALL) {
            const int ctas = std::max(1, std::min<int>(count, h->sms * h->cta_small_per_sm));
            k_solve_cta_small<<<ctas, THREADS_SMALL, SMEM_SMALL, st>>>(L);
        } else {
            const int ctas = std::max(1, std::min<int>(count, h->sms * h->cta_per_sm));
            k_solve_cta<<<ctas, THREADS, SMEM, st>>>(L);
        }
        CU(cudaGetLastError());
    }
    return RAMA_OK;
}

int solve_one(rama_context *h, const int32_t *d_i, const int32_t *d_j, const float *d_c, int64_t n,
              const rama_options *opts, int32_t *d_labels, int64_t cap, int64_t *num_labels, double *lb,
              cudaStream_t st)
{
    if (!h || !opts || n < 0 || (n > 0 && (!d_i || !d_j || !d_c))) return fail(RAMA_ERR_INVALID_ARG, "bad arguments");
    if (h->b_active) return fail(RAMA_ERR_INVALID_ARG, "a batch is in flight on this handle (call rama_batch_wait)");
    Options o = to_opts(opts);
    int team = opts->team;
    if (team < 1 || team > 3)
        team = n < h->tune.single_cluster_min ? 1 : (n < h->tune.single_grid_min ? 3 : 2);
    int rc = ensure_inst(h, 1);
    if (rc) return rc;
    // timeline buffer
    int32_t *tl = nullptr;
    int64_t tl_cap = 0;
    if (opts->dump_timeline) {
        tl_cap = std::min<int64_t>(std::min<int64_t>(cap, (int64_t)1 << 22) * 64, (int64_t)1 << 28);
        if (h->tl_cap < tl_cap) {
            if (h->d_timeline) cudaFree(h->d_timeline);
            CU(cudaMalloc(&h->d_timeline, sizeof(int32_t) * (size_t)tl_cap));
            h->tl_cap = tl_cap;
        }
        tl = h->d_timeline;
    }
    uint64_t need = h->ws_fixed ? h->ws_fixed : ws_estimate(n, opts->tri_memory_factor);
    for (int attempt = 0; attempt < 8; ++attempt) {
        rc = ensure_ws(h, need);
        if (rc) return rc;
        Instance hi{};
        hi.opts = o;
        hi.i = d_i;
        hi.j = d_j;
        hi.c = d_c;
        hi.n = n;
        hi.labels = d_labels;
        hi.labels_cap = cap;
        hi.timeline = tl;
        hi.timeline_cap = tl_cap;
        hi.prof = h->d_prof;
        hi.ws = h->ws;
        hi.ws_bytes = h->ws_bytes;
        CU(cudaMemsetAsync(h->d_prof, 0, sizeof(int64_t) * 2 * PH_COUNT, st));
        int32_t zero = 0;
        CU(cudaMemcpyAsync(h->d_inst, &hi, sizeof(Instance), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(h->d_order, &zero, sizeof(int32_t), cudaMemcpyHostToDevice, st));
        CU(cudaEventRecord(h->ev0, st));
        rc = launch_solve(h, 1, team, st, team == 3 ? 1 : 0, n);
        if (rc) return rc;
        CU(cudaEventRecord(h->ev1, st));
        Instance ho{};
        CU(cudaMemcpyAsync(&ho, h->d_inst, sizeof(Instance), cudaMemcpyDeviceToHost, st));
        CU(cudaStreamSynchronize(st));
        float ms = 0;
        cudaEventElapsedTime(&ms, h->ev0, h->ev1);
        // A solve that ran out of workspace runs again with more.  That
        // includes a dual that fell back to the trivial bound when a larger
        // workspace would have held its triangles: the reference allocates
        // device memory as it goes and falls back only when the device has
        // none left (src/dual_solver.cu:58-61), and so does this loop.
        const bool short_ws =
            (ho.status & ERR_ARENA) || (ho.dual_oom && (uint64_t)ho.arena_want > h->ws_bytes);
        if (short_ws && !h->ws_fixed) {
            size_t fr = 0, tot = 0;
            cudaMemGetInfo(&fr, &tot);
            const uint64_t avail = (uint64_t)((double)(fr + h->ws_bytes) * 0.9);
            if (h->ws_bytes < avail) {
                const uint64_t want = (uint64_t)((double)ho.arena_want * 1.25);
                need = std::min<uint64_t>(avail, std::max<uint64_t>(h->ws_bytes * 2, want));
                continue;
            }
            if (ho.status & ERR_ARENA) break;
            // the device is full: keep the trivial bound, as the reference does
        }
        h->stats.rounds = ho.rounds;
        h->stats.matching_rounds = ho.matching_rounds;
        h->stats.mst_rounds = ho.mst_rounds;
        h->stats.timeline_rounds = ho.timeline_rounds;
        h->stats.dual_oom = ho.dual_oom;
        h->stats.team = team;
        h->stats.triangles = ho.triangles_initial;
        h->stats.edges_after_dual = ho.edges_after_dual;
        h->stats.workspace_peak = ho.arena_peak;
        h->stats.device_ms = ms;
        h->stats.alg_bytes = ho.alg_bytes;
        {
            int64_t pr[2 * PH_COUNT];
            CU(cudaMemcpy(pr, h->d_prof, sizeof(pr), cudaMemcpyDeviceToHost));
            for (int k = 0; k < PH_COUNT && k < 32; ++k) {
                h->stats.phase_ms[k] = 1e-6 * (double)pr[k];
                h->stats.phase_bytes[k] = (double)pr[PH_COUNT + k];
            }
        }
        if (opts->dump_timeline && ho.timeline_rounds > 0) {
            h->tl_rounds = ho.timeline_rounds;
            h->tl_labels = ho.num_labels;
            h->timeline.resize((size_t)ho.timeline_rounds * (size_t)ho.num_labels);
            CU(cudaMemcpy(h->timeline.data(), h->d_timeline, sizeof(int32_t) * h->timeline.size(),
                          cudaMemcpyDeviceToHost));
        } else {
            h->tl_rounds = 0;
            h->tl_labels = ho.num_labels;
            h->timeline.clear();
        }
        if (num_labels) *num_labels = ho.num_labels;
        if (lb) *lb = ho.lb;
        if (ho.status) {
            std::string msg = "solver status bits " + std::to_string(ho.status);
            if (ho.status & ERR_INVALID_ARG) msg = "invalid input (negative id, self loop, or label buffer too small)";
            if (ho.status & ERR_BAD_CONTRACTION) msg = "Found bad contractions";
            return fail(status_from_bits(ho.status), msg);
        }
        return RAMA_OK;
    }
    return fail(RAMA_ERR_OOM, "solver workspace exhausted");
}

}  // namespace

extern "C" {

const char *rama_last_error(void) { return g_err.c_str(); }

int rama_options_init(rama_options *o, const char *mode)
{
    if (!o) return RAMA_ERR_INVALID_ARG;
    o->max_cycle_length_lb = 5;
    o->num_dual_itr_lb = 10;
    o->max_cycle_length_primal = 3;
    o->num_dual_itr_primal = 5;
    o->num_outer_itr_dual = 1;
    o->mean_multiplier_mm = 0.05f;
    o->matching_thresh_crossover_ratio = 0.05f;
    o->tri_memory_factor = 2.0f;
    o->only_compute_lb = 0;
    o->max_time_sec = -1;
    o->dump_timeline = 0;
    o->verbose = 0;
    o->sanitize_graph = 0;
    o->team = 0;
    o->woc_pentagons = 0;
    if (!mode) return RAMA_OK;
    if (!strcmp(mode, "P")) {
        o->max_cycle_length_lb = 0;
        o->num_dual_itr_lb = 0;
        o->max_cycle_length_primal = 0;
        o->num_dual_itr_primal = 0;
    } else if (!strcmp(mode, "PD+")) {
        o->max_cycle_length_lb = 5;
        o->num_dual_itr_lb = 10;
        o->max_cycle_length_primal = 5;
        o->num_dual_itr_primal = 10;
    } else if (!strcmp(mode, "D")) {
        o->max_cycle_length_lb = 5;
        o->num_dual_itr_lb = 10;
        o->num_outer_itr_dual = 5;
        o->only_compute_lb = 1;
    }
    return RAMA_OK;
}

int rama_create(int device, uint64_t workspace_bytes, rama_handle *out)
{
    if (!out) return fail(RAMA_ERR_INVALID_ARG, "null handle");
    *out = nullptr;
    CU(cudaSetDevice(device));
    rama_context *h = new rama_context();
    h->device = device;
    h->ws_fixed = workspace_bytes;
    cudaDeviceProp p;
    CU(cudaGetDeviceProperties(&p, device));
    h->sms = p.multiProcessorCount;
    // the sort stages a tile in shared memory: more than the default 48 KB
    for (const void *k : {(const void *)k_solve_grid, (const void *)k_solve_cta, (const void *)k_solve_mixed,
                          (const void *)k_step_grid, (const void *)k_step_cta, (const void *)k_objective,
                          (const void *)k_parse_grid})
        CU(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
    int per_sm = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve_grid, THREADS, SMEM));
    if (per_sm < 1) {
        delete h;
        return fail(RAMA_ERR_CUDA, "solver kernel does not fit on an SM");
    }
    h->grid_per_sm_max = per_sm;
    h->grid_ctas = per_sm * h->sms;
    h->tune.grid_ctas_per_sm = per_sm;
    h->tune.grid_small_ctas_per_sm = per_sm;
    h->tune.grid_small_max = 0;
    h->tune.cluster_ctas = DEFAULT_CLUSTER_CTAS;
    h->tune.single_cluster_min = DEFAULT_SINGLE_CLUSTER_MIN;
    h->tune.single_grid_min = DEFAULT_SINGLE_GRID_MIN;
    h->tune.batch_cluster_min = DEFAULT_BATCH_CLUSTER_MIN;
    h->tune.batch_cluster_share = DEFAULT_BATCH_CLUSTER_SHARE;
    h->tune.cta_threads = THREADS;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_grid, THREADS, SMEM));
    h->step_ctas = std::max(1, per_sm) * h->sms;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_objective, THREADS, SMEM));
    h->obj_ctas = std::max(1, per_sm) * h->sms;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_parse_grid, THREADS, SMEM));
    h->parse_ctas = std::max(1, per_sm) * h->sms;
    int per_sm_cta = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_cta, k_solve_cta, THREADS, SMEM));
    h->cta_per_sm = std::max(1, per_sm_cta);
    CU(cudaFuncSetAttribute((const void *)k_solve_cta_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            SMEM_SMALL));
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_cta, k_solve_cta_small, THREADS_SMALL, SMEM_SMALL));
    h->cta_small_per_sm = std::max(1, per_sm_cta);
    if (cluster_capacity(h, DEFAULT_CLUSTER_CTAS) < 1) {
        delete h;
        return fail(RAMA_ERR_CUDA, "no cluster of the solver kernel fits on the device");
    }
    CU(cudaMalloc(&h->d_queue, sizeof(int32_t) * 4));
    CU(cudaMalloc(&h->d_step, sizeof(rama_step_args)));
    CU(cudaMalloc(&h->d_scalar, sizeof(double) * 4));
    CU(cudaMalloc(&h->d_prof, sizeof(int64_t) * 2 * PH_COUNT));
    CU(cudaEventCreate(&h->ev0));
    CU(cudaEventCreate(&h->ev1));
    CU(cudaEventCreateWithFlags(&h->ev_done, cudaEventDisableTiming));
    *out = h;
    return RAMA_OK;
}

void rama_destroy(rama_handle h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    cudaFree(h->ws);
    cudaFree(h->d_inst);
    cudaFree(h->d_order);
    cudaFree(h->d_queue);
    cudaFree(h->d_step);
    cudaFree(h->d_scalar);
    cudaFree(h->d_timeline);
    cudaFree(h->d_prof);
    cudaFree(h->io_i);
    cudaFree(h->io_j);
    cudaFree(h->io_c);
    cudaFree(h->io_l);
    cudaFree(h->p_text);
    cudaEventDestroy(h->ev0);
    cudaEventDestroy(h->ev1);
    cudaEventDestroy(h->ev_done);
    if (h->io_stream) cudaStreamDestroy(h->io_stream);
    if (h->b_host) cudaFreeHost(h->b_host);
    delete h;
}

int rama_solve(rama_handle h, const int32_t *d_i, const int32_t *d_j, const float *d_costs, int64_t num_edges,
               const rama_options *opts, int32_t *d_labels, int64_t labels_cap, int64_t *num_labels, double *lb,
               void *stream)
{
    if (!h) return fail(RAMA_ERR_INVALID_ARG, "null handle");
    CU(cudaSetDevice(h->device));
    return solve_one(h, d_i, d_j, d_costs, num_edges, opts, d_labels, labels_cap, num_labels, lb,
                     (cudaStream_t)stream);
}

int rama_solve_host(rama_handle h, const int32_t *i, const int32_t *j, const float *costs, int64_t n,
                    const rama_options *opts, int32_t *labels, int64_t labels_cap, int64_t *num_labels, double *lb,
                    double *solve_ms)
{
    if (!h || !opts || n < 0 || (n > 0 && (!i || !j || !costs))) return fail(RAMA_ERR_INVALID_ARG, "bad arguments");
    CU(cudaSetDevice(h->device));
    if (!h->io_stream) CU(cudaStreamCreateWithFlags(&h->io_stream, cudaStreamNonBlocking));
    cudaStream_t st = h->io_stream;
    if (h->io_edges < std::max<int64_t>(n, 1)) {
        cudaFree(h->io_i);
        cudaFree(h->io_j);
        cudaFree(h->io_c);
        h->io_i = h->io_j = nullptr;
        h->io_c = nullptr;
        h->io_edges = 0;
        const size_t nb = sizeof(int32_t) * (size_t)std::max<int64_t>(n, 1);
        CU(cudaMalloc(&h->io_i, nb));
        CU(cudaMalloc(&h->io_j, nb));
        CU(cudaMalloc(&h->io_c, nb));
        h->io_edges = std::max<int64_t>(n, 1);
    }
    int32_t *di = h->io_i, *dj = h->io_j;
    float *dc = h->io_c;
    if (n > 0) {
        CU(cudaMemcpyAsync(di, i, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(dj, j, sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(dc, costs, sizeof(float) * n, cudaMemcpyHostToDevice, st));
    }
    // the label buffer holds max node id + 1 entries: the maximum comes from
    // the device copy of the edges, not from a scan on the host
    int32_t mx[2] = {-1, 0};
    int32_t *d_mx = reinterpret_cast<int32_t *>(h->d_scalar);
    CU(cudaMemcpyAsync(d_mx, mx, sizeof(mx), cudaMemcpyHostToDevice, st));
    if (n > 0) {
        const int64_t want = (n / 4 + 255) / 256;
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)h->sms * 8));
        k_max_id<<<blocks, 256, 0, st>>>(MaxIdLaunch{di, dj, n, d_mx});
        CU(cudaGetLastError());
    }
    CU(cudaMemcpyAsync(mx, d_mx, sizeof(mx), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    if (mx[1]) return fail(RAMA_ERR_INVALID_ARG, "invalid input (negative node id)");
    const int64_t cap = (int64_t)mx[0] + 1;
    if (h->io_labels < std::max<int64_t>(cap, 1)) {
        cudaFree(h->io_l);
        h->io_l = nullptr;
        h->io_labels = 0;
        CU(cudaMalloc(&h->io_l, sizeof(int32_t) * (size_t)std::max<int64_t>(cap, 1)));
        h->io_labels = std::max<int64_t>(cap, 1);
    }
    int32_t *dl = h->io_l;
    int64_t nl = 0;
    int rc = solve_one(h, di, dj, dc, n, opts, dl, cap, &nl, lb, st);
    if (rc == RAMA_OK) {
        if (nl > labels_cap)
            rc = fail(RAMA_ERR_INVALID_ARG, "label buffer too small");
        else if (nl > 0) {
            if (cudaMemcpyAsync(labels, dl, sizeof(int32_t) * nl, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)
                rc = fail(RAMA_ERR_CUDA, "copying labels failed");
        }
        if (num_labels) *num_labels = nl;
        if (solve_ms) *solve_ms = h->stats.device_ms;
    }
    return rc;
}

int rama_get_timeline(rama_handle h, int32_t *out, int64_t cap, int32_t *rounds, int64_t *num_labels)
{
    if (!h) return fail(RAMA_ERR_INVALID_ARG, "null handle");
    if (rounds) *rounds = h->tl_rounds;
    if (num_labels) *num_labels = h->tl_labels;
    if (out) {
        if ((int64_t)h->timeline.size() > cap) return fail(RAMA_ERR_INVALID_ARG, "timeline buffer too small");
        std::memcpy(out, h->timeline.data(), sizeof(int32_t) * h->timeline.size());
    }
    return RAMA_OK;
}

int rama_batch_launch(rama_handle h, const int32_t *d_i, const int32_t *d_j, const float *d_costs,
                      const int64_t *edge_offsets, int32_t count, const rama_options *opts, int32_t opts_count,
                      int32_t *d_labels, const int64_t *label_offsets, void *stream)
{
    if (!h || !opts || count < 0 || !edge_offsets || !label_offsets || (opts_count != 1 && opts_count != count))
        return fail(RAMA_ERR_INVALID_ARG, "bad arguments");
    if (h->b_active) return fail(RAMA_ERR_INVALID_ARG, "a batch is already in flight on this handle");
    CU(cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    h->b_count = count;
    h->b_stream = st;
    if (count == 0) {
        h->b_active = true;
        return RAMA_OK;
    }
    int rc = ensure_inst(h, count);
    if (rc) return rc;
    if (h->b_host_cap < count) {
        if (h->b_host) cudaFreeHost(h->b_host);
        h->b_host = nullptr;
        h->b_host_cap = 0;
        CU(cudaHostAlloc(&h->b_host, sizeof(Instance) * (size_t)count, cudaHostAllocDefault));
        h->b_host_cap = count;
    }
    h->b_in.assign(count, Instance{});
    h->b_cluster.assign(count, 0);
    h->b_order.resize(count);
    for (int32_t k = 0; k < count; ++k) {
        const int64_t a = edge_offsets[k], b = edge_offsets[k + 1];
        Instance &x = h->b_in[k];
        x.opts = to_opts(&opts[opts_count == 1 ? 0 : k]);
        x.i = d_i + a;
        x.j = d_j + a;
        x.c = d_costs + a;
        x.n = b - a;
        x.labels = d_labels + label_offsets[k];
        x.labels_cap = label_offsets[k + 1] - label_offsets[k];
        h->b_order[k] = k;
    }
    // Automatic teams: an instance goes to a cluster when one CTA alone would
    // take much longer than the batch as a whole, i.e. when it holds more than
    // 1.5 times the edges per CTA of the batch (a cluster finishes it sooner
    // but spends more CTA time on it).
    {
        int64_t total_edges = 0;
        for (int32_t k = 0; k < count; ++k) total_edges += h->b_in[k].n;
        const int64_t per_cta = total_edges / std::max(1, h->sms * h->cta_per_sm);
        const int64_t auto_min = std::max<int64_t>(h->tune.batch_cluster_min,
                                                   (int64_t)((double)per_cta * h->tune.batch_cluster_share));
        for (int32_t k = 0; k < count; ++k) {
            const int tm = opts[opts_count == 1 ? 0 : k].team;
            h->b_cluster[k] = (tm == 2 || tm == 3 || ((tm < 1 || tm > 3) && h->b_in[k].n >= auto_min)) ? 1 : 0;
        }
    }
    // queue order: cluster instances first, then by size, largest first
    std::stable_sort(h->b_order.begin(), h->b_order.end(), [&](int32_t x, int32_t y) {
        if (h->b_cluster[x] != h->b_cluster[y]) return h->b_cluster[x] > h->b_cluster[y];
        return h->b_in[x].n > h->b_in[y].n;
    });
    int32_t ncluster = 0;
    for (int32_t k = 0; k < count; ++k) ncluster += h->b_cluster[k];
    // every instance owns a workspace slice sized from its edge count; their
    // sum is the batch's device footprint
    uint64_t total = 0;
    for (int32_t k = 0; k < count; ++k) total += ws_slice(h->b_in[k].n, h->b_in[k].opts.tri_memory_factor);
    // a handle with a fixed workspace allocates all of it once and admits
    // batches up to that size
    if (h->ws_fixed && total > h->ws_fixed) return fail(RAMA_ERR_OOM, "batch exceeds the handle's fixed workspace");
    rc = ensure_ws(h, h->ws_fixed ? h->ws_fixed : total);
    if (rc) return rc;
    if (h->ws_bytes < total) return fail(RAMA_ERR_OOM, "workspace too small for the batch");
    {
        uint64_t off = 0;
        for (int32_t k = 0; k < count; ++k) {
            h->b_in[k].ws = h->ws + off;
            h->b_in[k].ws_bytes = ws_slice(h->b_in[k].n, h->b_in[k].opts.tri_memory_factor);
            off += h->b_in[k].ws_bytes;
        }
    }
    std::memcpy(h->b_host, h->b_in.data(), sizeof(Instance) * (size_t)count);
    CU(cudaMemcpyAsync(h->d_inst, h->b_host, sizeof(Instance) * count, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(h->d_order, h->b_order.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice, st));
    CU(cudaEventRecord(h->ev0, st));
    // a batch of one instance that asks for the whole GPU (team 2) runs on
    // the cooperative grid, in its slice at the start of the workspace
    if (count == 1 && opts[0].team == 2)
        rc = launch_solve(h, 1, 2, st, 0, h->b_in[0].n);
    else
        rc = launch_solve(h, count, 1, st, ncluster);
    if (rc) return rc;
    CU(cudaEventRecord(h->ev1, st));
    CU(cudaMemcpyAsync(h->b_host, h->d_inst, sizeof(Instance) * count, cudaMemcpyDeviceToHost, st));
    CU(cudaEventRecord(h->ev_done, st));
    h->b_active = true;
    return RAMA_OK;
}

int rama_batch_poll(rama_handle h)
{
    if (!h || !h->b_active) return fail(RAMA_ERR_INVALID_ARG, "no batch in flight");
    if (h->b_count == 0) return 1;
    cudaError_t e = cudaEventQuery(h->ev_done);
    if (e == cudaSuccess) return 1;
    if (e == cudaErrorNotReady) return 0;
    return -fail(RAMA_ERR_CUDA, std::string("batch: ") + cudaGetErrorString(e));
}

int rama_batch_wait(rama_handle h, int64_t *num_labels, double *lbs, int32_t *status)
{
    if (!h || !h->b_active) return fail(RAMA_ERR_INVALID_ARG, "no batch in flight");
    h->b_active = false;
    const int32_t count = h->b_count;
    if (count == 0) return RAMA_OK;
    CU(cudaSetDevice(h->device));
    CU(cudaEventSynchronize(h->ev_done));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    std::vector<Instance> out(h->b_host, h->b_host + count);
    // instances that ran out of workspace (a dual fallback included, when a
    // larger slice would have held it) are solved again with a larger slice:
    // twice the old one, or what the refused allocation needed
    auto bigger = [&](int32_t k) {
        return align4k(std::max<uint64_t>(h->b_in[k].ws_bytes * 2, (uint64_t)((double)out[k].arena_want * 1.25)));
    };
    for (int attempt = 0; attempt < 4; ++attempt) {
        std::vector<int32_t> redo;
        for (int32_t k = 0; k < count; ++k)
            if ((out[k].status & ERR_ARENA) || (out[k].dual_oom && (uint64_t)out[k].arena_want > h->b_in[k].ws_bytes))
                redo.push_back(k);
        if (redo.empty()) break;
        uint64_t total = 0;
        for (int32_t k : redo) total += bigger(k);
        if (h->ws_fixed && total > h->ws_fixed) break;  // they stay out of workspace
        int rc = ensure_ws(h, total);
        if (rc) return rc;
        std::vector<int32_t> order(redo.size());
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(),
                         [&](int32_t x, int32_t y) { return h->b_cluster[redo[x]] > h->b_cluster[redo[y]]; });
        int32_t ncl = 0;
        for (int32_t k : redo) ncl += h->b_cluster[k];
        std::vector<Instance> sub(redo.size());
        uint64_t off = 0;
        for (size_t q = 0; q < redo.size(); ++q) {
            Instance &x = h->b_in[redo[q]];
            x.ws_bytes = bigger(redo[q]);
            x.ws = h->ws + off;
            off += x.ws_bytes;
            if (off > h->ws_bytes) return fail(RAMA_ERR_OOM, "workspace exhausted");
            sub[q] = x;
        }
        CU(cudaMemcpyAsync(h->d_inst, sub.data(), sizeof(Instance) * sub.size(), cudaMemcpyHostToDevice, h->b_stream));
        CU(cudaMemcpyAsync(h->d_order, order.data(), sizeof(int32_t) * order.size(), cudaMemcpyHostToDevice,
                           h->b_stream));
        rc = launch_solve(h, (int32_t)sub.size(), 1, h->b_stream, ncl);
        if (rc) return rc;
        CU(cudaMemcpyAsync(sub.data(), h->d_inst, sizeof(Instance) * sub.size(), cudaMemcpyDeviceToHost, h->b_stream));
        CU(cudaStreamSynchronize(h->b_stream));
        for (size_t q = 0; q < redo.size(); ++q) out[redo[q]] = sub[q];
    }
    int worst = RAMA_OK;
    int64_t peak = 0;
    double alg = 0.0;
    for (int32_t k = 0; k < count; ++k) {
        if (num_labels) num_labels[k] = out[k].num_labels;
        if (lbs) lbs[k] = out[k].lb;
        if (status) status[k] = status_from_bits(out[k].status);
        if (out[k].status && worst == RAMA_OK) worst = status_from_bits(out[k].status);
        peak = std::max<int64_t>(peak, out[k].arena_peak);
        alg += out[k].alg_bytes;
    }
    h->stats = rama_stats{};
    h->stats.team = 1;
    h->stats.workspace_peak = peak;
    h->stats.device_ms = ms;
    h->stats.alg_bytes = alg;
    if (worst) return fail(worst, "at least one instance failed (see status)");
    return RAMA_OK;
}

int rama_solve_batch(rama_handle h, const int32_t *d_i, const int32_t *d_j, const float *d_costs,
                     const int64_t *edge_offsets, int32_t count, const rama_options *opts, int32_t *d_labels,
                     const int64_t *label_offsets, int64_t *num_labels, double *lbs, int32_t *status, void *stream)
{
    int rc = rama_batch_launch(h, d_i, d_j, d_costs, edge_offsets, count, opts, 1, d_labels, label_offsets, stream);
    if (rc) return rc;
    return rama_batch_wait(h, num_labels, lbs, status);
}

int rama_get_tuning(rama_handle h, rama_tuning *out)
{
    if (!h || !out) return fail(RAMA_ERR_INVALID_ARG, "bad arguments");
    *out = h->tune;
    return RAMA_OK;
}

int rama_set_tuning(rama_handle h, const rama_tuning *t)
{
    if (!h || !t) return fail(RAMA_ERR_INVALID_ARG, "bad arguments");
    CU(cudaSetDevice(h->device));
    if (t->grid_ctas_per_sm < 1 || t->grid_ctas_per_sm > h->grid_per_sm_max || t->grid_small_ctas_per_sm < 1 ||
        t->grid_small_ctas_per_sm > h->grid_per_sm_max || t->grid_small_max < 0)
        return fail(RAMA_ERR_INVALID_ARG,
                    "grid CTAs per SM must lie in [1, " + std::to_string(h->grid_per_sm_max) + "]");
    const int c = t->cluster_ctas;
    if (!(c == 2 || c == 4 || c == 8 || c == 16)) return fail(RAMA_ERR_INVALID_ARG, "cluster_ctas must be 2, 4, 8 or 16");
    if (cluster_capacity(h, c) < 1)
        return fail(RAMA_ERR_INVALID_ARG, "no cluster of " + std::to_string(c) + " CTAs fits on this device");
    if (t->cta_threads != THREADS && t->cta_threads != THREADS_SMALL)
        return fail(RAMA_ERR_INVALID_ARG, "cta_threads must be " + std::to_string(THREADS) + " or " +
                                              std::to_string(THREADS_SMALL));
    if (t->single_cluster_min < 0 || t->single_grid_min < 0 || t->batch_cluster_min < 0 ||
        !(t->batch_cluster_share > 0.0f))
        return fail(RAMA_ERR_INVALID_ARG, "thresholds must be non-negative and the share positive");
    h->tune = *t;
    return RAMA_OK;
}

int rama_get_stats(rama_handle h, rama_stats *out)
{
    if (!h || !out) return fail(RAMA_ERR_INVALID_ARG, "bad arguments");
    *out = h->stats;
    return RAMA_OK;
}

int rama_parse_multicut(rama_handle h, const char *d_text, int64_t len, int32_t *d_i, int32_t *d_j, float *d_costs,
                        int64_t cap, int64_t *num_edges, void *stream)
{
    if (!h || len < 0 || (len > 0 && !d_text) || cap < 0 || (cap > 0 && (!d_i || !d_j || !d_costs)) || !num_edges)
        return fail(RAMA_ERR_INVALID_ARG, "bad arguments");
    CU(cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    // tokens: 8 + 4 bytes for at most len / 2 of them, plus the scratch partials
    int rc = ensure_ws(h, std::max<uint64_t>(h->ws_bytes, (uint64_t)len * 7 + (64ull << 20)));
    if (rc) return rc;
    if (h->ws_bytes < (uint64_t)len * 7 + (4ull << 20)) return fail(RAMA_ERR_OOM, "workspace too small for the text");
    int64_t *d_out = reinterpret_cast<int64_t *>(h->d_scalar);
    ParseLaunch L{d_text, len, d_i, d_j, d_costs, cap, d_out, h->ws, h->ws_bytes};
    void *args[] = {&L};
    CU(cudaLaunchCooperativeKernel((void *)k_parse_grid, dim3(h->parse_ctas), dim3(THREADS), args, SMEM, st));
    int64_t n = 0;
    CU(cudaMemcpyAsync(&n, d_out, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    if (n == -1) return fail(RAMA_ERR_INVALID_ARG, "first line must be 'MULTICUT'");
    if (n < 0) return fail(RAMA_ERR_OOM, "workspace too small for the text");
    *num_edges = n;
    return RAMA_OK;
}

int rama_parse_multicut_host(rama_handle h, const char *text, int64_t len, int32_t *i, int32_t *j, float *costs,
                             int64_t cap, int64_t *num_edges)
{
    if (!h || len < 0 || (len > 0 && !text) || cap < 0 || (cap > 0 && (!i || !j || !costs)) || !num_edges)
        return fail(RAMA_ERR_INVALID_ARG, "bad arguments");
    CU(cudaSetDevice(h->device));
    if (h->p_cap < std::max<int64_t>(len, 1)) {
        cudaFree(h->p_text);
        h->p_text = nullptr;
        h->p_cap = 0;
        CU(cudaMalloc(&h->p_text, (size_t)std::max<int64_t>(len, 1)));
        h->p_cap = std::max<int64_t>(len, 1);
    }
    const int64_t room = std::max<int64_t>(std::min<int64_t>(cap, (len + 1) / 6 + 1), 1);
    if (h->io_edges < room) {
        cudaFree(h->io_i);
        cudaFree(h->io_j);
        cudaFree(h->io_c);
        h->io_i = h->io_j = nullptr;
        h->io_c = nullptr;
        h->io_edges = 0;
        CU(cudaMalloc(&h->io_i, sizeof(int32_t) * (size_t)room));
        CU(cudaMalloc(&h->io_j, sizeof(int32_t) * (size_t)room));
        CU(cudaMalloc(&h->io_c, sizeof(float) * (size_t)room));
        h->io_edges = room;
    }
    cudaStream_t st = nullptr;
    if (len > 0) CU(cudaMemcpyAsync(h->p_text, text, (size_t)len, cudaMemcpyHostToDevice, st));
    int64_t n = 0;
    int rc = rama_parse_multicut(h, h->p_text, len, h->io_i, h->io_j, h->io_c, room, &n, st);
    if (rc) return rc;
    if (n > cap) n = cap;
    if (n > 0) {
        CU(cudaMemcpy(i, h->io_i, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(j, h->io_j, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost));
        CU(cudaMemcpy(costs, h->io_c, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost));
    }
    *num_edges = n;
    return RAMA_OK;
}

int rama_objective(rama_handle h, const int32_t *d_i, const int32_t *d_j, const float *d_costs, int64_t n,
                   const int32_t *d_labels, double *obj, void *stream)
{
    if (!h || !obj) return fail(RAMA_ERR_INVALID_ARG, "bad arguments");
    CU(cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    int rc = ensure_ws(h, std::max<uint64_t>(h->ws_bytes, (uint64_t)n / 4096 * 16 + (8u << 20)));
    if (rc) return rc;
    void *args[] = {(void *)&d_i, (void *)&d_j, (void *)&d_costs, (void *)&n, (void *)&d_labels,
                    (void *)&h->d_scalar, (void *)&h->ws, (void *)&h->ws_bytes};
    CU(cudaLaunchCooperativeKernel((void *)k_objective, dim3(h->obj_ctas), dim3(THREADS), args, SMEM, st));
    CU(cudaMemcpyAsync(obj, h->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    return RAMA_OK;
}

int rama_step(rama_handle h, rama_step_args *a, void *stream)
{
    if (!h || !a) return fail(RAMA_ERR_INVALID_ARG, "bad arguments");
    CU(cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    int64_t scale = std::max<int64_t>({a->n, a->m, a->T * 3, a->adj_len, (int64_t)a->num_nodes, a->map_size});
    int rc = ensure_ws(h, h->ws_fixed ? h->ws_fixed
                                      : ws_estimate(scale, a->tri_memory_factor) + (uint64_t)a->num_nodes * 64);
    if (rc) return rc;
    a->status = 0;
    CU(cudaMemcpyAsync(h->d_step, a, sizeof(rama_step_args), cudaMemcpyHostToDevice, st));
    if (a->team == 2) {
        void *args[] = {(void *)&h->d_step, (void *)&h->ws, (void *)&h->ws_bytes};
        CU(cudaLaunchCooperativeKernel((void *)k_step_grid, dim3(h->step_ctas), dim3(THREADS), args, SMEM, st));
    } else {
        k_step_cta<<<1, THREADS, SMEM, st>>>(h->d_step, h->ws, h->ws_bytes);
        CU(cudaGetLastError());
    }
    CU(cudaMemcpyAsync(a, h->d_step, sizeof(rama_step_args), cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    if (a->status) return fail(status_from_bits(a->status), "step status bits " + std::to_string(a->status));
    return RAMA_OK;
}

}  // extern "C"
