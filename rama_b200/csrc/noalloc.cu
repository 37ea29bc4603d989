// noalloc.cu -- rama_solve_small_static: solve one small instance without
// allocating any device memory.
//
// Who needs it: callers that must not call cudaMalloc.  For example, an
// application whose GPU memory is already fully reserved by its own pool
// allocator (a training or inference framework that has claimed the device)
// where an extra cudaMalloc fails or fragments the pool; a latency-critical
// loop that cannot afford cudaMalloc/cudaFree, which may synchronise the
// whole device; or a process that runs under a fixed, audited device-memory
// budget.  This entry point takes its scratch memory from one fixed array
// that is part of the library itself, so a call allocates nothing: the
// caller passes the inputs and the output buffer, as with rama_solve.
//
// The array is STATIC_BYTES (32 MiB) of device memory on every GPU that
// loads the library, held until the process exits.  It bounds the instance
// size: at most RAMA_STATIC_MAX_EDGES edges and node ids below
// RAMA_STATIC_MAX_NODES.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/rama_b200.h"
#include "solver.cuh"

using namespace rama;

// error text shared with the other entry points (capi.cu)
void rama_set_last_error(const std::string &msg);

namespace {

constexpr int THREADS = 512;
constexpr int SMEM = sort_smem_bytes(THREADS) + 1024;
constexpr uint64_t STATIC_BYTES = 32ull << 20;
constexpr uint64_t HEADER_BYTES = 4096;  // the instance descriptor (inputs, options, results)
static_assert(sizeof(Instance) <= HEADER_BYTES, "instance descriptor does not fit its header");

// The scratch array.  Host code must not hand this name to a kernel: on the
// host it only stands in for the symbol.  The device address comes from
// cudaGetSymbolAddress (scratch_address below).
static __device__ __align__(256) char g_static_scratch[STATIC_BYTES];

__global__ void __launch_bounds__(THREADS, 2) k_solve_static(char *scratch)
{
    extern __shared__ __align__(16) char sm[];
    BlockTeam t;
    Instance *io = reinterpret_cast<Instance *>(scratch);
    char *base = scratch + HEADER_BYTES;
    Scratch sc = scratch_over(base, STATIC_BYTES - HEADER_BYTES);
    // node ids must stay below the limit that the fixed size assumes
    const int32_t *I = io->i, *J = io->j;
    const int32_t mx = team_max<BlockTeam, int32_t>(t, sc, sm, io->n, -1,
                                                    [&](int64_t e) { return I[e] > J[e] ? I[e] : J[e]; });
    if (mx >= RAMA_STATIC_MAX_NODES) {
        if (threadIdx.x == 0) {
            io->status = ERR_INVALID_ARG;
            io->num_labels = 0;
        }
        return;
    }
    solve_instance(t, sm, sc, io);
}

std::mutex g_mutex;
char *g_address[256] = {};

// Device address of the scratch array on `device`, looked up once per device
// with that device current; the same first call raises the kernel's shared
// memory limit.
int scratch_address(int device, char **out)
{
    std::lock_guard<std::mutex> lock(g_mutex);
    if (device < 0 || device >= 256) return RAMA_ERR_INVALID_ARG;
    if (!g_address[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) {
            rama_set_last_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return RAMA_ERR_CUDA;
        }
        e = cudaFuncSetAttribute((const void *)k_solve_static, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
        if (e != cudaSuccess) {
            rama_set_last_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
            return RAMA_ERR_CUDA;
        }
        g_address[device] = static_cast<char *>(p);
    }
    *out = g_address[device];
    return RAMA_OK;
}

Options options_of(const rama_options *o)
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
    r.dump_timeline = 0;  // no timeline: it would need memory of its own
    r.verbose = o->verbose;
    r.sanitize_graph = o->sanitize_graph;
    r.woc_pentagons = o->woc_pentagons;
    return r;
}

int fail_static(int code, const std::string &msg)
{
    rama_set_last_error(msg);
    return code;
}

}  // namespace

extern "C" int rama_solve_small_static(const int32_t *d_i, const int32_t *d_j, const float *d_costs,
                                       int64_t num_edges, const rama_options *opts, int32_t *d_labels,
                                       int64_t labels_cap, int64_t *num_labels, double *lb, void *stream)
{
    if (!opts || num_edges < 0 || (num_edges > 0 && (!d_i || !d_j || !d_costs)))
        return fail_static(RAMA_ERR_INVALID_ARG, "rama_solve_small_static: bad arguments");
    if (num_edges > RAMA_STATIC_MAX_EDGES)
        return fail_static(RAMA_ERR_INVALID_ARG,
                           "rama_solve_small_static: " + std::to_string(num_edges) + " edges exceed the limit of " +
                               std::to_string(RAMA_STATIC_MAX_EDGES) + " (use rama_solve for larger instances)");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail_static(RAMA_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    char *scratch = nullptr;
    int rc = scratch_address(device, &scratch);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // The descriptor is rewritten in full by every call (its result fields
    // start at zero); the solver initialises every part of the workspace it
    // reads, so nothing left by an earlier call needs clearing.
    Instance hi{};
    hi.opts = options_of(opts);
    hi.i = d_i;
    hi.j = d_j;
    hi.c = d_costs;
    hi.n = num_edges;
    hi.labels = d_labels;
    hi.labels_cap = labels_cap;
    hi.timeline = nullptr;
    hi.prof = nullptr;
    hi.ws = nullptr;
    hi.ws_bytes = 0;
    e = cudaMemcpyAsync(scratch, &hi, sizeof(Instance), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return fail_static(RAMA_ERR_CUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
    k_solve_static<<<1, THREADS, SMEM, st>>>(scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_static(RAMA_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    Instance ho{};
    e = cudaMemcpyAsync(&ho, scratch, sizeof(Instance), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail_static(RAMA_ERR_CUDA, std::string("solve: ") + cudaGetErrorString(e));
    if (num_labels) *num_labels = ho.num_labels;
    if (lb) *lb = ho.lb;
    if (ho.status & ERR_INVALID_ARG)
        return fail_static(RAMA_ERR_INVALID_ARG,
                           "rama_solve_small_static: invalid input (negative id, self loop, node id >= " +
                               std::to_string(RAMA_STATIC_MAX_NODES) + ", or label buffer too small)");
    // a dual that ran out of scratch fell back to the trivial bound (the
    // reference's caught bad_alloc) and the solve went on: a result, as in
    // rama_solve; only a primal phase that ran out is an error
    if (ho.status & ERR_ARENA)
        return fail_static(RAMA_ERR_OOM,
                           "rama_solve_small_static: the instance needs more than the fixed 32 MiB workspace "
                           "(use rama_solve)");
    if (ho.status & ERR_BAD_CONTRACTION) return fail_static(RAMA_ERR_BAD_CONTRACTION, "Found bad contractions");
    if (ho.status) return fail_static(RAMA_ERR_ITER_LIMIT, "rama_solve_small_static: a bounded device loop gave up");
    return RAMA_OK;
}
