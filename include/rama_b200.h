/*
 * rama_b200.h -- C ABI of the B200 multicut solver (librama_b200.so).
 *
 * Plain pointers, sizes and a stream handle; no C++ or torch types.  The C++
 * overloads of the reference (rama_cuda.h), the rama_py Python module and the
 * rama_text_input CLI are thin layers over these entry points.
 *
 * Device pointers are CUDA device memory on the handle's device; `stream` is
 * a cudaStream_t (NULL = the legacy default stream).  Every entry point
 * returns a rama_status; rama_last_error() describes the last failure of the
 * calling thread.
 */
#ifndef RAMA_B200_H
#define RAMA_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    RAMA_OK = 0,
    RAMA_ERR_INVALID_ARG = 1,    /* bad ids (negative, self loop), short output buffer */
    RAMA_ERR_OOM = 2,            /* device memory / workspace exhausted */
    RAMA_ERR_CUDA = 3,           /* a CUDA runtime call failed */
    RAMA_ERR_ITER_LIMIT = 4,     /* a bounded device loop gave up */
    RAMA_ERR_BAD_CONTRACTION = 5 /* a contraction produced a negative cluster cost */
} rama_status;

/* Solver options.  The first 13 fields mirror multicut_solver_options
 * (reference include/multicut_solver_options.h:4-19) with the same meaning
 * and defaults; `team` is specific to this solver. */
typedef struct {
    int32_t max_cycle_length_lb;
    int32_t num_dual_itr_lb;
    int32_t max_cycle_length_primal;
    int32_t num_dual_itr_primal;
    int32_t num_outer_itr_dual;
    float mean_multiplier_mm;
    float matching_thresh_crossover_ratio;
    float tri_memory_factor;
    int32_t only_compute_lb;
    int32_t max_time_sec;
    int32_t dump_timeline;
    int32_t verbose;
    int32_t sanitize_graph;
    /* execution team: 1 = one CTA, 2 = whole GPU (cooperative grid), 3 = one cluster of 8
     * CTAs, 0 = choose by size (one CTA below 4,000 edges, a cluster below 100,000, else the
     * whole GPU).  In a batch, 1 keeps an instance on one CTA, 2 and 3 put it on a cluster,
     * and 0 puts it on a cluster when it has at least 20,000 edges and more than 1.5 times
     * the batch's edges per CTA. */
    int32_t team;
    /* 1: the forest contraction also cuts conflicted 5-cycles of the forest
     * (check_pentagons_cuda, src/edge_contractions_woc.cu:81-139, which the
     * reference ships disabled); 0 (default) as the reference. */
    int32_t woc_pentagons;
} rama_options;

/* Presets of multicut_solver_options(const std::string&) (reference
 * include/multicut_solver_options.h:22-53): NULL or "PD" (default), "P",
 * "PD+", "D".  Unknown names keep the defaults, as the reference does. */
int rama_options_init(rama_options *opts, const char *mode);

typedef struct rama_context *rama_handle;

/* A handle owns the device workspace (reused across calls) and its streams.
 * workspace_bytes = 0 picks a size from the first problem and grows it when
 * needed.  workspace_bytes > 0 fixes the workspace: it is allocated whole at
 * the first call and never grows; a batch whose instance slices (1024 bytes
 * per edge + 1 MiB per instance, rounded up to 4 KiB) add up to more is
 * refused with RAMA_ERR_OOM.  Not thread-safe: use one handle per host
 * thread. */
int rama_create(int device, uint64_t workspace_bytes, rama_handle *out);
void rama_destroy(rama_handle h);

/* Solve statistics of the last call on a handle. */
typedef struct {
    int32_t rounds;          /* contraction rounds */
    int32_t matching_rounds;
    int32_t mst_rounds;
    int32_t timeline_rounds;
    int32_t dual_oom;        /* the dual ran out of workspace and fell back to the trivial bound */
    int32_t team;            /* 1 = CTA, 2 = grid, 3 = cluster */
    int64_t triangles;       /* triangle counter of the initial dual's last pass */
    int64_t edges_after_dual;
    int64_t workspace_peak;  /* bytes */
    double device_ms;        /* kernel time of the solve (CUDA events) */
    double alg_bytes;        /* algorithmic bytes of the solve: minimum edge, map, arc and triangle
                                traffic of each phase, tallied on the device; no sort temporaries */
    double phase_ms[32];     /* time per phase: [0] init, [1] cycle search (classification),
                                [2] MP build (rest), [3] MP iterations + bound, [4] dual commit,
                                [5] matching (threshold), [6] forest contraction set (rest),
                                [7] contraction (after its sort), [8] other, [9] matching iterations
                                after the first, [10] contraction sort of buckets beyond 4096 edges,
                                [11] CSR builds, [12..14] contraction sort (endpoints and slots,
                                scatter, ordering in buckets), [15] contraction runs, [16] matching
                                labels, [17] first matching iteration, [18] forest MSF, [19] forest
                                lists, [20] forest components / checks / thresholds, [21] forest
                                rooting, [22] forest path lengths and cuts, [23] cycle expansions,
                                [24] triangle normalisation, [25] MP chords and merged edges,
                                [26] MP correspondence and incidence order; [27..31] unused */
    double phase_bytes[32];  /* algorithmic bytes per phase (same order), the parts of alg_bytes */
} rama_stats;

/*
 * Solve one instance on device pointers.  Replaces rama_cuda(device_vector&&
 * i, j, costs, opts, device) (reference include/rama_cuda.h:9,
 * src/rama_cuda.cu:195-212) and rama_cuda_gpu_pointers (src/rama_py.cu:61-74).
 * i, j, costs: num_edges entries (undirected edges, i != j, ids >= 0).
 * labels: capacity labels_cap; receives max node id + 1 cluster labels
 * (0 labels with only_compute_lb).  lb: the dual lower bound.
 */
int rama_solve(rama_handle h, const int32_t *d_i, const int32_t *d_j, const float *d_costs, int64_t num_edges,
               const rama_options *opts, int32_t *d_labels, int64_t labels_cap, int64_t *num_labels, double *lb,
               void *stream);

/*
 * Same on host memory (copies in and out).  Replaces the host overload
 * rama_cuda(const std::vector<int>& i, j, costs, opts) (reference
 * include/rama_cuda.h:8, src/rama_cuda.cu:166-193).  solve_ms: device time of
 * the solve excluding the copies, like the reference's returned duration.
 */
int rama_solve_host(rama_handle h, const int32_t *i, const int32_t *j, const float *costs, int64_t num_edges,
                    const rama_options *opts, int32_t *labels, int64_t labels_cap, int64_t *num_labels, double *lb,
                    double *solve_ms);

/* Per-round label snapshots of the last solve with dump_timeline set
 * (reference src/rama_cuda.cu:145-150): rounds x num_labels int32, host. */
int rama_get_timeline(rama_handle h, int32_t *out, int64_t cap, int32_t *rounds, int64_t *num_labels);

/*
 * Batched solve: `count` independent instances packed as a disjoint union.
 * Instance k owns edges [edge_offsets[k], edge_offsets[k+1]) of d_i/d_j/d_costs
 * (node ids local to the instance) and writes its labels to
 * d_labels + label_offsets[k] (capacity label_offsets[k+1]-label_offsets[k]).
 * edge_offsets / label_offsets / num_labels / lbs / status are host arrays.
 * Every instance is solved by one CTA; instances are dealt to CTAs largest
 * first.  The result of an instance does not depend on the rest of the batch.
 */
int rama_solve_batch(rama_handle h, const int32_t *d_i, const int32_t *d_j, const float *d_costs,
                     const int64_t *edge_offsets, int32_t count, const rama_options *opts, int32_t *d_labels,
                     const int64_t *label_offsets, int64_t *num_labels, double *lbs, int32_t *status, void *stream);

/*
 * Asynchronous batch (continuous batching): rama_batch_launch enqueues a batch
 * on `stream` and returns at once; rama_batch_poll returns 1 when it has
 * finished (0 while running, negative on error); rama_batch_wait blocks,
 * then fills the host result arrays.  opts holds 1 entry (shared) or `count`
 * entries (per instance).  Each instance gets a workspace slice sized from
 * its edge count (about 1 KiB per edge); the sum is the batch's footprint.
 * A batch of one instance whose options ask for team 2 runs on the whole GPU
 * (a cooperative launch; it starts once the SMs are free of other kernels).
 * One batch in flight per handle: a server keeps one handle per concurrent
 * batch.  No counterpart in the reference (it solves one instance per call).
 */
int rama_batch_launch(rama_handle h, const int32_t *d_i, const int32_t *d_j, const float *d_costs,
                      const int64_t *edge_offsets, int32_t count, const rama_options *opts, int32_t opts_count,
                      int32_t *d_labels, const int64_t *label_offsets, void *stream);
int rama_batch_poll(rama_handle h);
int rama_batch_wait(rama_handle h, int64_t *num_labels, double *lbs, int32_t *status);

/*
 * Solve one small instance without allocating any device memory.  For callers
 * that must not call cudaMalloc: an application whose device memory is fully
 * reserved by its own pool allocator, a latency-critical loop that cannot
 * afford cudaMalloc's device-wide synchronisation, or a process with a fixed
 * device-memory budget.  No counterpart in the reference.
 *
 * Same inputs, outputs and results as rama_solve (one CTA solves the
 * instance), but the scratch memory is one fixed 32 MiB array inside the
 * library, held on every GPU that loads it until the process exits.  Limits:
 * at most RAMA_STATIC_MAX_EDGES edges and node ids below
 * RAMA_STATIC_MAX_NODES; larger instances are rejected with
 * RAMA_ERR_INVALID_ARG, and an instance whose solve needs more scratch than
 * the array returns RAMA_ERR_OOM.  As in rama_solve, a dual that runs out of
 * scratch falls back to the trivial bound and the call still succeeds.
 * dump_timeline is ignored.  The call is synchronous: it returns once the
 * solve on `stream` has finished.
 * The array is device memory of the library's module: CUDA reserves it on a
 * device when the module loads there, which with lazy module loading (the
 * default) is the first call into the library on that device.  A caller whose
 * pool allocator claims the device's memory should make one call (for example
 * an empty instance) before the pool reserves its memory.
 * The first call on a device also looks up the array's device address and
 * sets the kernel's shared-memory limit.  All calls share the one array:
 * calls that overlap on the GPU (other streams or host threads) race and must
 * be serialised by the caller.
 */
#define RAMA_STATIC_MAX_EDGES 30000
#define RAMA_STATIC_MAX_NODES 65536
int rama_solve_small_static(const int32_t *d_i, const int32_t *d_j, const float *d_costs, int64_t num_edges,
                            const rama_options *opts, int32_t *d_labels, int64_t labels_cap, int64_t *num_labels,
                            double *lb, void *stream);

/* Reads MULTICUT text on the device (the reference's read_file,
 * src/multicut_text_parser.cpp:6-31): a first line "MULTICUT" (one trailing
 * '\r' allowed), then whitespace-separated triples "i j cost" up to the first
 * token that is not a number of its kind (int32, int32, float rounded to
 * nearest like strtof; a cost beyond FLT_MAX ends the input as in the
 * reference's stream extraction).  d_text: the text in device memory.  The
 * triples go to d_i, d_j, d_costs (capacity `cap`; (len + 1) / 6 + 1 always
 * suffices); *num_edges receives their count.  RAMA_ERR_INVALID_ARG when the
 * first line is not "MULTICUT". */
int rama_parse_multicut(rama_handle h, const char *d_text, int64_t len, int32_t *d_i, int32_t *d_j, float *d_costs,
                        int64_t cap, int64_t *num_edges, void *stream);
/* The same with the text and the triples in host memory (the text is copied
 * to the device, parsed there, and the triples copied back). */
int rama_parse_multicut_host(rama_handle h, const char *text, int64_t len, int32_t *i, int32_t *j, float *costs,
                             int64_t cap, int64_t *num_edges);

/* Launch parameters of a handle.  None of them changes a result (every team
 * computes the same solve, bit for bit); they only decide how the GPU's SMs
 * are spent.  rama_create starts from built-in values;
 * rama_b200/autotune.py measures better ones per device and sets them.  No
 * counterpart in the reference (its launches have fixed shapes). */
typedef struct {
    int32_t grid_ctas_per_sm;    /* CTAs per SM of the whole-GPU solve (1 .. the occupancy maximum) ... */
    int32_t grid_small_ctas_per_sm; /* ... and of one of fewer than grid_small_max edges */
    int64_t grid_small_max;
    int32_t cluster_ctas;        /* CTAs of a cluster team: 2, 4, 8 or 16 */
    int64_t single_cluster_min;  /* a single solve of at least this many edges runs on a cluster ... */
    int64_t single_grid_min;     /* ... and from this many on on the whole GPU (else on one CTA) */
    int64_t batch_cluster_min;   /* batch instances below this size always run on one CTA; larger ones on */
    float batch_cluster_share;   /* a cluster when they hold more than this many times the batch's edges
                                    per CTA */
    int32_t cta_threads;         /* threads of a CTA that solves instances alone: 512 (two per SM) or
                                    256 (three per SM, more instances in flight) */
} rama_tuning;
int rama_get_tuning(rama_handle h, rama_tuning *out);
/* RAMA_ERR_INVALID_ARG for a value outside its range or a cluster size that
 * does not fit on the device. */
int rama_set_tuning(rama_handle h, const rama_tuning *t);

int rama_get_stats(rama_handle h, rama_stats *out);
const char *rama_last_error(void);

/* Objective of a labelling: sum of the costs of edges whose endpoints carry
 * different labels, a compensated FP64 sum (reference get_obj,
 * include/rama_utils.h:192-205). */
int rama_objective(rama_handle h, const int32_t *d_i, const int32_t *d_j, const float *d_costs, int64_t num_edges,
                   const int32_t *d_labels, double *obj, void *stream);

/* ---- single solver steps, for parity tests and profiling ---------------- */
enum {
    RAMA_STEP_INIT = 1,       /* (i,j,c) -> sorted graph            dCOO::init       src/dCOO.cu:28-55 */
    RAMA_STEP_CONTRACT = 2,   /* graph + map -> contracted graph     contract_cuda    src/dCOO.cu:57-95 */
    RAMA_STEP_MATCHING = 3,   /* graph -> map, nr                    rama_cuda.cu:54-62 */
    RAMA_STEP_WOC = 4,        /* graph -> map, nr                    edge_contractions_woc.cu:387-423
                                 (max_cycle_length >= 5 adds the pentagon check, :81-139) */
    RAMA_STEP_MSF = 5,        /* (i,j,w) -> chosen flags             gpuMST.cu:364-388 */
    RAMA_STEP_CC = 6,         /* CSR -> labels                       ECL-CC_11.cu:315-350 */
    RAMA_STEP_CYCLES = 7,     /* graph -> triangles                  conflicted_cycles_cuda.cu:222-343 */
    RAMA_STEP_MP = 8,         /* graph + triangles -> lb0, lb1, reparametrised edges (multicut_message_passing.cu) */
    RAMA_STEP_DUAL = 9,       /* graph -> lb, reparametrised graph   dual_solver.cu:37-63 */
    RAMA_STEP_CSUM = 10,      /* float array -> compensated sum */
    RAMA_STEP_SORT = 11,      /* (uint64 key, int32 value) pairs -> stable sorted */
    RAMA_STEP_COARSEN = 12    /* graph + map -> the solver's contraction: contract_cuda, has_bad_contractions
                                 and remove_diagonal (src/dCOO.cu:57-152); out_nr = 1 on a bad contraction */
};

typedef struct {
    int32_t op;
    int32_t team; /* 1 = one CTA, 2 = cooperative grid */
    /* sorted graph input */
    const int32_t *row, *col;
    const float *cost;
    int64_t n;
    int32_t rows, cols;
    /* raw edge / array input */
    const int32_t *i, *j;
    const float *c;
    int64_t m;
    const uint64_t *keys;
    int32_t key_bits;
    /* node map input */
    const int32_t *map;
    int64_t map_size;
    /* triangle input */
    const int32_t *t1, *t2, *t3;
    int64_t T;
    /* CSR input */
    const int32_t *offsets, *adj;
    int32_t num_nodes;
    int64_t adj_len;
    /* parameters */
    int32_t max_cycle_length, num_iter, num_outer;
    float tri_memory_factor, mean_multiplier_mm, tol;
    /* outputs (device) */
    int32_t *out_row, *out_col;
    float *out_cost;
    int64_t out_cap;
    int32_t *out_map;
    int64_t out_map_cap;
    int32_t *out_t1, *out_t2, *out_t3;
    int64_t out_tri_cap;
    uint8_t *out_flags;
    uint64_t *out_keys;
    /* scalar outputs */
    int64_t out_n;
    int32_t out_rows, out_cols;
    int64_t out_count, out_raw;
    int32_t out_nr;
    double out_lb0, out_lb1;
    int32_t status;
} rama_step_args;

int rama_step(rama_handle h, rama_step_args *args, void *stream);

#ifdef __cplusplus
}
#endif
#endif
