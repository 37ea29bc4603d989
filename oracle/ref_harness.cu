// ref_harness.cu -- C entry points onto the reference solver's own components
// (TEST INFRASTRUCTURE).  Compiled together with the reference sources, where
// they lie, by oracle/build_ref.sh into oracle/_ref/librama_ref.so.  Tests call
// these to check the CPU oracle and the CUDA path step by step against the
// reference on identical inputs; bench.py's reference arm calls ref_rama*.
//
// Every entry point takes host pointers, copies them into the reference's
// containers, calls the reference function named in its comment and copies
// the result back.  Exceptions become negative return codes.
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include <thrust/copy.h>
#include <thrust/device_vector.h>
#include <thrust/host_vector.h>

#include "ECLgraph.h"
#include "conflicted_cycles_cuda.h"
#include "dCOO.h"
#include "dual_solver.h"
// The forest contraction's 5-cycle check is a private member that the
// reference never calls (the call at src/edge_contractions_woc.cu:414 is
// commented out).  To pin the oracle's optional pentagon step against the
// reference's own kernel, this test harness opens the class and runs the same
// sequence as find_contraction_mapping with that call enabled.
#define private public
#include "edge_contractions_woc.h"
#undef private
#include "edge_contractions_woc_thrust.h"
#include "gpuMST.h"
#include "maximum_matching_vertex_based.h"
#include "multicut_message_passing.h"
#include "multicut_solver_options.h"
#include "rama_cuda.h"
#include "rama_utils.h"

namespace {
thread_local std::string g_err;

dCOO make_sorted(int64_t E, const int *row, const int *col, const float *cost, int rows, int cols)
{
    thrust::device_vector<int> r(row, row + E), c(col, col + E);
    thrust::device_vector<float> w(cost, cost + E);
    return dCOO(rows, cols, std::move(c), std::move(r), std::move(w), true, true);
}

void export_coo(const dCOO &A, int64_t *E_out, int *row_out, int *col_out, float *cost_out, int *rows_out,
                int *cols_out, int64_t cap)
{
    const int64_t E = (int64_t)A.nnz();
    *E_out = E;
    if (rows_out) *rows_out = (int)A.rows();
    if (cols_out) *cols_out = (int)A.cols();
    if (E > cap) throw std::runtime_error("output capacity too small");
    thrust::copy(A.get_row_ids().begin(), A.get_row_ids().end(), row_out);
    thrust::copy(A.get_col_ids().begin(), A.get_col_ids().end(), col_out);
    thrust::copy(A.get_data().begin(), A.get_data().end(), cost_out);
}

multicut_solver_options make_opts(const int32_t *oi, const float *of)
{
    multicut_solver_options o;
    o.max_cycle_length_lb = oi[0];
    o.num_dual_itr_lb = oi[1];
    o.max_cycle_length_primal = oi[2];
    o.num_dual_itr_primal = oi[3];
    o.num_outer_itr_dual = oi[4];
    o.only_compute_lb = oi[5] != 0;
    o.max_time_sec = oi[6];
    o.dump_timeline = oi[7] != 0;
    o.sanitize_graph = oi[8] != 0;
    o.verbose = false;
    o.mean_multiplier_mm = of[0];
    o.matching_thresh_crossover_ratio = of[1];
    o.tri_memory_factor = of[2];
    return o;
}
}  // namespace

#define GUARD_BEGIN try {
#define GUARD_END                                  \
    }                                              \
    catch (const std::bad_alloc &e)                \
    {                                              \
        g_err = e.what();                          \
        return -2;                                 \
    }                                              \
    catch (const std::exception &e)                \
    {                                              \
        g_err = e.what();                          \
        return -1;                                 \
    }                                              \
    return 0;

extern "C" {

const char *ref_last_error() { return g_err.c_str(); }

// dCOO(i, j, costs, directed) + init (src/dCOO.cu:28-55)
int ref_init(int64_t E, const int *i, const int *j, const float *c, int64_t *E_out, int *row_out, int *col_out,
             float *cost_out, int *rows_out, int *cols_out)
{
    GUARD_BEGIN
    thrust::device_vector<int> di(i, i + E), dj(j, j + E);
    thrust::device_vector<float> dc(c, c + E);
    dCOO A(std::move(di), std::move(dj), std::move(dc), true);
    export_coo(A, E_out, row_out, col_out, cost_out, rows_out, cols_out, E);
    GUARD_END
}

// dCOO::contract_cuda (src/dCOO.cu:57-95)
int ref_contract(int64_t E, const int *row, const int *col, const float *cost, int rows, int cols, const int *map,
                 int64_t map_size, int64_t *E_out, int *row_out, int *col_out, float *cost_out, int *rows_out,
                 int *cols_out)
{
    GUARD_BEGIN
    dCOO A = make_sorted(E, row, col, cost, rows, cols);
    thrust::device_vector<int> m(map, map + map_size);
    dCOO B = A.contract_cuda(m);
    export_coo(B, E_out, row_out, col_out, cost_out, rows_out, cols_out, E);
    GUARD_END
}

// filter_edges_by_matching_vertex_based + compress_label_sequence (src/rama_cuda.cu:54-62)
int ref_matching(int64_t E, const int *row, const int *col, const float *cost, int rows, int cols, float mm,
                 int *map_out, int64_t map_cap, int64_t *map_size, int *nr)
{
    GUARD_BEGIN
    dCOO A = make_sorted(E, row, col, cost, rows, cols);
    thrust::device_vector<int> node_mapping;
    int nr_matched;
    std::tie(node_mapping, nr_matched) = filter_edges_by_matching_vertex_based(A.export_undirected(), mm, false);
    thrust::device_vector<int> comp = compress_label_sequence(node_mapping, node_mapping.size() - 1);
    if ((int64_t)comp.size() > map_cap) throw std::runtime_error("map capacity too small");
    thrust::copy(comp.begin(), comp.end(), map_out);
    *map_size = (int64_t)comp.size();
    *nr = nr_matched;
    GUARD_END
}

// computeCC_gpu (external/ECL-CC/ECL-CC_11.cu:315-350)
int ref_cc(int n, const int *offsets, int64_t m, const int *cols, int *labels)
{
    GUARD_BEGIN
    thrust::device_vector<int> off(offsets, offsets + n + 1), c(cols, cols + m), lab(n);
    computeCC_gpu(n, (int)m, thrust::raw_pointer_cast(off.data()), thrust::raw_pointer_cast(c.data()),
                  thrust::raw_pointer_cast(lab.data()), 0);
    cudaDeviceSynchronize();
    thrust::copy(lab.begin(), lab.end(), labels);
    GUARD_END
}

// MST_boruvka::maximum_spanning_tree (external/cudaMST/gpuMST/gpuMST.cu:364-388)
int ref_msf(int64_t m, const int *i, const int *j, const float *w, int *mi, int *mj, float *mw, int64_t *k)
{
    GUARD_BEGIN
    thrust::device_vector<int> di(i, i + m), dj(j, j + m);
    thrust::device_vector<float> dw(w, w + m);
    thrust::device_vector<int> ri, rj;
    thrust::device_vector<float> rw;
    std::tie(ri, rj, rw) = MST_boruvka::maximum_spanning_tree(di, dj, dw);
    thrust::copy(ri.begin(), ri.end(), mi);
    thrust::copy(rj.begin(), rj.end(), mj);
    thrust::copy(rw.begin(), rw.end(), mw);
    *k = (int64_t)ri.size();
    GUARD_END
}

// conflicted_cycles_cuda (src/conflicted_cycles_cuda.cu:222-343); returns all
// slots the reference returns (zero padding included when the budget is hit)
int ref_conflicted_cycles(int64_t E, const int *row, const int *col, const float *cost, int rows, int cols,
                          int max_len, float tri_factor, float tol, int *tri_out, int64_t cap, int64_t *num)
{
    GUARD_BEGIN
    dCOO A = make_sorted(E, row, col, cost, rows, cols);
    thrust::device_vector<int> t1, t2, t3;
    std::tie(t1, t2, t3) = conflicted_cycles_cuda(A, max_len, tri_factor, tol, false);
    const int64_t T = (int64_t)t1.size();
    *num = T;
    if (T > cap) throw std::runtime_error("triangle capacity too small");
    std::vector<int> h1(T), h2(T), h3(T);
    thrust::copy(t1.begin(), t1.end(), h1.begin());
    thrust::copy(t2.begin(), t2.end(), h2.begin());
    thrust::copy(t3.begin(), t3.end(), h3.begin());
    for (int64_t k = 0; k < T; ++k) {
        tri_out[3 * k] = h1[k];
        tri_out[3 * k + 1] = h2[k];
        tri_out[3 * k + 2] = h3[k];
    }
    GUARD_END
}

// multicut_message_passing (src/multicut_message_passing.cu:65-360): build,
// LB, optional send_messages_to_triplets, `iters` iterations, LB, export edges.
int ref_mp(int64_t E, const int *row, const int *col, const float *cost, int rows, int cols, int64_t T,
           const int *t1, const int *t2, const int *t3, int pre_triplets, int iters, double *lb0, double *lb1,
           int64_t *E_out, int *row_out, int *col_out, float *cost_out, int64_t cap)
{
    GUARD_BEGIN
    dCOO A = make_sorted(E, row, col, cost, rows, cols);
    thrust::device_vector<int> a(t1, t1 + T), b(t2, t2 + T), c(t3, t3 + T);
    multicut_message_passing mp(A, std::move(a), std::move(b), std::move(c), false);
    *lb0 = mp.lower_bound();
    if (pre_triplets) mp.send_messages_to_triplets();
    for (int k = 0; k < iters; ++k) mp.iteration();
    *lb1 = mp.lower_bound();
    const auto &rep = mp.reparametrized_edge_costs();
    const auto &ri = std::get<0>(rep);
    const auto &rj = std::get<1>(rep);
    const auto &rc = std::get<2>(rep);
    *E_out = (int64_t)ri.size();
    if ((int64_t)ri.size() > cap) throw std::runtime_error("edge capacity too small");
    thrust::copy(ri.begin(), ri.end(), row_out);
    thrust::copy(rj.begin(), rj.end(), col_out);
    thrust::copy(rc.begin(), rc.end(), cost_out);
    GUARD_END
}

// dual_solver (src/dual_solver.cu:37-63): replaces A, returns the LB
int ref_dual(int64_t E, const int *row, const int *col, const float *cost, int rows, int cols, int max_len,
             int num_iter, float tri_factor, int num_outer, double *lb, int64_t *E_out, int *row_out, int *col_out,
             float *cost_out, int *rows_out, int *cols_out, int64_t cap)
{
    GUARD_BEGIN
    dCOO A = make_sorted(E, row, col, cost, rows, cols);
    *lb = dual_solver(A, max_len, num_iter, tri_factor, num_outer, 1e-4, false);
    export_coo(A, E_out, row_out, col_out, cost_out, rows_out, cols_out, cap);
    GUARD_END
}

// edge_contractions_woc (src/edge_contractions_woc.cu:341-423)
int ref_woc(int64_t E, const int *row, const int *col, const float *cost, int rows, int cols, int *map_out,
            int64_t map_cap, int64_t *map_size, int *nr)
{
    GUARD_BEGIN
    dCOO A = make_sorted(E, row, col, cost, rows, cols);
    edge_contractions_woc w(A, false);
    thrust::device_vector<int> m;
    int n;
    std::tie(m, n) = w.find_contraction_mapping();
    if ((int64_t)m.size() > map_cap) throw std::runtime_error("map capacity too small");
    thrust::copy(m.begin(), m.end(), map_out);
    *map_size = (int64_t)m.size();
    *nr = n;
    GUARD_END
}

// edge_contractions_woc::find_contraction_mapping (src/edge_contractions_woc.cu:386-423)
// with its commented-out check_pentagons() call (:414) enabled
int ref_woc_pentagons(int64_t E, const int *row, const int *col, const float *cost, int rows, int cols, int *map_out,
                      int64_t map_cap, int64_t *map_size, int *nr)
{
    GUARD_BEGIN
    dCOO A = make_sorted(E, row, col, cost, rows, cols);
    edge_contractions_woc w(A, false);
    *map_size = 0;
    *nr = 0;
    if (w.mst_row_ids.size() > 0) {
        w.filter_by_cc();
        if (w.check_triangles()) w.filter_by_cc();
        w.check_quadrangles();
        w.check_pentagons();
        edge_contractions_woc_thrust mapper(w.num_nodes, std::move(w.mst_row_ids), std::move(w.mst_col_ids),
                                            std::move(w.mst_data), std::move(w.rep_row_ids),
                                            std::move(w.rep_col_ids), std::move(w.cc_labels), false);
        thrust::device_vector<int> m;
        int n;
        std::tie(m, n) = mapper.find_contraction_mapping();
        if ((int64_t)m.size() > map_cap) throw std::runtime_error("map capacity too small");
        thrust::copy(m.begin(), m.end(), map_out);
        *map_size = (int64_t)m.size();
        *nr = n;
    }
    GUARD_END
}

// rama_cuda host overload (src/rama_cuda.cu:166-193)
int ref_rama(int64_t E, const int *i, const int *j, const float *c, const int32_t *oi, const float *of,
             int *labels_out, int64_t cap, int64_t *num_labels, double *lb, int *time_ms)
{
    GUARD_BEGIN
    std::vector<int> vi(i, i + E), vj(j, j + E);
    std::vector<float> vc(c, c + E);
    multicut_solver_options o = make_opts(oi, of);
    std::vector<int> labels;
    double l;
    int t;
    std::vector<std::vector<int>> tl;
    std::tie(labels, l, t, tl) = rama_cuda(vi, vj, vc, o);
    *num_labels = (int64_t)labels.size();
    if ((int64_t)labels.size() > cap) throw std::runtime_error("label capacity too small");
    std::memcpy(labels_out, labels.data(), sizeof(int) * labels.size());
    *lb = l;
    *time_ms = t;
    GUARD_END
}

// rama_cuda device overload (src/rama_cuda.cu:195-212) on device pointers
// (the rama_cuda_gpu_pointers path, src/rama_py.cu:61-74)
int ref_rama_device(int64_t E, const int *d_i, const int *d_j, const float *d_c, const int32_t *oi, const float *of,
                    int *d_labels_out, int64_t cap, int64_t *num_labels, double *lb)
{
    GUARD_BEGIN
    thrust::device_vector<int> vi(thrust::device_pointer_cast(d_i), thrust::device_pointer_cast(d_i) + E);
    thrust::device_vector<int> vj(thrust::device_pointer_cast(d_j), thrust::device_pointer_cast(d_j) + E);
    thrust::device_vector<float> vc(thrust::device_pointer_cast(d_c), thrust::device_pointer_cast(d_c) + E);
    multicut_solver_options o = make_opts(oi, of);
    thrust::device_vector<int> labels;
    double l;
    std::vector<std::vector<int>> tl;
    int dev = 0;
    cudaGetDevice(&dev);
    std::tie(labels, l, tl) = rama_cuda(std::move(vi), std::move(vj), std::move(vc), o, dev);
    *num_labels = (int64_t)labels.size();
    if ((int64_t)labels.size() > cap) throw std::runtime_error("label capacity too small");
    thrust::copy(labels.begin(), labels.end(), thrust::device_pointer_cast(d_labels_out));
    cudaDeviceSynchronize();
    *lb = l;
    GUARD_END
}

}  // extern "C"
