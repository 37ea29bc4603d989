// prims.cuh -- team-generic parallel primitives (scan, canonical sums,
// stable compaction, LSD radix sort, CSR offsets, connected components).
//
// All results are independent of the team size: order-sensitive primitives
// split the input into one contiguous chunk per CTA, and the floating-point
// sums follow fixed reduction trees (CSUM, RSUM) that are defined by element
// index only.
#pragma once
#include <cstdint>
#include <type_traits>

#include "team.cuh"

namespace rama {

constexpr unsigned FULL = 0xffffffffu;

// ---------------------------------------------------------------------------
// per-team scratch: double-buffered block partials (a primitive that writes a
// partial array always uses the buffer its predecessor did not use, so a CTA
// that runs ahead never overwrites partials another CTA is still reading),
// plus the arena.
// ---------------------------------------------------------------------------
struct Scratch {
    Arena arena;
    char *part[2];  // each >= 16 * (nblocks + 2) bytes
    int32_t *err;   // set when a bounded wait gave up (zeroed at the start of a solve)
    int parity;
    double alg_bytes;  // algorithmic bytes of the work done (team-uniform tally)
    int64_t *prof;     // optional: per-phase nanoseconds [0, PH_COUNT), then per-phase
                       // algorithmic bytes [PH_COUNT, 2 PH_COUNT) (leader only)
    uint64_t tlast;
    double alg_last;   // alg_bytes at the last phase mark
    __device__ __forceinline__ char *next_part()
    {
        parity ^= 1;
        return part[parity];
    }
};

// A workspace of `bytes` bytes at `base` (256-byte aligned) holds the two
// partial buffers, the error word and then the arena.
constexpr uint64_t SCRATCH_PART_BYTES = 16 * 4096;  // >= 16 * (max CTAs + 2)

__device__ __forceinline__ Scratch scratch_over(char *base, uint64_t bytes)
{
    Scratch sc;
    sc.part[0] = base;
    sc.part[1] = base + SCRATCH_PART_BYTES;
    sc.err = reinterpret_cast<int32_t *>(base + 2 * SCRATCH_PART_BYTES);
    sc.parity = 0;
    sc.alg_bytes = 0.0;
    sc.prof = nullptr;
    sc.tlast = 0;
    sc.alg_last = 0.0;
    sc.arena.base = base;
    sc.arena.cap = bytes - 256;
    sc.arena.lo = 2 * SCRATCH_PART_BYTES + 256;
    sc.arena.top = sc.arena.cap;
    sc.arena.peak = sc.arena.lo;
    sc.arena.want = 0;
    sc.arena.failed = 0;
    return sc;
}

// Phase timing: the team leader charges the time since the last mark, and
// the algorithmic bytes tallied since then, to `phase`.  Marks sit right
// after team syncs, so a phase's time is the span in which the whole team
// worked on it.
enum Phase : int {
    PH_INIT = 0,
    PH_CYCLES = 1,
    PH_MP_BUILD = 2,
    PH_MP_ITER = 3,
    PH_DUAL_COMMIT = 4,
    PH_MATCHING = 5,
    PH_WOC = 6,
    PH_CONTRACT = 7,
    PH_OTHER = 8,
    PH_MATCH_ITER = 9,    // the offer / match iterations of a matching round
    PH_CSORT_BIG = 10,    // contraction sort: the buckets of more than BUCKET_MAX edges
    PH_CSR = 11,          // symmetric CSR builds (cycle search, forest)
    PH_CSORT_SLOT = 12,   // contraction sort: endpoints and bucket slots
    PH_CSORT_SCATTER = 13,  // ... bucket starts and the scatter
    PH_CSORT_RANK = 14,   // ... ordering within the buckets
    PH_CONTRACT_RUNS = 15,  // contraction: run heads, sums, the new edges
    PH_MATCH_LABELS = 16,   // matching: labels of the contraction map
    PH_MATCH_FIRST = 17,    // matching: the first offer / match iteration (reads every edge)
    PH_WOC_MSF = 18,        // forest: attractive edges and their maximum spanning forest
    PH_WOC_CSR = 19,        // forest: the forest's symmetric lists
    PH_WOC_CHECKS = 20,     // forest: components, cycle checks, thresholds
    PH_WOC_ROOT = 21,       // forest: rooting (level-synchronous BFS)
    PH_WOC_PATHS = 22,      // forest: path lengths and bottleneck cuts
    PH_CYC_SEARCH = 23,     // cycle search: the expansions after the CSR
    PH_MP_NORM = 24,        // message passing: triangle normalisation
    PH_MP_CHORDS = 25,      // message passing: chords and the merged edge list
    PH_MP_INCID = 26,       // message passing: triangle-edge correspondence, incidence order
    PH_COUNT = 27
};

__device__ __forceinline__ uint64_t prof_now()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <class Team>
__device__ __forceinline__ void prof_mark(const Team &t, Scratch &sc, int phase)
{
    if (sc.prof && t.leader()) {
        uint64_t now = prof_now();
        sc.prof[phase] += (int64_t)(now - sc.tlast);
        sc.prof[PH_COUNT + phase] += (int64_t)(sc.alg_bytes - sc.alg_last);
        sc.tlast = now;
    }
    sc.alg_last = sc.alg_bytes;
}

// ---------------------------------------------------------------------------
// block-level helpers (all threads of the CTA must call)
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ T warp_incl_scan(T v)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T n = __shfl_up_sync(FULL, v, o);
        if (lane_id() >= o) v += n;
    }
    return v;
}

template <class T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// exclusive scan over the CTA; `sm` needs 34 * sizeof(T) bytes
template <class T>
__device__ __forceinline__ T block_excl_scan(T v, T *sm, T &total)
{
    const int w = warp_in_block(), nw = blockDim.x >> 5;
    T inc = warp_incl_scan(v);
    if (lane_id() == 31) sm[w] = inc;
    __syncthreads();
    if (w == 0) {
        T x = lane_id() < nw ? sm[lane_id()] : T(0);
        T xi = warp_incl_scan(x);
        sm[lane_id()] = xi - x;
        if (lane_id() == 31) sm[32] = xi;
    }
    __syncthreads();
    T r = sm[w] + inc - v;
    total = sm[32];
    __syncthreads();
    return r;
}

template <class T>
__device__ __forceinline__ T block_sum(T v, T *sm)
{
    T t;
    block_excl_scan(v, sm, t);
    return t;
}

template <class T>
__device__ __forceinline__ T block_max(T v, T *sm)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T n = __shfl_xor_sync(FULL, v, o);
        v = n > v ? n : v;
    }
    if (lane_id() == 0) sm[warp_in_block()] = v;
    __syncthreads();
    T r = sm[0];
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) r = sm[k] > r ? sm[k] : r;
    __syncthreads();
    return r;
}

template <class T>
__device__ __forceinline__ T block_min(T v, T *sm)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T n = __shfl_xor_sync(FULL, v, o);
        v = n < v ? n : v;
    }
    if (lane_id() == 0) sm[warp_in_block()] = v;
    __syncthreads();
    T r = sm[0];
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) r = sm[k] < r ? sm[k] : r;
    __syncthreads();
    return r;
}

// contiguous chunk of [0,n) owned by this CTA (multiple of blockDim)
template <class Team>
__device__ __forceinline__ void block_chunk(const Team &t, int64_t n, int64_t &lo, int64_t &hi)
{
    const int64_t nb = t.nblocks();
    int64_t ch = (n + nb - 1) / nb;
    ch = (ch + blockDim.x - 1) / blockDim.x * blockDim.x;
    lo = (int64_t)t.block() * ch;
    hi = lo + ch;
    if (lo > n) lo = n;
    if (hi > n) hi = n;
}

// ---------------------------------------------------------------------------
// team reductions (integer / min / max): one team sync
// ---------------------------------------------------------------------------

// Combines the per-CTA partials part[0, nb) written before the last team
// sync.  Every warp reads them with independent L2 loads (ld.global.cg: the
// values come from other SMs, so L1 must not serve them) spread over its
// lanes, then combines the lanes; the result is valid on every lane.  Only
// for exact operations (integer sums, min, max), whose result does not depend
// on the combination order.
template <class T, class Op>
__device__ __forceinline__ T warp_fold_parts(const T *part, int nb, T init, Op op)
{
    T r = init;
    for (int b = lane_id(); b < nb; b += 32) r = op(r, __ldcg(part + b));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = op(r, __shfl_xor_sync(FULL, r, o));
    return r;
}

// Grid-stride loop over [0, n) in batches of U strides: load(i) for every
// item of a batch first (loads only), then store(i, value) for each, so a
// batch waits for one memory round trip instead of U.  Per thread the items
// keep their order; a load must not read what the store of an earlier item
// of the same thread writes.
template <int U = 4, class Team, class Load, class Store>
__device__ __forceinline__ void team_for_batched(const Team &t, int64_t n, Load load, Store store)
{
    const int64_t S = t.size();
    int64_t i0 = t.rank();
    for (; i0 + (U - 1) * S < n; i0 += S * U) {
        decltype(load(int64_t(0))) v[U];
#pragma unroll
        for (int k = 0; k < U; ++k) v[k] = load(i0 + k * S);
#pragma unroll
        for (int k = 0; k < U; ++k) store(i0 + k * S, v[k]);
    }
    for (; i0 < n; i0 += S) store(i0, load(i0));
}

// the sum over the team of one value per thread; one team sync
template <class Team, class T>
__device__ T team_total(const Team &t, Scratch &sc, char *sm, T v)
{
    const T s = block_sum<T>(v, reinterpret_cast<T *>(sm));
    T *part = reinterpret_cast<T *>(sc.next_part());
    if (threadIdx.x == 0) part[t.block()] = s;
    t.sync();
    return warp_fold_parts<T>(part, t.nblocks(), T(0), [](T a, T b) { return a + b; });
}

template <class Team, class T, class Get>
__device__ T team_sum(const Team &t, Scratch &sc, char *sm, int64_t n, Get get)
{
    T s = T(0);
    {
        // four strides at a time, loads issued together
        constexpr int U = 4;
        const int64_t S = t.size();
        int64_t i = t.rank();
        for (; i + (U - 1) * S < n; i += U * S) {
            T v[U];
#pragma unroll
            for (int k = 0; k < U; ++k) v[k] = get(i + k * S);
#pragma unroll
            for (int k = 0; k < U; ++k) s += v[k];
        }
        for (; i < n; i += S) s += get(i);
    }
    s = block_sum<T>(s, reinterpret_cast<T *>(sm));
    T *part = reinterpret_cast<T *>(sc.next_part());
    if (threadIdx.x == 0) part[t.block()] = s;
    t.sync();
    return warp_fold_parts<T>(part, t.nblocks(), T(0), [](T a, T b) { return a + b; });
}

template <class Team, class T, class Get>
__device__ T team_max(const Team &t, Scratch &sc, char *sm, int64_t n, T init, Get get)
{
    T s = init;
    {
        constexpr int U = 4;
        const int64_t S = t.size();
        int64_t i = t.rank();
        for (; i + (U - 1) * S < n; i += U * S) {
            T x[U];
#pragma unroll
            for (int k = 0; k < U; ++k) x[k] = get(i + k * S);
#pragma unroll
            for (int k = 0; k < U; ++k) s = x[k] > s ? x[k] : s;
        }
        for (; i < n; i += S) {
            T x = get(i);
            s = x > s ? x : s;
        }
    }
    s = block_max<T>(s, reinterpret_cast<T *>(sm));
    T *part = reinterpret_cast<T *>(sc.next_part());
    if (threadIdx.x == 0) part[t.block()] = s;
    t.sync();
    return warp_fold_parts<T>(part, t.nblocks(), init, [](T a, T b) { return b > a ? b : a; });
}

template <class Team, class T, class Get>
__device__ T team_min(const Team &t, Scratch &sc, char *sm, int64_t n, T init, Get get)
{
    T s = init;
    for (int64_t i = t.rank(); i < n; i += t.size()) {
        T x = get(i);
        s = x < s ? x : s;
    }
    s = block_min<T>(s, reinterpret_cast<T *>(sm));
    T *part = reinterpret_cast<T *>(sc.next_part());
    if (threadIdx.x == 0) part[t.block()] = s;
    t.sync();
    return warp_fold_parts<T>(part, t.nblocks(), init, [](T a, T b) { return b < a ? b : a; });
}

// The maximum of ia(i) and the minimum of fb(i) over [0, n) in one pass and
// one team sync (both exact, so the result does not depend on the order).
template <class Team, class IA, class FB>
__device__ void team_maxi_minf(const Team &t, Scratch &sc, char *sm, int64_t n, int32_t iinit, float finit, IA ia,
                               FB fb, int32_t &imax, float &fmin)
{
    int32_t a = iinit;
    float b = finit;
    {
        constexpr int U = 4;
        const int64_t S = t.size();
        int64_t i = t.rank();
        for (; i + (U - 1) * S < n; i += U * S) {
            int32_t x[U];
            float y[U];
#pragma unroll
            for (int k = 0; k < U; ++k) {
                x[k] = ia(i + k * S);
                y[k] = fb(i + k * S);
            }
#pragma unroll
            for (int k = 0; k < U; ++k) {
                a = x[k] > a ? x[k] : a;
                b = y[k] < b ? y[k] : b;
            }
        }
        for (; i < n; i += S) {
            const int32_t x = ia(i);
            const float y = fb(i);
            a = x > a ? x : a;
            b = y < b ? y : b;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int32_t x = __shfl_xor_sync(FULL, a, o);
        const float y = __shfl_xor_sync(FULL, b, o);
        a = x > a ? x : a;
        b = y < b ? y : b;
    }
    int32_t *sa = reinterpret_cast<int32_t *>(sm);
    float *sb = reinterpret_cast<float *>(sm + 128);
    if (lane_id() == 0) {
        sa[warp_in_block()] = a;
        sb[warp_in_block()] = b;
    }
    __syncthreads();
    a = sa[0];
    b = sb[0];
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
        a = sa[k] > a ? sa[k] : a;
        b = sb[k] < b ? sb[k] : b;
    }
    __syncthreads();
    int32_t *part = reinterpret_cast<int32_t *>(sc.next_part());  // 16 B per block
    if (threadIdx.x == 0) {
        part[2 * t.block()] = a;
        part[2 * t.block() + 1] = __float_as_int(b);
    }
    t.sync();
    a = iinit;
    b = finit;
    for (int k = lane_id(); k < t.nblocks(); k += 32) {
        const int32_t x = __ldcg(part + 2 * k);
        const float y = __int_as_float(__ldcg(part + 2 * k + 1));
        a = x > a ? x : a;
        b = y < b ? y : b;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int32_t x = __shfl_xor_sync(FULL, a, o);
        const float y = __shfl_xor_sync(FULL, b, o);
        a = x > a ? x : a;
        b = y < b ? y : b;
    }
    imax = a;
    fmin = b;
}

// ---------------------------------------------------------------------------
// team exclusive scan: out(i, prefix, value) is called for every i in [0,n)
// in chunk order; returns the total.  Two team syncs; outputs are visible to
// the whole team on return.  The second pass takes tiles of blockDim * ITEMS
// elements (ITEMS = 4 for 8-byte sums, 8 for 4-byte ones): each warp a contiguous segment of 32 * SCAN_ITEMS,
// lane l its elements l, l + 32, ... (coalesced loads); the warp scans them
// in order with shuffles, and one block scan of the warp totals per tile
// keeps the CTA's barriers few.  Integer sums only, so the result does not
// depend on the tiling.
// ---------------------------------------------------------------------------
template <class T>
struct ScanItems {
    static constexpr int value = sizeof(T) == 8 ? 4 : 8;
};

template <class Team, class T, class In, class Out>
__device__ T team_scan(const Team &t, Scratch &sc, char *sm, int64_t n, In in, Out out)
{
    constexpr int ITEMS = ScanItems<T>::value;
    T *tsm = reinterpret_cast<T *>(sm);
    int64_t lo, hi;
    block_chunk(t, n, lo, hi);
    T s = T(0);
    {
        // four strides at a time, loads issued together
        constexpr int U = 4;
        const int64_t S = blockDim.x;
        int64_t i = lo + threadIdx.x;
        for (; i + (U - 1) * S < hi; i += U * S) {
            T v[U];
#pragma unroll
            for (int k = 0; k < U; ++k) v[k] = in(i + k * S);
#pragma unroll
            for (int k = 0; k < U; ++k) s += v[k];
        }
        for (; i < hi; i += S) s += in(i);
    }
    s = block_sum<T>(s, tsm);
    T *part = reinterpret_cast<T *>(sc.next_part());
    if (threadIdx.x == 0) part[t.block()] = s;
    t.sync();
    T base = T(0), total = T(0);
    for (int b = lane_id(); b < t.nblocks(); b += 32) {
        T x = __ldcg(part + b);
        if (b < t.block()) base += x;
        total += x;
    }
    base = warp_sum(base);
    total = warp_sum(total);
    const int64_t TILE = (int64_t)blockDim.x * ITEMS;
    const int64_t wseg = (int64_t)warp_in_block() * 32 * ITEMS;
    for (int64_t tile = lo; tile < hi; tile += TILE) {
        const int64_t i0 = tile + wseg + lane_id();
        T v[ITEMS], ex[ITEMS];
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) v[k] = i0 + 32 * k < hi ? in(i0 + 32 * k) : T(0);
        T wrun = T(0);
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
            const T x = warp_incl_scan(v[k]);
            ex[k] = wrun + x - v[k];
            wrun += __shfl_sync(FULL, x, 31);
        }
        T ts;
        const T wofs = base + block_excl_scan<T>(lane_id() == 0 ? wrun : T(0), tsm, ts);
        const T wbase = __shfl_sync(FULL, wofs, 0);
#pragma unroll
        for (int k = 0; k < ITEMS; ++k)
            if (i0 + 32 * k < hi) out(i0 + 32 * k, wbase + ex[k], v[k]);
        base += ts;
    }
    t.sync();
    return total;
}

// stable compaction: emit(i, pos) for every kept i; returns the count
template <class Team, class Keep, class Emit>
__device__ int64_t team_compact(const Team &t, Scratch &sc, char *sm, int64_t n, Keep keep, Emit emit)
{
    return team_scan<Team, int64_t>(
        t, sc, sm, n, [&](int64_t i) -> int64_t { return keep(i) ? 1 : 0; },
        [&](int64_t i, int64_t pos, int64_t v) {
            if (v) emit(i, pos);
        });
}

// ---------------------------------------------------------------------------
// CSUM: compensated FP64 sum over a fixed tree (chunks of 4096 elements, 32
// lane-strided TwoSum partials per chunk, pairwise tree over lanes; the same
// scheme over the chunk partials).  Bit-identical to the CPU oracle.
// ---------------------------------------------------------------------------
struct csum_t {
    double s, c;
};

__device__ __forceinline__ csum_t cs_merge(csum_t a, csum_t b)
{
    double s = __dadd_rn(a.s, b.s);
    double bb = __dsub_rn(s, a.s);
    double e = __dadd_rn(__dsub_rn(a.s, __dsub_rn(s, bb)), __dsub_rn(b.s, bb));
    csum_t r;
    r.s = s;
    r.c = __dadd_rn(__dadd_rn(a.c, b.c), e);
    return r;
}

__device__ __forceinline__ csum_t cs_warp_tree(csum_t a)
{
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        csum_t o;
        o.s = __shfl_down_sync(FULL, a.s, off);
        o.c = __shfl_down_sync(FULL, a.c, off);
        if ((lane_id() & (2 * off - 1)) == 0) a = cs_merge(a, o);
    }
    return a;
}

// returns the sum on every thread; two team syncs.  *count receives the
// number of k with cnt(k) (an exact integer sum computed in the same pass).
template <class Team, class Get, class Cnt>
__device__ double team_csum_count(const Team &t, Scratch &sc, int64_t n, Get get, Cnt cnt, int64_t *count)
{
    const int64_t nch = (n + 4095) / 4096;
    uint64_t m = sc.arena.mark();
    csum_t *parts = sc.arena.take<csum_t>(nch + 1);
    int64_t *pcnt = sc.arena.take<int64_t>(nch + 1);
    double *res = reinterpret_cast<double *>(sc.next_part());
    if (sc.arena.ok()) {
        const int64_t w = team_warp(t), nw = team_nwarps(t);
        for (int64_t ch = w; ch < nch; ch += nw) {
            csum_t a = {0.0, 0.0};
            int64_t c = 0;
            const int64_t b0 = ch * 4096 + lane_id();
            // 8 of the lane's 128 elements loaded at a time, merged in order;
            // the values stay as get returns them (a float takes one register)
            // until their merge, and full chunks need no bounds checks
            using V = decltype(get(int64_t(0)));
            if (ch * 4096 + 4096 <= n) {
                for (int k = 0; k < 128; k += 8) {
                    V x[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int64_t idx = b0 + 32 * (k + j);
                        x[j] = get(idx);
                        c += cnt(idx) ? 1 : 0;
                    }
#pragma unroll
                    for (int j = 0; j < 8; ++j) a = cs_merge(a, csum_t{(double)x[j], 0.0});
                }
            } else {
                for (int k = 0; k < 128; ++k) {
                    const int64_t idx = b0 + 32 * k;
                    if (idx < n) {
                        a = cs_merge(a, csum_t{(double)get(idx), 0.0});
                        c += cnt(idx) ? 1 : 0;
                    }
                }
            }
            a = cs_warp_tree(a);
            c = warp_sum(c);
            if (lane_id() == 0) {
                parts[ch] = a;
                pcnt[ch] = c;
            }
        }
    }
    t.sync();
    if (sc.arena.ok() && t.block() == 0 && warp_in_block() == 0) {
        csum_t a = {0.0, 0.0};
        int64_t c = 0;
        // a lane merges partials k, k + 32, ... in order, eight loaded at a time
        int64_t k = lane_id();
        for (; k + 7 * 32 < nch; k += 8 * 32) {
            csum_t x[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                x[j] = parts[k + 32 * j];
                c += pcnt[k + 32 * j];
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) a = cs_merge(a, x[j]);
        }
        for (; k < nch; k += 32) {
            a = cs_merge(a, parts[k]);
            c += pcnt[k];
        }
        a = cs_warp_tree(a);
        c = warp_sum(c);
        if (lane_id() == 0) {
            res[0] = __dadd_rn(a.s, a.c);
            reinterpret_cast<int64_t *>(res)[1] = c;
        }
    }
    t.sync();
    double r = uread(&res[0]);
    *count = uread(&reinterpret_cast<int64_t *>(res)[1]);
    sc.arena.release(m);
    // `res` lies in one of the two partial buffers: the next primitive uses the
    // other one, and the one after it can write this one only after a team
    // sync that every thread reaches after this read
    return r;
}

// The same in a function of its own.  Inlined into the whole-GPU solve, the
// matching threshold's sum took about 1.7x as long as called out of line
// (the solver's live state crowds the FP64 loop).  Elsewhere (the bound of
// message passing, the smaller teams) the call cost more than it saved, so
// only that call site uses it.
template <class Team, class Get, class Cnt>
__device__ __noinline__ double team_csum_count_outlined(const Team &t, Scratch &sc, int64_t n, Get get, Cnt cnt,
                                                        int64_t *count)
{
    return team_csum_count(t, sc, n, get, cnt, count);
}

template <class Team, class Get>
__device__ double team_csum(const Team &t, Scratch &sc, int64_t n, Get get)
{
    int64_t unused = 0;
    return team_csum_count(t, sc, n, get, [](int64_t) { return false; }, &unused);
}

// RSUM over values v(k), k in [0,n) by ONE thread (n <= 32): the oracle's
// 32-lane FP64 sum with one element per lane, then a pairwise tree over the
// lanes (empty lanes hold +0.0).  Computed with a stack of complete subtrees,
// which merges exactly the same pairs in the same order.
template <class Get>
__device__ __forceinline__ float rsum_serial(int n, Get v)
{
    double st[7];
    int sz[7];
    int top = 0;
    for (int k = 0; k < n; ++k) {
        double x = __dadd_rn(0.0, (double)v(k));
        int s = 1;
        while (top > 0 && sz[top - 1] == s) {
            x = __dadd_rn(st[top - 1], x);
            s <<= 1;
            --top;
        }
        st[top] = x;
        sz[top] = s;
        ++top;
    }
    double r = 0.0;
    if (top > 0) {
        r = st[top - 1];
        for (int q = top - 2; q >= 0; --q) r = __dadd_rn(st[q], r);
    }
    return (float)r;
}

// The same sum by one thread for n <= 8 values at p[0, n): the loads are
// independent and issued together, then a fixed tree over 8 values padded
// with +0.0.  Adding an exact zero changes no sum, so this equals
// rsum_serial(n, p[k]).
constexpr int RSUM_THREAD_MAX = 8;

__device__ __forceinline__ float rsum_upto8(const float *p, int n)
{
    double x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = k < n ? __dadd_rn(0.0, (double)p[k]) : 0.0;
    const double a = __dadd_rn(__dadd_rn(x[0], x[1]), __dadd_rn(x[2], x[3]));
    const double b = __dadd_rn(__dadd_rn(x[4], x[5]), __dadd_rn(x[6], x[7]));
    return (float)__dadd_rn(a, b);
}

// The same sum by one thread for n <= 32 values at p[0, n): the complete
// tree over 32 lanes (+0.0 in the empty ones) is the pairwise sum of four
// complete trees over 8 (each as in rsum_upto8), so this equals
// rsum_serial(n, p[k]); the loads of a group of 8 are issued together.
__device__ __forceinline__ float rsum_upto32(const float *p, int n)
{
    double g[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        double x[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = 8 * q + k < n ? __dadd_rn(0.0, (double)p[8 * q + k]) : 0.0;
        g[q] = __dadd_rn(__dadd_rn(__dadd_rn(x[0], x[1]), __dadd_rn(x[2], x[3])),
                         __dadd_rn(__dadd_rn(x[4], x[5]), __dadd_rn(x[6], x[7])));
    }
    return (float)__dadd_rn(__dadd_rn(g[0], g[1]), __dadd_rn(g[2], g[3]));
}

// Sums of more than RSUM_CHUNK values are defined by chunks: each chunk of
// RSUM_CHUNK consecutive values is summed as above (kept in double), and the
// chunk sums are summed the same way (chunk c to lane c mod 32), so that many
// warps can share one long sum.
constexpr int64_t RSUM_CHUNK = 4096;

// the pairwise tree over a warp's 32 lane values; the result on every lane
__device__ __forceinline__ double rsum_lane_tree(double a)
{
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        double o = __shfl_down_sync(FULL, a, off);
        if ((lane_id() & (2 * off - 1)) == 0) a = __dadd_rn(a, o);
    }
    return __shfl_sync(FULL, a, 0);
}

// the RSUM of at most RSUM_CHUNK values v(0..len) by a warp, in double (not
// rounded); a lane adds its values k, k + 32, ... in that order, eight of them
// loaded at a time
template <class Get>
__device__ __forceinline__ double rsum_chunk_warp(int64_t len, Get v)
{
    double a = 0.0;
    int64_t k = lane_id();
    for (; k + 7 * 32 < len; k += 8 * 32) {
        float x[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = v(k + 32 * j);
#pragma unroll
        for (int j = 0; j < 8; ++j) a = __dadd_rn(a, (double)x[j]);
    }
    for (; k < len; k += 32) a = __dadd_rn(a, (double)v(k));
    return rsum_lane_tree(a);
}

// the same sum by a whole warp (any n); result valid on every lane
template <class Get>
__device__ __forceinline__ float rsum_warp(int64_t n, Get v)
{
    if (n <= RSUM_CHUNK) return (float)rsum_chunk_warp(n, v);
    double acc = 0.0;  // this lane's chunks: c = lane, lane + 32, ...
    for (int64_t c = 0; c * RSUM_CHUNK < n; ++c) {
        const int64_t base = c * RSUM_CHUNK;
        const int64_t len = n - base < RSUM_CHUNK ? n - base : RSUM_CHUNK;
        const double d = rsum_chunk_warp(len, [&](int64_t k) { return v(base + k); });
        if (lane_id() == (int)(c & 31)) acc = __dadd_rn(acc, d);
    }
    return (float)rsum_lane_tree(acc);
}

// ---------------------------------------------------------------------------
// LSD radix sort of (uint64 key, 4- or 8-byte value) pairs, 8-bit digits, stable.
// The sorted data ends in (*keys, *vals) (pointers may be swapped with the
// spare buffers).
//
// One read of the keys counts the digits of every pass at once (a pass only
// permutes the keys, so its digit totals are known up front).  Each pass then
// moves the data once.  The input is cut into tiles of blockDim * SORT_ITEMS
// keys (half as many with 8-byte values); CTA b takes tiles b, b + nblocks,
// ... in increasing order.  Per tile it
//   - ranks the keys stably: per-warp digit counters, and ballots over the
//     digit bits for the lanes holding the same digit;
//   - finds the tile's output offset per digit by decoupled look-back over
//     the counts the preceding tiles published;
//   - stages the tile in digit order in shared memory and writes each digit's
//     run contiguously.
// One team sync per pass.  The look-back waits are bounded; a wait that gives
// up sets the scratch error word and the sort stops with the last complete
// pass (a permutation of the input).  A single-CTA team keeps running
// offsets instead of looking back.  A pass in which one digit holds every key
// is the identity and is skipped.
// ---------------------------------------------------------------------------
constexpr int SORT_ITEMS = 8;
constexpr uint64_t LB_VALUE = (uint64_t(1) << 58) - 1;
constexpr uint64_t LB_AGG = uint64_t(1) << 62;     // tile count published
constexpr uint64_t LB_PREFIX = uint64_t(2) << 62;  // inclusive prefix published
constexpr int LB_SPIN_LIMIT = 1 << 20;

__device__ __forceinline__ uint64_t ld_relaxed(const uint64_t *p)
{
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint64_t *p, uint64_t v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// values travel through shared memory as raw 4- or 8-byte words
template <class V>
struct SortWord {
    static_assert(sizeof(V) == 4 || sizeof(V) == 8, "sort values are 4 or 8 bytes");
    using type = typename std::conditional<sizeof(V) == 8, uint64_t, uint32_t>::type;
    static __device__ __forceinline__ type to(V v)
    {
        type u;
        memcpy(&u, &v, sizeof(V));
        return u;
    }
    static __device__ __forceinline__ V from(type u)
    {
        V v;
        memcpy(&v, &u, sizeof(V));
        return v;
    }
};

// Decoupled look-back of one tile for all 256 digits: the exclusive count of
// digit d over tiles [0, tile) in the words of pass tag `tag`.  The CTA loads
// the published words of LB_WINDOW preceding tiles per digit at once (into
// `win`, LB_WINDOW * 256 words of shared memory); each digit's thread then
// adds tile counts from the nearest tile back until it meets an inclusive
// prefix, or a tile that has not published yet (the next window starts
// there).  Called by every thread of the CTA; returns the count on threads
// d < 256.  Waits are bounded: after LB_SPIN_LIMIT rounds without progress
// the error word is set and the count is left incomplete.
constexpr int LB_WINDOW = 16;

// bytes of the sort's staging area: a tile of keys and values, or the
// look-back window, whichever is larger
__host__ __device__ constexpr int sort_stage_bytes(int threads)
{
    return threads * SORT_ITEMS * 12 > LB_WINDOW * 256 * 8 ? threads * SORT_ITEMS * 12 : LB_WINDOW * 256 * 8;
}

__device__ __forceinline__ int64_t sort_lookback(const uint64_t *flags, int64_t tile, uint64_t tag, uint64_t *win,
                                                 int64_t *posS, int32_t *err)
{
    const int d = threadIdx.x;
    int64_t excl = 0;
    bool done = tile == 0;
    if (d < 256) posS[d] = done ? -1 : tile - 1;
    int idle = 0;
    for (;;) {
        if (!__syncthreads_or(d < 256 && !done)) break;
        for (int x = threadIdx.x; x < LB_WINDOW * 256; x += blockDim.x) {
            const int64_t j = posS[x & 255] - (x >> 8);
            if (posS[x & 255] >= 0) win[x] = j >= 0 ? ld_relaxed(flags + j * 256 + (x & 255)) : (LB_PREFIX | tag);
        }
        __syncthreads();
        bool stuck = false;
        if (d < 256 && !done) {
            int64_t pos = posS[d];
            int k = 0;
            for (; k < LB_WINDOW; ++k) {
                const uint64_t w = win[k * 256 + d];
                if ((w & (uint64_t(15) << 58)) != tag || !(w >> 62)) break;  // not published yet
                excl += (int64_t)(w & LB_VALUE);
                if ((w >> 62) == 2) {
                    done = true;
                    break;
                }
            }
            stuck = k == 0 && !done;
            pos -= k;
            if (done) pos = -1;
            posS[d] = pos;
        }
        if (__syncthreads_or(stuck)) {
            if (++idle > LB_SPIN_LIMIT || (idle % 1024 == 0 && *(volatile int32_t *)err)) {
                if (d == 0) atomicOr(err, 1);
                break;
            }
            if (idle > 16) __nanosleep(256);
        } else {
            idle = 0;
        }
    }
    return excl;
}

// Lanes of the warp holding the same 9-bit label (a digit, or 256 for "no
// key"), from nine ballots over the label's bits.
__device__ __forceinline__ unsigned warp_peers9(unsigned label)
{
    unsigned m = FULL;
#pragma unroll
    for (int b = 0; b < 9; ++b) {
        const unsigned bit = (label >> b) & 1u;
        const unsigned ball = __ballot_sync(FULL, bit);
        m &= bit ? ball : ~ball;
    }
    return m;
}

template <class Team, class V>
__device__ void team_sort_pairs(const Team &t, Scratch &sc, char *sm, uint64_t *&keys, V *&vals, uint64_t *&keys2,
                                V *&vals2, int64_t n, int bits)
{
    if (n <= 1 || bits <= 0) return;
    using W = typename SortWord<V>::type;
    constexpr int ITEMS = sizeof(V) == 8 ? SORT_ITEMS / 2 : SORT_ITEMS;
    const int P = (bits + 7) / 8;
    const int nb = t.nblocks();
    const int NW = blockDim.x >> 5;
    const int TILE = blockDim.x * ITEMS;
    const int64_t ntiles = (n + TILE - 1) / TILE;
    uint64_t am = sc.arena.mark();
    uint32_t *ghist = sc.arena.take<uint32_t>(8 * 256);
    uint64_t *flags = nb > 1 ? sc.arena.take<uint64_t>((uint64_t)ntiles * 256) : nullptr;
    if (!sc.arena.ok()) return;
    uint32_t *wcnt = reinterpret_cast<uint32_t *>(sm);  // NW * 256
    uint64_t *skeys = reinterpret_cast<uint64_t *>(sm + NW * 1024);
    W *svals = reinterpret_cast<W *>(sm + NW * 1024 + TILE * 8);
    char *q = sm + NW * 1024 + sort_stage_bytes(blockDim.x);  // staging area: either tile or the window
    uint32_t *tstart = reinterpret_cast<uint32_t *>(q);
    int64_t *gbase = reinterpret_cast<int64_t *>(q + 1024);
    int64_t *bucket = reinterpret_cast<int64_t *>(q + 3072);
    int64_t *run = reinterpret_cast<int64_t *>(q + 5120);
    int64_t *ssm = reinterpret_cast<int64_t *>(q + 7168);   // 34
    int64_t *posS = reinterpret_cast<int64_t *>(q + 7440);  // 256
    uint64_t *win = skeys;                                  // LB_WINDOW * 256, look-back only
    uint32_t *lh = reinterpret_cast<uint32_t *>(skeys);    // P * 256, counting only
    const int w = warp_in_block();

    // 0. digit totals of every pass
    for (int i = threadIdx.x; i < P * 256; i += blockDim.x) lh[i] = 0;
    for (int64_t i = t.rank(); i < 8 * 256; i += t.size()) ghist[i] = 0;
    if (flags)
        for (int64_t i = t.rank(); i < ntiles * 256; i += t.size()) flags[i] = 0;
    __syncthreads();
    for (int64_t i = t.rank(); i < n; i += t.size()) {
        const uint64_t k = keys[i];
        for (int p = 0; p < P; ++p) atomicAdd(&lh[p * 256 + (int)((k >> (8 * p)) & 255)], 1u);
    }
    __syncthreads();
    t.sync();
    for (int i = threadIdx.x; i < P * 256; i += blockDim.x)
        if (lh[i]) atomicAdd(&ghist[i], lh[i]);
    t.sync();

    for (int p = 0; p < P; ++p) {
        const int shift = 8 * p;
        const uint64_t tag = (uint64_t)(p + 1) << 58;
        const int64_t tot = threadIdx.x < 256 ? (int64_t)__ldcg(ghist + p * 256 + threadIdx.x) : 0;
        int64_t all;
        const int64_t ex = block_excl_scan<int64_t>(tot, ssm, all);
        if (threadIdx.x < 256) {
            bucket[threadIdx.x] = ex;
            run[threadIdx.x] = 0;
        }
        if (__syncthreads_or(threadIdx.x < 256 && tot == n)) continue;  // identity pass
        for (int64_t tile = t.block(); tile < ntiles; tile += nb) {
            const int64_t t0 = tile * TILE;
            const int tn = (int)((n - t0) < TILE ? (n - t0) : TILE);
            for (int d = lane_id(); d < 256; d += 32) wcnt[w * 256 + d] = 0;
            uint64_t mk[ITEMS];
            W mv[ITEMS];
            uint32_t mr[ITEMS];
            const int wb = w * 32 * ITEMS;
#pragma unroll
            for (int k = 0; k < ITEMS; ++k) {
                const int li = wb + k * 32 + lane_id();
                const bool valid = li < tn;
                mk[k] = valid ? keys[t0 + li] : 0;
                mv[k] = valid ? SortWord<V>::to(vals[t0 + li]) : W(0);
            }
            __syncwarp();
            // 1. stable rank within the warp
#pragma unroll
            for (int k = 0; k < ITEMS; ++k) {
                const bool valid = wb + k * 32 + lane_id() < tn;
                const int d = valid ? (int)((mk[k] >> shift) & 255) : 256;
                const unsigned peers = warp_peers9((unsigned)d);
                const int leader = __ffs(peers) - 1;
                uint32_t b0 = 0;
                if (valid && lane_id() == leader) {
                    b0 = wcnt[w * 256 + d];
                    wcnt[w * 256 + d] = b0 + __popc(peers);
                }
                b0 = __shfl_sync(FULL, b0, leader);
                mr[k] = b0 + __popc(peers & lanemask_lt());
                __syncwarp();
            }
            __syncthreads();
            // 2. per digit: offsets of the warps, the tile's count and start
            uint32_t cnt = 0;
            if (threadIdx.x < 256) {
                for (int qw = 0; qw < NW; ++qw) {
                    const uint32_t c = wcnt[qw * 256 + threadIdx.x];
                    wcnt[qw * 256 + threadIdx.x] = cnt;
                    cnt += c;
                }
            }
            int64_t tt;
            const int64_t ts = block_excl_scan<int64_t>((int64_t)cnt, ssm, tt);
            // 3. output offset of the tile per digit
            if (threadIdx.x < 256) tstart[threadIdx.x] = (uint32_t)ts;
            int64_t excl = 0;
            if (nb == 1) {
                if (threadIdx.x < 256) {
                    excl = run[threadIdx.x];
                    run[threadIdx.x] = excl + cnt;
                }
            } else {
                if (threadIdx.x < 256)
                    st_relaxed(flags + tile * 256 + threadIdx.x, (tile == 0 ? LB_PREFIX : LB_AGG) | tag | (uint64_t)cnt);
                excl = sort_lookback(flags, tile, tag, win, posS, sc.err);
                if (threadIdx.x < 256 && tile > 0)
                    st_relaxed(flags + tile * 256 + threadIdx.x, LB_PREFIX | tag | (uint64_t)(excl + cnt));
            }
            if (threadIdx.x < 256) gbase[threadIdx.x] = bucket[threadIdx.x] + excl;
            __syncthreads();
            // 4. stage the tile in digit order
#pragma unroll
            for (int k = 0; k < ITEMS; ++k) {
                if (wb + k * 32 + lane_id() < tn) {
                    const int d = (int)((mk[k] >> shift) & 255);
                    const uint32_t loc = tstart[d] + wcnt[w * 256 + d] + mr[k];
                    skeys[loc] = mk[k];
                    svals[loc] = mv[k];
                }
            }
            __syncthreads();
            // 5. write the digit runs
            for (int i = threadIdx.x; i < tn; i += blockDim.x) {
                const uint64_t key = skeys[i];
                const int d = (int)((key >> shift) & 255);
                const int64_t dst = gbase[d] + (i - (int64_t)tstart[d]);
                if (dst >= 0 && dst < n) {
                    keys2[dst] = key;
                    vals2[dst] = SortWord<V>::from(svals[i]);
                }
            }
            __syncthreads();
        }
        t.sync();
        if (__ldcg(sc.err)) break;  // keep the last complete pass
        uint64_t *tk = keys;
        keys = keys2;
        keys2 = tk;
        V *tv = vals;
        vals = vals2;
        vals2 = tv;
    }
    sc.arena.release(am);
}

// shared-memory bytes the sort needs for a CTA of `threads` threads
__host__ __device__ constexpr int sort_smem_bytes(int threads)
{
    return (threads / 32) * 1024 + sort_stage_bytes(threads) + 7440 + 256 * 8;
}

// ---------------------------------------------------------------------------
// Bucket sort: n items ordered by (bucket(i), sub(i)), bucket(i) in [0, nb),
// sub(i) below 2^64 - 1.  Items with equal (bucket, sub) end in no particular
// order: callers fold the item index into sub when the order must be stable,
// and otherwise use it only where equal keys stand for equal items.  Each item takes a slot in
// its bucket by an atomic counter (one atomic per bucket and warp), an
// exclusive scan of the counts gives the bucket starts, one scatter places
// the items, and each bucket is then sorted by its sub keys: buckets of up to
// 64 items by ranking every item (it lands after the keys of its bucket that
// are smaller), up to 256 items by a warp and up to BUCKET_MAX by a CTA
// (bitonic networks in shared memory).  The
// atomic slots only decide where an item lands before its bucket is sorted,
// so with distinct keys the result is the one sorted order.
// Outputs: keys_out[p] = sub of the p-th item, idx_out[p] = its index,
// bstart[0, nb] = first position of each bucket.  Returns false, having
// written nothing useful, when a bucket holds more than BUCKET_MAX items (the
// caller then sorts with team_sort_pairs).
// ---------------------------------------------------------------------------
constexpr int BUCKET_MAX = 4096;

// bitonic sort of (key, idx) pairs in shared memory, `m` items padded to the
// power of two P with +inf keys; threads [lo, lo + nth) of the group work,
// `bar` synchronises them
template <class Bar>
__device__ __forceinline__ void smem_bitonic(uint64_t *key, int32_t *idx, int m, int P, int lane, int nth, Bar bar)
{
    for (int i = m + lane; i < P; i += nth) {
        key[i] = ~uint64_t(0);
        idx[i] = -1;
    }
    bar();
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < P; i += nth) {
                const int x = i ^ j;
                if (x > i) {
                    const uint64_t a = key[i], b = key[x];
                    if ((a > b) == ((i & k) == 0)) {
                        key[i] = b;
                        key[x] = a;
                        const int32_t t = idx[i];
                        idx[i] = idx[x];
                        idx[x] = t;
                    }
                }
            }
            bar();
        }
    }
}

// The general form: the slot pass calls bk_slot(i) once per item (it may
// store what it computes for the scatter pass), the scatter pass calls
// bucket(i), sub(i) and pay(i); idx_out receives pay(i) of each item instead of
// its index (team_bucket_sort below: pay(i) = i), and bucket_out, if given, the
// bucket of each sorted position.
//
// Buckets of more than BUCKET_MAX items: with big_bits > 0 their items are
// taken out in input order and sorted by a stable LSD radix sort of
// big_key(i) (big_bits bits), which must order them as (bucket, sub) does
// once equal keys keep their input order -- e.g. (bucket, hi) when sub is
// (hi, item index).  With big_bits == 0 such a bucket makes the sort return
// false.
struct NoBigKey {
    __device__ uint64_t operator()(int64_t) const { return 0; }
};
struct NoNote {
    __device__ void operator()(int64_t, int64_t) const {}
};

// Items handled at once by a thread in the sort's streaming passes: their
// loads are issued together, so a pass waits for one memory round trip per
// batch instead of one per item.
constexpr int SORT_BATCH = 4;

// bk_slot(i) must only load: its value carries the bucket in the low 32 bits
// (the high 32 bits are the caller's), and note(i, value) stores whatever the
// caller keeps of it once the batch's loads are done.
template <class Team, class BkSlot, class Bk, class Sub, class Pay, class BigKey = NoBigKey, class Note = NoNote>
__device__ bool team_bucket_sort_ex(const Team &t, Scratch &sc, char *sm, int64_t n, int32_t nb, BkSlot bk_slot,
                                    Bk bucket, Sub sub, Pay pay, uint64_t *keys_out, int32_t *idx_out,
                                    int32_t *bstart, int32_t *bucket_out = nullptr, int detail_phase = -1,
                                    BigKey big_key = BigKey(), int big_bits = 0, Note note = Note())
{
    uint64_t am = sc.arena.mark();
    int32_t *slot = sc.arena.take<int32_t>(n + 1);
    int32_t *tb = sc.arena.take<int32_t>(n + 1);    // bucket of the item at each scattered position
    int32_t *ti = sc.arena.take<int32_t>(n + 1);    // item index at each scattered position
    uint64_t *tk = sc.arena.take<uint64_t>(n + 1);  // sub key at each scattered position
    int32_t *lists = sc.arena.take<int32_t>(2 * ((int64_t)nb + 1));  // warp buckets, CTA buckets
    int32_t *nlist = sc.arena.take<int32_t>(4);
    if (!sc.arena.ok()) return false;
    int32_t *wlist = lists, *clist = lists + nb + 1;
    for (int64_t b = t.rank(); b <= nb; b += t.size()) bstart[b] = 0;
    if (t.rank() < 4) nlist[t.rank()] = 0;
    t.sync();
    // slots: the lanes of a warp that share a bucket take theirs with one
    // atomic; a warp handles SORT_BATCH strides at once (item k of a batch is
    // base + k * size + lane)
    {
        constexpr int U = SORT_BATCH;
        const int64_t S = t.size();
        for (int64_t base = (int64_t)t.rank() - lane_id(); base < n; base += S * U) {
            int64_t w[U];
#pragma unroll
            for (int k = 0; k < U; ++k) {
                const int64_t i = base + k * S + lane_id();
                w[k] = i < n ? (int64_t)bk_slot(i) : int64_t(-1);
            }
            int32_t s0[U];
            unsigned peers[U];
#pragma unroll
            for (int k = 0; k < U; ++k) {
                const int64_t i = base + k * S + lane_id();
                const int32_t b = i < n ? (int32_t)(uint32_t)w[k] : -1;
                peers[k] = __match_any_sync(FULL, b);
                s0[k] = 0;
                if (i < n && lane_id() == __ffs(peers[k]) - 1) s0[k] = atomicAdd(&bstart[b], __popc(peers[k]));
            }
#pragma unroll
            for (int k = 0; k < U; ++k) {
                const int64_t i = base + k * S + lane_id();
                const int32_t s = __shfl_sync(FULL, s0[k], __ffs(peers[k]) - 1);
                if (i < n) {
                    slot[i] = s + __popc(peers[k] & lanemask_lt());
                    note(i, w[k]);
                }
            }
        }
    }
    t.sync();
    if (detail_phase >= 0) prof_mark(t, sc, detail_phase);
    // bucket starts; buckets of more than 64 items go to the warp and CTA
    // lists (any order); one of more than BUCKET_MAX ends the sort
    team_scan<Team, int64_t>(
        t, sc, sm, nb, [&](int64_t b) -> int64_t { return bstart[b]; },
        [&](int64_t b, int64_t pre, int64_t c) {
            bstart[b] = (int32_t)pre;
            if (c > BUCKET_MAX)
                nlist[2] = 1;
            else if (c > 256)
                clist[atomicAdd(&nlist[1], 1)] = (int32_t)b;
            else if (c > 64)
                wlist[atomicAdd(&nlist[0], 1)] = (int32_t)b;
        });
    const bool has_big = uread(&nlist[2]) != 0;
    if (has_big && big_bits <= 0) {
        sc.arena.release(am);
        return false;
    }
    if (t.rank() == 0) bstart[nb] = (int32_t)n;
    t.sync();
    {
        // full batches of SORT_BATCH strides (loads first, then the
        // gathers of the bucket starts, then the stores), then one at a time
        constexpr int U = SORT_BATCH;
        const int64_t S = t.size();
        int64_t i0 = t.rank();
        for (; i0 + (U - 1) * S < n; i0 += U * S) {
            int32_t b[U], p[U], pv[U];
            uint64_t kv[U];
#pragma unroll
            for (int k = 0; k < U; ++k) {
                b[k] = (int32_t)bucket(i0 + k * S);
                p[k] = slot[i0 + k * S];
                kv[k] = sub(i0 + k * S);
                pv[k] = pay(i0 + k * S);
            }
#pragma unroll
            for (int k = 0; k < U; ++k) p[k] += bstart[b[k]];
#pragma unroll
            for (int k = 0; k < U; ++k) {
                tk[p[k]] = kv[k];
                ti[p[k]] = pv[k];
                tb[p[k]] = b[k];
            }
        }
        for (; i0 < n; i0 += S) {
            const int32_t b = (int32_t)bucket(i0);
            const int64_t p = (int64_t)bstart[b] + slot[i0];
            tk[p] = sub(i0);
            ti[p] = pay(i0);
            tb[p] = b;
        }
    }
    t.sync();
    if (detail_phase >= 0) prof_mark(t, sc, detail_phase + 1);
    // up to 64 items: each item's rank in its bucket is the number of smaller
    // keys there (neighbouring threads read the same bucket)
    {
        // the rank of item p in its bucket; -1: sorted below (a bucket of
        // 65..BUCKET_MAX items is copied as it is) or by the big path
        auto rank_in_bucket = [&](int64_t p, int32_t s, int32_t e, uint64_t key) -> int32_t {
            if (e - s > 64) return e - s <= BUCKET_MAX ? (int32_t)p : -1;
            int32_t r = 0;
            for (int32_t q = s; q < e; ++q) {
                const uint64_t o = tk[q];
                r += o < key || (o == key && q < p);
            }
            return s + r;
        };
        constexpr int U = SORT_BATCH;
        const int64_t S = t.size();
        int64_t p0 = t.rank();
        for (; p0 + (U - 1) * S < n; p0 += U * S) {
            int32_t b[U], s[U], e[U], iv[U], dst[U];
            uint64_t kv[U];
#pragma unroll
            for (int k = 0; k < U; ++k) {
                b[k] = tb[p0 + k * S];
                kv[k] = tk[p0 + k * S];
                iv[k] = ti[p0 + k * S];
            }
#pragma unroll
            for (int k = 0; k < U; ++k) {
                s[k] = bstart[b[k]];
                e[k] = bstart[b[k] + 1];
            }
#pragma unroll
            for (int k = 0; k < U; ++k) dst[k] = rank_in_bucket(p0 + k * S, s[k], e[k], kv[k]);
#pragma unroll
            for (int k = 0; k < U; ++k)
                if (dst[k] >= 0) {
                    keys_out[dst[k]] = kv[k];
                    idx_out[dst[k]] = iv[k];
                    if (bucket_out) bucket_out[dst[k]] = b[k];
                }
        }
        for (; p0 < n; p0 += S) {
            const int32_t b = tb[p0];
            const uint64_t key = tk[p0];
            const int32_t dst = rank_in_bucket(p0, bstart[b], bstart[b + 1], key);
            if (dst >= 0) {
                keys_out[dst] = key;
                idx_out[dst] = ti[p0];
                if (bucket_out) bucket_out[dst] = b;
            }
        }
    }
    t.sync();
    // 65..256 items: a warp, bitonic in its share of the staging area
    {
        const int NW = blockDim.x >> 5;
        const int w = warp_in_block();
        char *stage = sm + NW * 1024;
        uint64_t *wk = reinterpret_cast<uint64_t *>(stage) + w * 256;
        int32_t *wi = reinterpret_cast<int32_t *>(stage + NW * 256 * 8) + w * 256;
        const int32_t nw = uread(&nlist[0]);
        for (int64_t q = team_warp(t); q < nw; q += team_nwarps(t)) {
            const int32_t b = wlist[q], s = bstart[b], m = bstart[b + 1] - s;
            int P = 32;
            while (P < m) P <<= 1;
            for (int x = lane_id(); x < m; x += 32) {
                wk[x] = keys_out[s + x];
                wi[x] = idx_out[s + x];
            }
            __syncwarp();
            smem_bitonic(wk, wi, m, P, lane_id(), 32, [] { __syncwarp(); });
            for (int x = lane_id(); x < m; x += 32) {
                keys_out[s + x] = wk[x];
                idx_out[s + x] = wi[x];
            }
            __syncwarp();
        }
    }
    __syncthreads();
    // 257..BUCKET_MAX items: a CTA
    {
        const int NW = blockDim.x >> 5;
        char *stage = sm + NW * 1024;
        uint64_t *ck = reinterpret_cast<uint64_t *>(stage);
        int32_t *ci = reinterpret_cast<int32_t *>(stage + BUCKET_MAX * 8);
        const int32_t nc = uread(&nlist[1]);
        for (int64_t q = t.block(); q < nc; q += t.nblocks()) {
            const int32_t b = clist[q], s = bstart[b], m = bstart[b + 1] - s;
            int P = 512;
            while (P < m) P <<= 1;
            for (int x = threadIdx.x; x < m; x += blockDim.x) {
                ck[x] = keys_out[s + x];
                ci[x] = idx_out[s + x];
            }
            __syncthreads();
            smem_bitonic(ck, ci, m, P, threadIdx.x, blockDim.x, [] { __syncthreads(); });
            for (int x = threadIdx.x; x < m; x += blockDim.x) {
                keys_out[s + x] = ck[x];
                idx_out[s + x] = ci[x];
            }
            __syncthreads();
        }
    }
    t.sync();
    if (detail_phase >= 0) prof_mark(t, sc, detail_phase + 2);
    // (compiled only for callers that give a big key)
    if constexpr (!std::is_same<BigKey, NoBigKey>::value) if (has_big) {
        // the buckets beyond BUCKET_MAX: their items in input order, a stable
        // radix sort of big_key, then each into its bucket's range
        auto bsize = [&](int64_t i) {
            const int32_t b = (int32_t)bucket(i);
            return bstart[b + 1] - bstart[b];
        };
        uint64_t bm = sc.arena.mark();
        const int64_t nbig = team_sum<Team, int64_t>(t, sc, sm, n, [&](int64_t i) -> int64_t {
            return bsize(i) > BUCKET_MAX ? 1 : 0;
        });
        uint64_t *bk1 = sc.arena.take<uint64_t>(nbig + 1), *bk2 = sc.arena.take<uint64_t>(nbig + 1);
        int32_t *bv1 = sc.arena.take<int32_t>(nbig + 1), *bv2 = sc.arena.take<int32_t>(nbig + 1);
        int32_t *kfirst = sc.arena.take<int32_t>((int64_t)nb + 1);
        if (!sc.arena.ok()) return false;
        team_compact(
            t, sc, sm, n, [&](int64_t i) { return bsize(i) > BUCKET_MAX; },
            [&](int64_t i, int64_t k) {
                bk1[k] = big_key(i);
                bv1[k] = (int32_t)i;
            });
        team_sort_pairs(t, sc, sm, bk1, bv1, bk2, bv2, nbig, big_bits);
        for (int64_t k = t.rank(); k < nbig; k += t.size()) {
            const int32_t b = (int32_t)bucket(bv1[k]);
            if (k == 0 || (int32_t)bucket(bv1[k - 1]) != b) kfirst[b] = (int32_t)k;
        }
        t.sync();
        for (int64_t k = t.rank(); k < nbig; k += t.size()) {
            const int64_t i = bv1[k];
            const int32_t b = (int32_t)bucket(i);
            const int64_t p = (int64_t)bstart[b] + (k - kfirst[b]);
            keys_out[p] = sub(i);
            idx_out[p] = pay(i);
            if (bucket_out) bucket_out[p] = b;
        }
        t.sync();
        sc.arena.release(bm);
        if (detail_phase >= 0) prof_mark(t, sc, PH_CSORT_BIG);
    }
    sc.arena.release(am);
    return true;
}

template <class Team, class Bk, class Sub>
__device__ bool team_bucket_sort(const Team &t, Scratch &sc, char *sm, int64_t n, int32_t nb, Bk bucket, Sub sub,
                                 uint64_t *keys_out, int32_t *idx_out, int32_t *bstart)
{
    return team_bucket_sort_ex(
        t, sc, sm, n, nb, bucket, bucket, sub, [](int64_t i) { return (int32_t)i; }, keys_out, idx_out, bstart);
}

// ---------------------------------------------------------------------------
// off[v] = first k with ids(k) >= v, v in [0, nv]; ids sorted ascending
// ---------------------------------------------------------------------------
template <class Team, class Ids>
__device__ void team_offsets(const Team &t, int64_t n, int32_t nv, Ids ids, int32_t *off)
{
    for (int64_t k = t.rank(); k <= n; k += t.size()) {
        int32_t cur = k < n ? ids(k) : nv;
        int32_t prev = k == 0 ? -1 : ids(k - 1);
        for (int32_t v = prev + 1; v <= cur; ++v) off[v] = (int32_t)k;
    }
    t.sync();
}

// ---------------------------------------------------------------------------
// connected components: lab[v] = minimum vertex id of v's component.
// Edges are given as pairs (a(e), b(e)), e in [0,m).  Hook-and-compress with
// parent[x] <= x throughout (so chains strictly decrease and every loop ends);
// repeats until no edge joins two trees, at most 64 rounds.
// ---------------------------------------------------------------------------
template <class Team, class EA, class EB>
__device__ bool team_cc(const Team &t, Scratch &sc, int32_t nv, int64_t m, EA ea, EB eb, int32_t *lab)
{
    uint64_t am = sc.arena.mark();
    int32_t *flags = sc.arena.take<int32_t>(65);
    if (!sc.arena.ok()) return false;
    for (int64_t v = t.rank(); v < nv; v += t.size()) lab[v] = (int32_t)v;
    for (int k = t.rank(); k < 65; k += t.size()) flags[k] = 0;
    t.sync();
    bool converged = false;
    for (int it = 0; it < 64; ++it) {
        for (int64_t e = t.rank(); e < m; e += t.size()) {
            int32_t a = ea(e), b = eb(e);
            if (a == b) continue;
            int32_t ra = a, rb = b;
            for (int s = 0; s < 1 << 16; ++s) {
                int32_t p = ((volatile int32_t *)lab)[ra];
                if (p == ra) break;
                ra = p;
            }
            for (int s = 0; s < 1 << 16; ++s) {
                int32_t p = ((volatile int32_t *)lab)[rb];
                if (p == rb) break;
                rb = p;
            }
            if (ra != rb) {
                int32_t hi = ra > rb ? ra : rb, lo = ra > rb ? rb : ra;
                atomicMin(&lab[hi], lo);
                flags[it] = 1;
            }
        }
        t.sync();
        for (int64_t v = t.rank(); v < nv; v += t.size()) {
            int32_t x = lab[v];
            for (int s = 0; s < 1 << 16; ++s) {
                int32_t p = ((volatile int32_t *)lab)[x];
                if (p == x) break;
                x = p;
            }
            lab[v] = x;
        }
        t.sync();
        if (!uread(&flags[it])) {
            converged = true;
            break;
        }
    }
    sc.arena.release(am);
    return converged;
}

}  // namespace rama
