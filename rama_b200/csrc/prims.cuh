// prims.cuh -- team-generic parallel primitives (scan, canonical sums,
// stable compaction, LSD radix sort, CSR offsets, connected components).
//
// All results are independent of the team size: order-sensitive primitives
// split the input into one contiguous chunk per CTA, and the floating-point
// sums follow fixed reduction trees (CSUM, RSUM) that are defined by element
// index only.
#pragma once
#include <cstdint>

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
    int parity;
    double alg_bytes;  // algorithmic bytes of the work done (team-uniform tally)
    int64_t *prof;     // optional per-phase nanoseconds (leader only)
    uint64_t tlast;
    __device__ __forceinline__ char *next_part()
    {
        parity ^= 1;
        return part[parity];
    }
};

// Phase timing: the team leader charges the time since the last mark to
// `phase`.  Marks sit right after team syncs, so a phase's time is the span
// in which the whole team worked on it.
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
    PH_COUNT = 10
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
        sc.tlast = now;
    }
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

template <class Team, class T, class Get>
__device__ T team_sum(const Team &t, Scratch &sc, char *sm, int64_t n, Get get)
{
    T s = T(0);
    for (int64_t i = t.rank(); i < n; i += t.size()) s += get(i);
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
    for (int64_t i = t.rank(); i < n; i += t.size()) {
        T x = get(i);
        s = x > s ? x : s;
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

// ---------------------------------------------------------------------------
// team exclusive scan: out(i, prefix, value) is called for every i in [0,n)
// in chunk order; returns the total.  Two team syncs; outputs are visible to
// the whole team on return.
// ---------------------------------------------------------------------------
template <class Team, class T, class In, class Out>
__device__ T team_scan(const Team &t, Scratch &sc, char *sm, int64_t n, In in, Out out)
{
    T *tsm = reinterpret_cast<T *>(sm);
    int64_t lo, hi;
    block_chunk(t, n, lo, hi);
    T s = T(0);
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) s += in(i);
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
    for (int64_t tile = lo; tile < hi; tile += blockDim.x) {
        int64_t i = tile + threadIdx.x;
        T v = i < hi ? in(i) : T(0);
        T ts;
        T ex = block_excl_scan<T>(v, tsm, ts);
        if (i < hi) out(i, base + ex, v);
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

// returns the sum on every thread; three team syncs
template <class Team, class Get>
__device__ double team_csum(const Team &t, Scratch &sc, int64_t n, Get get)
{
    const int64_t nch = (n + 4095) / 4096;
    uint64_t m = sc.arena.mark();
    csum_t *parts = sc.arena.take<csum_t>(nch + 1);
    double *res = reinterpret_cast<double *>(sc.next_part());
    if (sc.arena.ok()) {
        const int64_t w = team_warp(t), nw = team_nwarps(t);
        for (int64_t ch = w; ch < nch; ch += nw) {
            csum_t a = {0.0, 0.0};
            const int64_t b0 = ch * 4096 + lane_id();
            for (int k = 0; k < 128; ++k) {
                int64_t idx = b0 + 32 * k;
                if (idx < n) a = cs_merge(a, csum_t{get(idx), 0.0});
            }
            a = cs_warp_tree(a);
            if (lane_id() == 0) parts[ch] = a;
        }
    }
    t.sync();
    if (sc.arena.ok() && t.block() == 0 && warp_in_block() == 0) {
        csum_t a = {0.0, 0.0};
        for (int64_t k = lane_id(); k < nch; k += 32) a = cs_merge(a, parts[k]);
        a = cs_warp_tree(a);
        if (lane_id() == 0) res[0] = __dadd_rn(a.s, a.c);
    }
    t.sync();
    double r = uread(&res[0]);
    sc.arena.release(m);
    t.sync();  // `res` may be reused by the next primitive only after everyone read it
    return r;
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

// the same sum by a whole warp (any n); result valid on every lane
template <class Get>
__device__ __forceinline__ float rsum_warp(int64_t n, Get v)
{
    double a = 0.0;
    for (int64_t k = lane_id(); k < n; k += 32) a = __dadd_rn(a, (double)v(k));
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        double o = __shfl_down_sync(FULL, a, off);
        if ((lane_id() & (2 * off - 1)) == 0) a = __dadd_rn(a, o);
    }
    return (float)__shfl_sync(FULL, a, 0);
}

// ---------------------------------------------------------------------------
// LSD radix sort of (uint64 key, V value) pairs, 8-bit digits, stable.
// The sorted data ends in (*keys, *vals) (pointers may be swapped with the
// spare buffers).  Per pass: each CTA counts the digits of its contiguous
// chunk into a digit-major table (digit, CTA); an exclusive team scan of that
// table gives every (digit, CTA) its first output position; each CTA then
// scatters its chunk tile by tile, ranking keys stably within a warp by
// match_any.  Four team syncs per pass.
// ---------------------------------------------------------------------------
constexpr int SORT_ITEMS = 4;

template <class Team, class V>
__device__ void team_sort_pairs(const Team &t, Scratch &sc, char *sm, uint64_t *&keys, V *&vals, uint64_t *&keys2,
                                V *&vals2, int64_t n, int bits)
{
    if (n <= 1 || bits <= 0) return;
    const int nb = t.nblocks();
    const int NW = blockDim.x >> 5;
    uint64_t am = sc.arena.mark();
    uint32_t *ghist = sc.arena.take<uint32_t>((uint64_t)nb * 256);
    int64_t *gpos = sc.arena.take<int64_t>((uint64_t)nb * 256);
    if (!sc.arena.ok()) return;
    uint32_t *wcnt = reinterpret_cast<uint32_t *>(sm);              // NW * 256
    int64_t *pos = reinterpret_cast<int64_t *>(sm + NW * 256 * 4);  // 256
    uint32_t *tcnt = reinterpret_cast<uint32_t *>(sm + NW * 256 * 4 + 256 * 8);
    int64_t lo, hi;
    block_chunk(t, n, lo, hi);
    const int w = warp_in_block();
    for (int shift = 0; shift < bits; shift += 8) {
        // 1. per-CTA digit histogram
        for (int d = threadIdx.x; d < 256; d += blockDim.x) tcnt[d] = 0;
        __syncthreads();
        for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) atomicAdd(&tcnt[(keys[i] >> shift) & 255], 1u);
        __syncthreads();
        for (int d = threadIdx.x; d < 256; d += blockDim.x) ghist[(int64_t)d * nb + t.block()] = tcnt[d];
        t.sync();
        // 2. first output position of every (digit, CTA)
        team_scan<Team, int64_t>(
            t, sc, sm, (int64_t)nb * 256, [&](int64_t i) -> int64_t { return __ldcg(ghist + i); },
            [&](int64_t i, int64_t pre, int64_t) { gpos[i] = pre; });
        for (int d = threadIdx.x; d < 256; d += blockDim.x) pos[d] = __ldcg(gpos + (int64_t)d * nb + t.block());
        __syncthreads();
        // 3. stable scatter, one tile of blockDim*SORT_ITEMS keys at a time
        const int64_t TILE = (int64_t)blockDim.x * SORT_ITEMS;
        for (int64_t tile = lo; tile < hi; tile += TILE) {
            for (int d = lane_id(); d < 256; d += 32) wcnt[w * 256 + d] = 0;
            __syncwarp();
            const int64_t sub = tile + (int64_t)w * 32 * SORT_ITEMS;
            uint64_t mk[SORT_ITEMS];
            V mv[SORT_ITEMS];
            int md[SORT_ITEMS];
            uint32_t mr[SORT_ITEMS];
#pragma unroll
            for (int k = 0; k < SORT_ITEMS; ++k) {
                int64_t idx = sub + k * 32 + lane_id();
                bool valid = idx < hi;
                uint64_t key = valid ? keys[idx] : 0;
                int d = valid ? int((key >> shift) & 255) : 256;
                unsigned peers = __match_any_sync(FULL, d);
                int leader = __ffs(peers) - 1;
                uint32_t b0 = 0;
                if (valid && lane_id() == leader) {
                    b0 = wcnt[w * 256 + d];
                    wcnt[w * 256 + d] = b0 + __popc(peers);
                }
                b0 = __shfl_sync(FULL, b0, leader);
                __syncwarp();
                mk[k] = key;
                mv[k] = valid ? vals[idx] : V();
                md[k] = d;
                mr[k] = b0 + __popc(peers & lanemask_lt());
            }
            __syncthreads();
            for (int d = threadIdx.x; d < 256; d += blockDim.x) {
                uint32_t s = 0;
                for (int q = 0; q < NW; ++q) {
                    uint32_t c = wcnt[q * 256 + d];
                    wcnt[q * 256 + d] = s;
                    s += c;
                }
                tcnt[d] = s;
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < SORT_ITEMS; ++k) {
                if (md[k] < 256) {
                    int64_t p = pos[md[k]] + wcnt[w * 256 + md[k]] + mr[k];
                    keys2[p] = mk[k];
                    vals2[p] = mv[k];
                }
            }
            __syncthreads();
            for (int d = threadIdx.x; d < 256; d += blockDim.x) pos[d] += tcnt[d];
            __syncthreads();
        }
        t.sync();
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
    return (threads / 32) * 256 * 4 + 256 * 8 + 256 * 4 + 34 * 8;
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
