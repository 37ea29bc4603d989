// k_misc.cu -- the small kernels around a solve: the MULTICUT text parser on
// the cooperative grid, the compensated objective and the maximum node id of
// an edge list (rama_solve_host sizes its label buffer with it).
#include "kernels.cuh"
#include "parse.cuh"

using namespace rama;

__global__ void __launch_bounds__(THREADS, 2) k_parse_grid(ParseLaunch L)
{
    extern __shared__ __align__(16) char sm[];
    GridTeam t;
    Scratch sc = make_scratch(L.ws, L.ws_bytes);
    if (t.rank() == 0) *sc.err = 0;
    t.sync();
    const int64_t n = parse_multicut(t, sc, sm, L.text, L.len, L.i, L.j, L.c, L.cap);
    if (t.leader()) L.out[0] = sc.arena.ok() ? n : -2;
}

// objective: CSUM over edges whose endpoints carry different labels
__global__ void __launch_bounds__(THREADS, 2) k_objective(const int32_t *I, const int32_t *J, const float *C, int64_t n,
                                                          const int32_t *lab, double *out, char *ws, uint64_t bytes)
{
    extern __shared__ __align__(16) char sm[];
    GridTeam t;
    Scratch sc = make_scratch(ws, bytes);
    double s = team_csum(t, sc, n, [&](int64_t e) -> float { return lab[I[e]] != lab[J[e]] ? C[e] : 0.0f; });
    if (t.leader()) *out = s;
}

// Maximum id over i and j (out[0], which the caller sets to -1 first) and
// whether any id is negative (out[1], set to 0 first).  128-bit loads where
// the arrays are 16-byte aligned; a grid-stride loop of int4 words with the
// tail read one by one.
__global__ void __launch_bounds__(256) k_max_id(MaxIdLaunch L)
{
    int32_t mx = -1;
    int neg = 0;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nth = (int64_t)gridDim.x * blockDim.x;
    const bool vec = ((reinterpret_cast<uintptr_t>(L.i) | reinterpret_cast<uintptr_t>(L.j)) & 15) == 0;
    int64_t done = 0;
    if (vec) {
        const int64_t nv = L.n / 4;
        const int4 *I4 = reinterpret_cast<const int4 *>(L.i);
        const int4 *J4 = reinterpret_cast<const int4 *>(L.j);
        for (int64_t k = tid; k < nv; k += nth) {
            const int4 a = __ldcs(I4 + k), b = __ldcs(J4 + k);
            mx = max(mx, max(max(a.x, a.y), max(a.z, a.w)));
            mx = max(mx, max(max(b.x, b.y), max(b.z, b.w)));
            neg |= (a.x | a.y | a.z | a.w | b.x | b.y | b.z | b.w) < 0;
        }
        done = nv * 4;
    }
    for (int64_t e = done + tid; e < L.n; e += nth) {
        const int32_t a = L.i[e], b = L.j[e];
        mx = max(mx, max(a, b));
        neg |= (a | b) < 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = max(mx, __shfl_xor_sync(FULL, mx, o));
        neg |= __shfl_xor_sync(FULL, neg, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (mx >= 0) atomicMax(&L.out[0], mx);
        if (neg) atomicOr(&L.out[1], 1);
    }
}
