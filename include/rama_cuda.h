// rama_cuda.h -- the reference's C++ entry points (reference
// include/rama_cuda.h:8-9), implemented inline over the C ABI of
// librama_b200.so.  Failures throw std::runtime_error (bad contractions keep
// the reference's message "Found bad contractions"); an exhausted workspace
// throws std::bad_alloc.
#pragma once
#include <algorithm>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "multicut_solver_options.h"
#include "rama_b200.h"

namespace rama_detail {
inline void check(int rc)
{
    if (rc == RAMA_OK) return;
    if (rc == RAMA_ERR_OOM) throw std::bad_alloc();
    throw std::runtime_error(rama_last_error());
}

// one handle per thread and device, kept for the lifetime of the thread
inline rama_handle handle(int device)
{
    struct holder {
        std::vector<std::pair<int, rama_handle>> hs;
        ~holder()
        {
            for (auto &p : hs) rama_destroy(p.second);
        }
    };
    thread_local holder H;
    for (auto &p : H.hs)
        if (p.first == device) return p.second;
    rama_handle h = nullptr;
    check(rama_create(device, 0, &h));
    H.hs.push_back({device, h});
    return h;
}

inline std::vector<std::vector<int>> timeline(rama_handle h)
{
    int32_t rounds = 0;
    int64_t nl = 0;
    check(rama_get_timeline(h, nullptr, 0, &rounds, &nl));
    std::vector<int32_t> flat((size_t)rounds * (size_t)nl);
    check(rama_get_timeline(h, flat.data(), (int64_t)flat.size(), &rounds, &nl));
    std::vector<std::vector<int>> out((size_t)rounds);
    for (int32_t r = 0; r < rounds; ++r) out[r].assign(flat.begin() + (size_t)r * nl, flat.begin() + (size_t)(r + 1) * nl);
    return out;
}
}  // namespace rama_detail

// Host overload: returns (labels, lower bound, solve time in ms, timeline).
inline std::tuple<std::vector<int>, double, int, std::vector<std::vector<int>>> rama_cuda(
    const std::vector<int> &i, const std::vector<int> &j, const std::vector<float> &costs,
    const multicut_solver_options &opts)
{
    if (i.size() != j.size() || i.size() != costs.size()) throw std::runtime_error("Input shapes must match");
    rama_handle h = rama_detail::handle(0);
    int mx = -1;
    for (size_t e = 0; e < i.size(); ++e) mx = std::max(mx, std::max(i[e], j[e]));
    std::vector<int> labels((size_t)std::max(mx + 1, 1));
    int64_t nl = 0;
    double lb = 0, ms = 0;
    rama_options o = opts.to_c();
    rama_detail::check(rama_solve_host(h, i.data(), j.data(), costs.data(), (int64_t)costs.size(), &o, labels.data(),
                                       (int64_t)labels.size(), &nl, &lb, &ms));
    labels.resize((size_t)nl);
    std::vector<std::vector<int>> tl;
    if (opts.dump_timeline) tl = rama_detail::timeline(h);
    return {labels, lb, (int)ms, tl};
}

#if defined(__CUDACC__) || defined(RAMA_WITH_THRUST)
#include <thrust/device_vector.h>
#include <thrust/extrema.h>
// Device overload: consumes the inputs, returns (labels, lower bound, timeline).
inline std::tuple<thrust::device_vector<int>, double, std::vector<std::vector<int>>> rama_cuda(
    thrust::device_vector<int> &&i, thrust::device_vector<int> &&j, thrust::device_vector<float> &&costs,
    const multicut_solver_options &opts, const int device)
{
    rama_handle h = rama_detail::handle(device);
    if (i.size() != j.size() || i.size() != costs.size()) throw std::runtime_error("Input shapes must match");
    int mx = -1;
    if (!i.empty()) {
        mx = std::max(*thrust::max_element(i.begin(), i.end()), *thrust::max_element(j.begin(), j.end()));
    }
    thrust::device_vector<int> labels((size_t)std::max(mx + 1, 1));
    int64_t nl = 0;
    double lb = 0;
    rama_options o = opts.to_c();
    rama_detail::check(rama_solve(h, thrust::raw_pointer_cast(i.data()), thrust::raw_pointer_cast(j.data()),
                                  thrust::raw_pointer_cast(costs.data()), (int64_t)costs.size(), &o,
                                  thrust::raw_pointer_cast(labels.data()), (int64_t)labels.size(), &nl, &lb,
                                  nullptr));
    labels.resize((size_t)nl);
    thrust::device_vector<int>().swap(i);
    thrust::device_vector<int>().swap(j);
    thrust::device_vector<float>().swap(costs);
    std::vector<std::vector<int>> tl;
    if (opts.dump_timeline) tl = rama_detail::timeline(h);
    return {std::move(labels), lb, tl};
}
#endif
