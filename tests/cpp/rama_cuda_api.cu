// rama_cuda_api.cu -- drives the reference-shaped C++ entry points of
// include/rama_cuda.h (the reference's include/rama_cuda.h:8-9) the way a
// caller of the reference would, compiled with nvcc so that the
// thrust::device_vector overload is built too.
//
//   rama_cuda_api thrust : a small grid solved through the host overload and
//                          through the device overload (which consumes its
//                          inputs); labels and bound must agree.
//   rama_cuda_api bad    : an input whose contraction yields a negative
//                          cluster cost; the host overload must throw
//                          std::runtime_error("Found bad contractions")
//                          (reference src/rama_cuda.cu:136-137).
// Prints "ok" and exits 0 on success.
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <utility>
#include <vector>

#include "rama_cuda.h"

namespace {

// 20x20 4-connected grid with costs from a fixed linear congruential sequence
void grid(std::vector<int> &i, std::vector<int> &j, std::vector<float> &c)
{
    const int W = 20;
    uint32_t s = 12345u;
    auto next = [&]() {
        s = s * 1664525u + 1013904223u;
        return (float)((s >> 8) & 0xffff) / 65535.0f * 4.0f - 1.5f;
    };
    for (int y = 0; y < W; ++y)
        for (int x = 0; x < W; ++x) {
            const int v = y * W + x;
            if (x + 1 < W) {
                i.push_back(v);
                j.push_back(v + 1);
                c.push_back(next());
            }
            if (y + 1 < W) {
                i.push_back(v);
                j.push_back(v + W);
                c.push_back(next());
            }
        }
}

int run_thrust()
{
    std::vector<int> i, j;
    std::vector<float> c;
    grid(i, j, c);
    multicut_solver_options opts("PD");
    opts.verbose = false;
    auto host = rama_cuda(i, j, c, opts);
    thrust::device_vector<int> di(i.begin(), i.end()), dj(j.begin(), j.end());
    thrust::device_vector<float> dc(c.begin(), c.end());
    auto dev = rama_cuda(std::move(di), std::move(dj), std::move(dc), opts, 0);
    const std::vector<int> &hl = std::get<0>(host);
    std::vector<int> dl(std::get<0>(dev).size());
    thrust::copy(std::get<0>(dev).begin(), std::get<0>(dev).end(), dl.begin());
    if (hl != dl) {
        std::printf("labels differ between the host and device overloads\n");
        return 1;
    }
    if (std::get<1>(host) != std::get<1>(dev)) {
        std::printf("bounds differ: %.17g vs %.17g\n", std::get<1>(host), std::get<1>(dev));
        return 1;
    }
    if (!di.empty() || !dj.empty() || !dc.empty()) {
        std::printf("the device overload did not consume its inputs\n");
        return 1;
    }
    std::printf("ok %zu labels, lb %.6f\n", hl.size(), std::get<1>(host));
    return 0;
}

int run_bad()
{
    // two parallel edges 0-1 (+5 and -10): matching joins 0 and 1 along the
    // +5 edge, and their cluster's internal cost is then -5
    std::vector<int> i = {0, 0, 1}, j = {1, 1, 2};
    std::vector<float> c = {5.0f, -10.0f, 1.0f};
    multicut_solver_options opts("P");
    opts.verbose = false;
    try {
        rama_cuda(i, j, c, opts);
    } catch (const std::runtime_error &e) {
        if (std::strcmp(e.what(), "Found bad contractions") == 0) {
            std::printf("ok\n");
            return 0;
        }
        std::printf("runtime_error with another message: %s\n", e.what());
        return 1;
    }
    std::printf("no exception\n");
    return 1;
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc > 1 && !std::strcmp(argv[1], "thrust")) return run_thrust();
    if (argc > 1 && !std::strcmp(argv[1], "bad")) return run_bad();
    std::printf("usage: rama_cuda_api thrust|bad\n");
    return 2;
}
