// rama_text_input -- command-line solver with the reference's arguments and
// output (reference src/rama_text_input.cu:8-51, text format
// src/multicut_text_parser.cpp:6-31).
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <iterator>
#include <numeric>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "multicut_solver_options.h"
#include "rama_cuda.h"

// MULTICUT text: a first line "MULTICUT", then "i j cost" triples until the
// first token that does not parse.  The bytes are read on the host and parsed
// on the GPU (rama_parse_multicut_host).
static std::tuple<std::vector<int>, std::vector<int>, std::vector<float>> read_file(const std::string &filename)
{
    std::FILE *f = std::fopen(filename.c_str(), "rb");
    if (!f) throw std::runtime_error("Could not open multicut input file " + filename);
    std::string buf;
    {
        char tmp[1 << 16];
        size_t k;
        while ((k = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.append(tmp, k);
        std::fclose(f);
    }
    const int64_t len = (int64_t)buf.size();
    const int64_t cap = (len + 1) / 6 + 1;
    std::vector<int> iv((size_t)cap), jv((size_t)cap);
    std::vector<float> cv((size_t)cap);
    rama_handle h = nullptr;
    if (rama_create(0, 0, &h) != RAMA_OK) throw std::runtime_error(rama_last_error());
    int64_t n = 0;
    const int rc = rama_parse_multicut_host(h, buf.data(), len, iv.data(), jv.data(), cv.data(), cap, &n);
    const std::string msg = rc ? rama_last_error() : "";
    rama_destroy(h);
    if (rc) throw std::runtime_error(msg);
    iv.resize((size_t)n);
    jv.resize((size_t)n);
    cv.resize((size_t)n);
    return {iv, jv, cv};
}

int main(int argc, char **argv)
{
    multicut_solver_options opts;
    int e = opts.from_cl(argc, argv);
    if (e != -1) return e;
    std::vector<int> i, j;
    std::vector<float> costs;
    std::tie(i, j, costs) = read_file(opts.input_file);
    std::vector<int> h_node_mapping;
    double lb;
    int dur;
    std::vector<std::vector<int>> timeline;
    std::tie(h_node_mapping, lb, dur, timeline) = rama_cuda(i, j, costs, opts);
    double obj = 0;
    if (!opts.only_compute_lb) {
        for (size_t k = 0; k < costs.size(); ++k)
            if (h_node_mapping[i[k]] != h_node_mapping[j[k]]) obj += costs[k];
        std::cout << "\tcost w.r.t original objective: " << obj << "\n";
    }
    std::cout << "\tfinal lower bound: " << lb << "\n";
    std::cout << "\tGPU compute time: " << dur << "ms\n";
    if (opts.output_sol_file != "") {
        std::ofstream sol_file;
        sol_file.open(opts.output_sol_file);
        std::cout << "Writing solution to file: " << opts.output_sol_file << "\n";
        if (!h_node_mapping.empty()) {
            const int num_clusters = *std::max_element(h_node_mapping.begin(), h_node_mapping.end()) + 1;
            std::vector<std::vector<int>> members((size_t)std::max(num_clusters, 0));
            for (size_t v = 0; v < h_node_mapping.size(); ++v)
                if (h_node_mapping[v] >= 0) members[(size_t)h_node_mapping[v]].push_back((int)v);
            for (int c = 0; c != num_clusters; ++c) {
                std::copy(members[c].begin(), members[c].end(), std::ostream_iterator<int>(sol_file, "\t"));
                sol_file << "\n";
            }
        }
        sol_file.close();
    }
    return 0;
}
