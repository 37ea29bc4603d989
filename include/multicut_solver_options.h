// multicut_solver_options.h -- solver options with the reference's fields,
// presets and command line (reference include/multicut_solver_options.h:4-127).
// The command line is parsed here directly; the reference uses CLI11.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "rama_b200.h"

struct multicut_solver_options {
    std::string input_file;
    std::string output_sol_file = "";
    int max_cycle_length_lb = 5;
    int num_dual_itr_lb = 10;
    int max_cycle_length_primal = 3;
    int num_dual_itr_primal = 5;
    int num_outer_itr_dual = 1;
    float mean_multiplier_mm = 0.05;
    float matching_thresh_crossover_ratio = 0.05;
    float tri_memory_factor = 2.0;
    bool only_compute_lb = false;
    int max_time_sec = -1;
    bool dump_timeline = false;
    bool verbose = true;
    bool sanitize_graph = false;
    // not in the reference: also cut conflicted 5-cycles in the forest
    // contraction (its check_pentagons_cuda, shipped disabled there)
    bool woc_pentagons = false;

    multicut_solver_options() {}
    multicut_solver_options(const std::string &solver_type)
    {
        if (solver_type == "PD") {
            std::cout << "Running solver type PD which offers best compute time versus quality tradeoff." << std::endl;
        } else if (solver_type == "P") {
            std::cout << "Running purely primal solver (better runtime, worse quality)" << std::endl;
            max_cycle_length_lb = 0;
            num_dual_itr_lb = 0;
            max_cycle_length_primal = 0;
            num_dual_itr_primal = 0;
        } else if (solver_type == "PD+") {
            std::cout << "Running PD+ solver (worse runtime, better quality)" << std::endl;
            max_cycle_length_lb = 5;
            num_dual_itr_lb = 10;
            max_cycle_length_primal = 5;
            num_dual_itr_primal = 10;
        } else if (solver_type == "D") {
            std::cout << "Running dual solver to compute only the lower bound." << std::endl;
            max_cycle_length_lb = 5;
            num_dual_itr_lb = 10;
            num_outer_itr_dual = 5;
            only_compute_lb = true;
        }
        // an unknown type keeps the defaults (the reference constructs, but
        // does not throw, its runtime_error)
    }

    multicut_solver_options(const int _max_cycle_length_lb, const int _num_dual_itr_lb,
                            const int _max_cycle_length_primal, const int _num_dual_itr_primal,
                            const int _num_outer_itr_dual, const float _mean_multiplier_mm,
                            const float _matching_thresh_crossover_ratio, const float _tri_memory_factor,
                            const bool _only_compute_lb, const int _max_time_sec, const bool _dump_timeline = false,
                            const bool _sanitize_graph = false)
        : max_cycle_length_lb(_max_cycle_length_lb), num_dual_itr_lb(_num_dual_itr_lb),
          max_cycle_length_primal(_max_cycle_length_primal), num_dual_itr_primal(_num_dual_itr_primal),
          num_outer_itr_dual(_num_outer_itr_dual), mean_multiplier_mm(_mean_multiplier_mm),
          matching_thresh_crossover_ratio(_matching_thresh_crossover_ratio), tri_memory_factor(_tri_memory_factor),
          only_compute_lb(_only_compute_lb), max_time_sec(_max_time_sec), dump_timeline(_dump_timeline),
          sanitize_graph(_sanitize_graph)
    {
    }

    rama_options to_c(int team = 0) const
    {
        rama_options o;
        rama_options_init(&o, nullptr);
        o.max_cycle_length_lb = max_cycle_length_lb;
        o.num_dual_itr_lb = num_dual_itr_lb;
        o.max_cycle_length_primal = max_cycle_length_primal;
        o.num_dual_itr_primal = num_dual_itr_primal;
        o.num_outer_itr_dual = num_outer_itr_dual;
        o.mean_multiplier_mm = mean_multiplier_mm;
        o.matching_thresh_crossover_ratio = matching_thresh_crossover_ratio;
        o.tri_memory_factor = tri_memory_factor;
        o.only_compute_lb = only_compute_lb;
        o.max_time_sec = max_time_sec;
        o.dump_timeline = dump_timeline;
        o.verbose = verbose;
        o.sanitize_graph = sanitize_graph;
        o.team = team;
        o.woc_pentagons = woc_pentagons;
        return o;
    }

    // Command line of the reference (:82-105): -f/--file or the first
    // positional, -o/--out_sol_file, positional numeric options, three flags.
    // Returns -1 on success, otherwise the process exit code.
    int from_cl(int argc, char **argv)
    {
        std::vector<std::string> pos;
        bool have_file = false;
        for (int k = 1; k < argc; ++k) {
            std::string a = argv[k];
            if (a == "-h" || a == "--help") {
                std::cout << usage(argv[0]);
                return 0;
            } else if (a == "-f" || a == "--file") {
                if (k + 1 >= argc) return err("-f requires an argument");
                input_file = argv[++k];
                have_file = true;
            } else if (a == "-o" || a == "--out_sol_file") {
                if (k + 1 >= argc) return err("-o requires an argument");
                output_sol_file = argv[++k];
            } else if (a == "--only_lb")
                only_compute_lb = true;
            else if (a == "--dump_timeline")
                dump_timeline = true;
            else if (a == "--sanitize_graph")
                sanitize_graph = true;
            else if (a == "--woc_pentagons")
                woc_pentagons = true;
            else if (a.size() > 1 && a[0] == '-' && !(a[1] >= '0' && a[1] <= '9') && a[1] != '.')
                return err("The following argument was not expected: " + a);
            else
                pos.push_back(a);
        }
        size_t p = 0;
        if (!have_file) {
            if (pos.empty()) return err("--file is required");
            input_file = pos[p++];
        }
        struct stat sb;
        if (stat(input_file.c_str(), &sb) != 0) return err("--file: Path does not exist: " + input_file);
        try {
            if (p < pos.size()) max_cycle_length_lb = range_int(pos[p++], 0, 5, "max_cycle_dual");
            if (p < pos.size()) num_dual_itr_lb = nonneg_int(pos[p++], "dual_itr");
            if (p < pos.size()) max_cycle_length_primal = range_int(pos[p++], 0, 5, "max_cycle_primal");
            if (p < pos.size()) num_dual_itr_primal = nonneg_int(pos[p++], "dual_itr_primal");
            if (p < pos.size()) num_outer_itr_dual = nonneg_int(pos[p++], "dual_itr_outer");
            if (p < pos.size()) mean_multiplier_mm = nonneg_float(pos[p++], "mean_multiplier_mm");
            if (p < pos.size()) matching_thresh_crossover_ratio = nonneg_float(pos[p++], "matching_thresh_crossover_ratio");
            if (p < pos.size()) {
                tri_memory_factor = nonneg_float(pos[p++], "tri_memory_factor");
                if (!(tri_memory_factor > 0)) throw std::runtime_error("tri_memory_factor: Value must be positive");
            }
            if (p < pos.size()) throw std::runtime_error("The following argument was not expected: " + pos[p]);
        } catch (const std::exception &e) {
            return err(e.what());
        }
        return -1;
    }

    std::string get_string() const
    {
        return std::string("<multicut_solver_options>:") + "max_cycle_length_lb: " +
               std::to_string(max_cycle_length_lb) + ", num_dual_itr_lb: " + std::to_string(num_dual_itr_lb) +
               ", num_dual_itr_primal: " + std::to_string(num_dual_itr_primal) +
               ", max_cycle_length_primal: " + std::to_string(max_cycle_length_primal) +
               ", num_outer_itr_dual: " + std::to_string(num_outer_itr_dual) +
               ", mean_multiplier_mm: " + std::to_string(mean_multiplier_mm) +
               ", matching_thresh_crossover_ratio: " + std::to_string(matching_thresh_crossover_ratio) +
               ", tri_memory_factor: " + std::to_string(tri_memory_factor) +
               ", only_compute_lb: " + std::to_string(only_compute_lb) +
               ", max_time_sec: " + std::to_string(max_time_sec) +
               ", sanitize_graph: " + std::to_string(sanitize_graph) + ", verbose: " + std::to_string(verbose) + "\n";
    }

    void print() const { std::cout << this->get_string(); }

  private:
    static int err(const std::string &m)
    {
        std::cerr << m << "\nRun with --help for more information.\n";
        return 106;
    }
    static std::string usage(const char *prog)
    {
        return std::string("Solver for multicut problem. \nUsage: ") + prog +
               " [OPTIONS] file_pos [max_cycle_dual] [dual_itr] [max_cycle_primal] [dual_itr_primal] "
               "[dual_itr_outer] [mean_multiplier_mm] [matching_thresh_crossover_ratio] [tri_memory_factor]\n"
               "  -f,--file FILE           Path to multicut instance (.txt)\n"
               "  -o,--out_sol_file FILE   Path to save node labeling (.txt)\n"
               "  --only_lb                Only compute the lower bound.\n"
               "  --dump_timeline          Return the output of each contraction step.\n"
               "  --sanitize_graph         Relabel nodes without edges; their label is -1.\n"
               "  --woc_pentagons          Also cut conflicted 5-cycles in forest contractions.\n";
    }
    static int range_int(const std::string &s, int lo, int hi, const char *name)
    {
        size_t k = 0;
        int v = std::stoi(s, &k);
        if (k != s.size() || v < lo || v > hi)
            throw std::runtime_error(std::string(name) + ": Value " + s + " not in range " + std::to_string(lo) +
                                     " to " + std::to_string(hi));
        return v;
    }
    static int nonneg_int(const std::string &s, const char *name)
    {
        size_t k = 0;
        int v = std::stoi(s, &k);
        if (k != s.size() || v < 0) throw std::runtime_error(std::string(name) + ": Value must be non-negative");
        return v;
    }
    static float nonneg_float(const std::string &s, const char *name)
    {
        size_t k = 0;
        float v = std::stof(s, &k);
        if (k != s.size() || v < 0) throw std::runtime_error(std::string(name) + ": Value must be non-negative");
        return v;
    }
};
