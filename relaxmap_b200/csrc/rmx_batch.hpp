// The opaque handle behind rmx_batch_*: the graphs of a batch held in host
// memory until they are packed into device waves by rmx_batch_optimize.
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/relaxmap_b200.h"

struct rmx_batch {
    int32_t G = 0;
    std::vector<int32_t> n;          // nodes per graph
    std::vector<int64_t> noff, eoff;  // node and edge offsets of the graphs, G + 1
    std::vector<int32_t> src, dst;   // graph-local node ids
    std::vector<double> w, nw;
    bool has_w = false, has_nw = false;
    // wave budget: link and node copies held on the device at once
    int64_t wave_links = int64_t(1) << 27, wave_nodes = int64_t(1) << 25;
    // last rmx_batch_optimize
    int32_t last_waves = 0;
    int64_t last_instances = 0;
    double last_ms = 0.0;

    void create(int32_t g, const int32_t *n_nodes, const int64_t *n_edges, const int32_t *src, const int32_t *dst,
                const double *w, const double *node_w);
    void optimize(const rmx_opts &o, int32_t *part_out, double *L_out, int32_t *n_modules, int32_t *best_attempt);
};
