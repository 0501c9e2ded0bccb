// Batched multi-graph x multi-attempt optimisation (rmx_batch_*).
//
// The reference optimises one network per process run, its #attempts
// (OmpRelaxmap.cpp:181-219, one stochastic_greedy_partition run per attempt)
// one after another. Here many graphs, each repeated once per attempt, are
// packed into waves; a wave is ONE disjoint-union graph on the device whose
// components (graph-attempt copies) are independent instances of the engine:
// every stop rule of the superstep loop is applied per instance, the flow is
// computed once per graph (one block per graph) and shared by its copies, and
// all instances advance in the same kernel launches. Copies of a graph differ
// in their random choices (sub-batch assignment and empty-module bids hash
// the unit id), as attempts with different seeds do. The best attempt of every
// graph (lowest code length, then lowest attempt index) is kept, its modules
// renumbered 0.. in order of first appearance.
#include <algorithm>
#include <cmath>
#include <memory>
#include <stdexcept>
#include <vector>

#include "rmx_batch.hpp"
#include "rmx_graph.hpp"
#include "rmx_io.hpp"

void rmx_batch::create(int32_t g, const int32_t *n_nodes, const int64_t *n_edges, const int32_t *s, const int32_t *d,
                       const double *wt, const double *node_weights) {
    if (g <= 0) throw std::invalid_argument("a batch needs at least one graph");
    if (!n_nodes || !n_edges) throw std::invalid_argument("n_nodes / n_edges missing");
    G = g;
    n.assign(n_nodes, n_nodes + g);
    noff.assign(g + 1, 0);
    eoff.assign(g + 1, 0);
    for (int32_t k = 0; k < g; k++) {
        if (n[k] <= 0) throw std::invalid_argument("every graph needs at least one node");
        if (n_edges[k] < 0) throw std::invalid_argument("negative edge count");
        noff[k + 1] = noff[k] + n[k];
        eoff[k + 1] = eoff[k] + n_edges[k];
    }
    const int64_t E = eoff[g];
    if (E > 0 && (!s || !d)) throw std::invalid_argument("edge arrays missing");
    for (int32_t k = 0; k < g; k++)
        for (int64_t e = eoff[k]; e < eoff[k + 1]; e++)
            if ((uint32_t)s[e] >= (uint32_t)n[k] || (uint32_t)d[e] >= (uint32_t)n[k])
                throw std::invalid_argument("edge endpoint outside 0..n-1 of its graph");
    src.assign(s, s + E);
    dst.assign(d, d + E);
    has_w = wt != nullptr;
    if (has_w) w.assign(wt, wt + E);
    has_nw = node_weights != nullptr;
    if (has_nw) nw.assign(node_weights, node_weights + noff[g]);
}

void rmx_batch::optimize(const rmx_opts &o, int32_t *part_out, double *L_out, int32_t *n_modules,
                         int32_t *best_attempt) {
    const int32_t A = std::max(1, o.attempts);
    rmx_opts one = o;
    one.attempts = 1;
    last_waves = 0;
    last_ms = 0.0;
    last_instances = 0;
    int32_t g0 = 0;
    while (g0 < G) {
        const rmx::NvtxRange range("rmx batch wave");
        // the next wave: whole graphs (all their attempts) up to the link budget
        int32_t g1 = g0;
        int64_t links = 0, nodes = 0;
        while (g1 < G) {
            const int64_t l = (eoff[g1 + 1] - eoff[g1]) * A, v = (int64_t)n[g1] * A;
            if (g1 > g0 && (links + l > wave_links || nodes + v > wave_nodes)) break;
            links += l;
            nodes += v;
            g1++;
        }
        if (nodes >= (int64_t(1) << 31) - 1 || links >= (int64_t(1) << 31) - 1)
            throw std::invalid_argument("one graph's attempts exceed 2^31-1 nodes or links");
        const int32_t K = (g1 - g0) * A;
        // the canonical copies' edges (nodes renumbered over the wave's graphs);
        // the device writes the other copies from them
        const int64_t ec = eoff[g1] - eoff[g0];
        const int64_t nc = noff[g1] - noff[g0];
        std::vector<int32_t> us(ec), ud(ec), node_inst(nodes), canon(K);
        std::vector<double> uw(has_w ? ec : 0), unw(has_nw ? nodes : 0);
        std::vector<int64_t> inoff(K + 1, 0);
        // graphs packed on host threads: graph g's canonical links fill
        // [eoff[g], eoff[g+1]) - eoff[g0], its copy a (instance (g-g0)*A + a)
        // the nodes from A * (noff[g] - noff[g0]) + a * n[g]
        const int T = (int)std::min<int64_t>(16, std::max<int64_t>(1, (ec + nodes) >> 21));
        rmx::run_parallel(T, [&](int t) {
            for (int32_t g = g0 + t; g < g1; g += T) {
                const int32_t cb = (int32_t)(noff[g] - noff[g0]);
                for (int64_t e = eoff[g]; e < eoff[g + 1]; e++) {
                    us[e - eoff[g0]] = src[e] + cb;
                    ud[e - eoff[g0]] = dst[e] + cb;
                }
                if (has_w) std::copy(w.begin() + eoff[g], w.begin() + eoff[g + 1], uw.begin() + (eoff[g] - eoff[g0]));
                const int32_t first = (g - g0) * A;
                for (int32_t a = 0; a < A; a++) {
                    const int32_t k = first + a;
                    const int64_t vb = (int64_t)A * cb + (int64_t)a * n[g];
                    canon[k] = first;
                    inoff[k] = vb;
                    std::fill(node_inst.begin() + vb, node_inst.begin() + vb + n[g], k);
                    if (has_nw) std::copy(nw.begin() + noff[g], nw.begin() + noff[g + 1], unw.begin() + vb);
                }
            }
        });
        inoff[K] = nodes;
        UnionSpec spec{K, node_inst.data(), inoff.data(), canon.data(), (int32_t)nc, links};
        std::unique_ptr<rmx_graph> U(new rmx_graph());
        U->create(us.data(), ud.data(), has_w ? uw.data() : nullptr, ec, (int32_t)nodes,
                  has_nw ? unw.data() : nullptr, &spec);
        const std::vector<double> L = U->run_union(one);
        std::vector<int32_t> part(nodes);
        RMX_CUDA(cudaMemcpyAsync(part.data(), U->nmod, sizeof(int32_t) * nodes, cudaMemcpyDeviceToHost, U->stream));
        RMX_CUDA(cudaStreamSynchronize(U->stream));
        last_ms += U->prof.total_ms;
        last_waves++;
        last_instances += K;
        // best attempt per graph, modules renumbered by first appearance
        std::vector<int32_t> label;
        int32_t k = 0;
        for (int32_t g = g0; g < g1; g++, k += A) {
            int32_t best = 0;
            for (int32_t a = 1; a < A; a++)
                if (L[k + a] < L[k + best]) best = a;
            if (L_out) L_out[g] = L[k + best];
            if (best_attempt) best_attempt[g] = best;
            const int64_t base = inoff[k + best];
            if (label.size() < (size_t)nodes) label.assign(nodes, -1);
            int32_t nm = 0;
            for (int32_t i = 0; i < n[g]; i++) {
                const int32_t m = part[base + i];
                if (label[m] < 0) label[m] = nm++;
                if (part_out) part_out[noff[g] + i] = label[m];
            }
            for (int32_t i = 0; i < n[g]; i++) label[part[base + i]] = -1;
            if (n_modules) n_modules[g] = nm;
        }
        g0 = g1;
    }
}
