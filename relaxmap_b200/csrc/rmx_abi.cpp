// extern "C" boundary: every entry point converts exceptions into rmx_status
// and records a thread-local message (no C++ exception crosses the ABI).
#include <sys/stat.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <utility>

#include "rmx_batch.hpp"
#include "rmx_graph.hpp"
#include "rmx_io.hpp"

namespace {

thread_local std::string g_last_error;

// The parse a size query of rmx_parse_file (all buffers NULL) made, kept for
// the next call on this thread when it names the same path and thread count
// and the file is unchanged (device, inode, size, modification time).
struct ParseCache {
    bool valid = false;
    std::string path;
    int32_t threads = 0;
    struct stat st {};
    rmx::ParsedGraph pg;
};
thread_local ParseCache g_parse_cache;

bool same_file(const struct stat &a, const struct stat &b) {
    return a.st_dev == b.st_dev && a.st_ino == b.st_ino && a.st_size == b.st_size &&
           a.st_mtim.tv_sec == b.st_mtim.tv_sec && a.st_mtim.tv_nsec == b.st_mtim.tv_nsec;
}

rmx_status fail(rmx_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}

template <typename F>
rmx_status guard(F &&f) {
    try {
        f();
        return RMX_OK;
    } catch (const rmx::CudaError &e) {
        return fail(e.code == cudaErrorMemoryAllocation ? RMX_ERR_OOM : RMX_ERR_CUDA, e.what());
    } catch (const rmx::NoConvergence &e) {
        return fail(RMX_ERR_NO_CONVERGENCE, e.what());
    } catch (const rmx::FormatError &e) {
        return fail(RMX_ERR_FORMAT, e.what());
    } catch (const rmx::IoError &e) {
        return fail(RMX_ERR_IO, e.what());
    } catch (const std::invalid_argument &e) {
        return fail(RMX_ERR_INVALID, e.what());
    } catch (const std::bad_alloc &) {
        return fail(RMX_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(RMX_ERR_CUDA, e.what());
    }
}

void need(const void *p, const char *what) {
    if (!p) throw std::invalid_argument(std::string(what) + " is NULL");
}

}  // namespace

extern "C" {

const char *rmx_last_error(void) { return g_last_error.c_str(); }

const char *rmx_version(void) { return "relaxmap_b200 0.1 (sm_100a)"; }

void rmx_opts_default(rmx_opts *o) {
    if (!o) return;
    o->seed = 1;
    o->threads = 1;
    o->attempts = 1;
    o->threshold = 1e-3;
    o->vthresh = 0.0;
    o->max_iter = 10;
    o->prior = 1;
    o->sub_batches = 0;
    o->verbose = 0;
}

rmx_status rmx_graph_create(const int32_t *src, const int32_t *dst, const double *w, int64_t n_edges, int32_t n_nodes,
                            const double *node_w, rmx_graph **out) {
    if (!out) return fail(RMX_ERR_INVALID, "out is NULL");
    *out = nullptr;
    rmx_graph *g = nullptr;
    rmx_status st = guard([&] {
        g = new rmx_graph();
        g->create(src, dst, w, n_edges, n_nodes, node_w);
    });
    if (st != RMX_OK) {
        delete g;
        return st;
    }
    *out = g;
    return RMX_OK;
}

rmx_status rmx_graph_load_file(const char *path, int32_t threads, rmx_graph **out) {
    if (!out) return fail(RMX_ERR_INVALID, "out is NULL");
    if (!path) return fail(RMX_ERR_INVALID, "path is NULL");
    *out = nullptr;
    rmx_graph *g = nullptr;
    rmx_status st = guard([&] {
        rmx::ParsedGraph pg = rmx::parse_file(path, threads);
        if (pg.n <= 0) throw rmx::FormatError(std::string("no nodes in ") + path);
        g = new rmx_graph();
        g->create(pg.src.data(), pg.dst.data(), pg.w.data(), (int64_t)pg.src.size(), pg.n,
                  pg.node_w.empty() ? nullptr : pg.node_w.data());
        g->n_self += pg.n_self;
        g->names.swap(pg.names);
    });
    if (st != RMX_OK) {
        delete g;
        return st;
    }
    *out = g;
    return RMX_OK;
}

rmx_status rmx_parse_file(const char *path, int32_t threads, int32_t *n_nodes, int64_t *n_edges, int64_t *n_self,
                          int32_t *src, int32_t *dst, double *w, double *node_w) {
    return guard([&] {
        need(path, "path");
        struct stat st {};
        const bool have_st = stat(path, &st) == 0;
        ParseCache &c = g_parse_cache;
        rmx::ParsedGraph pg;
        if (c.valid && have_st && c.path == path && c.threads == threads && same_file(c.st, st)) {
            pg = std::move(c.pg);
        } else {
            c = ParseCache();
            pg = rmx::parse_file(path, threads);
        }
        c = ParseCache();
        if (!src && !dst && !w && !node_w && have_st) {  // a size query: the fill call follows
            c.valid = true;
            c.path = path;
            c.threads = threads;
            c.st = st;
        }
        if (n_nodes) *n_nodes = pg.n;
        if (n_edges) *n_edges = (int64_t)pg.src.size();
        if (n_self) *n_self = pg.n_self;
        const size_t m = pg.src.size();
        if (src) std::memcpy(src, pg.src.data(), sizeof(int32_t) * m);
        if (dst) std::memcpy(dst, pg.dst.data(), sizeof(int32_t) * m);
        if (w) std::memcpy(w, pg.w.data(), sizeof(double) * m);
        if (node_w)
            for (int32_t i = 0; i < pg.n; i++) node_w[i] = pg.node_w.empty() ? 1.0 : pg.node_w[i];
        if (c.valid) c.pg = std::move(pg);
    });
}

rmx_status rmx_graph_destroy(rmx_graph *g) {
    return guard([&] { delete g; });
}

rmx_status rmx_graph_info(const rmx_graph *g, int32_t *n_nodes, int64_t *n_links, int64_t *n_self_links) {
    return guard([&] {
        need(g, "graph");
        if (n_nodes) *n_nodes = g->N;
        if (n_links) *n_links = g->E;
        if (n_self_links) *n_self_links = g->n_self;
    });
}

rmx_status rmx_graph_links(const rmx_graph *g, int64_t *off, int32_t *dst, double *w, double *teleport) {
    return guard([&] {
        need(g, "graph");
        cudaStream_t s = g->stream;
        if (off) RMX_CUDA(cudaMemcpyAsync(off, g->out_off, sizeof(int64_t) * (g->N + 1), cudaMemcpyDeviceToHost, s));
        if (dst && g->E) RMX_CUDA(cudaMemcpyAsync(dst, g->out_dst, sizeof(int32_t) * g->E, cudaMemcpyDeviceToHost, s));
        if (w && g->E) RMX_CUDA(cudaMemcpyAsync(w, g->out_w0, sizeof(double) * g->E, cudaMemcpyDeviceToHost, s));
        if (teleport) RMX_CUDA(cudaMemcpyAsync(teleport, g->tw, sizeof(double) * g->N, cudaMemcpyDeviceToHost, s));
        RMX_CUDA(cudaStreamSynchronize(s));
    });
}

rmx_status rmx_initiate(rmx_graph *g, double *p, double *f, double *exitpr, uint8_t *dangling, int32_t *iters,
                        double *L0) {
    return guard([&] {
        need(g, "graph");
        g->initiate();
        cudaStream_t s = g->stream;
        if (p) RMX_CUDA(cudaMemcpyAsync(p, g->p, sizeof(double) * g->N, cudaMemcpyDeviceToHost, s));
        if (f && g->E) RMX_CUDA(cudaMemcpyAsync(f, g->out_f, sizeof(double) * g->E, cudaMemcpyDeviceToHost, s));
        if (dangling) RMX_CUDA(cudaMemcpyAsync(dangling, g->dangling, g->N, cudaMemcpyDeviceToHost, s));
        if (exitpr) {
            size_t mk = g->scratch.mark();
            double *ex = g->scratch.alloc<double>(g->N);
            rmx::singleton_exits(g->N, g->out_off, g->out_f, g->p, g->tw, g->dangling, ex, s);
            RMX_CUDA(cudaMemcpyAsync(exitpr, ex, sizeof(double) * g->N, cudaMemcpyDeviceToHost, s));
            RMX_CUDA(cudaStreamSynchronize(s));
            g->scratch.release(mk);
        }
        RMX_CUDA(cudaStreamSynchronize(s));
        if (iters) *iters = g->power_iters;
        if (L0) *L0 = g->L0;
    });
}

rmx_status rmx_reset_flow(rmx_graph *g) {
    return guard([&] {
        need(g, "graph");
        RMX_CUDA(cudaStreamSynchronize(g->stream));
        g->initiated = false;
    });
}

rmx_status rmx_codelength(rmx_graph *g, const int32_t *part, double *L) {
    return guard([&] {
        need(g, "graph");
        need(part, "part");
        need(L, "L");
        *L = g->codelength_fp64(part);
    });
}

rmx_status rmx_batch_create(int32_t n_graphs, const int32_t *n_nodes, const int64_t *n_edges, const int32_t *src,
                            const int32_t *dst, const double *w, const double *node_w, rmx_batch **out) {
    if (!out) return fail(RMX_ERR_INVALID, "out is NULL");
    *out = nullptr;
    rmx_batch *b = nullptr;
    rmx_status st = guard([&] {
        b = new rmx_batch();
        b->create(n_graphs, n_nodes, n_edges, src, dst, w, node_w);
    });
    if (st != RMX_OK) {
        delete b;
        return st;
    }
    *out = b;
    return RMX_OK;
}

rmx_status rmx_batch_set_wave(rmx_batch *b, int64_t max_links, int64_t max_nodes) {
    return guard([&] {
        need(b, "batch");
        if (max_links < 1 || max_nodes < 1) throw std::invalid_argument("wave budget must be positive");
        b->wave_links = max_links;
        b->wave_nodes = max_nodes;
    });
}

rmx_status rmx_batch_optimize(rmx_batch *b, const rmx_opts *opts, int32_t *part_out, double *L_out,
                              int32_t *n_modules, int32_t *best_attempt) {
    return guard([&] {
        need(b, "batch");
        rmx_opts o;
        rmx_opts_default(&o);
        if (opts) o = *opts;
        b->optimize(o, part_out, L_out, n_modules, best_attempt);
    });
}

rmx_status rmx_batch_info(const rmx_batch *b, int32_t *n_graphs, int32_t *waves, int64_t *instances,
                          double *device_ms) {
    return guard([&] {
        need(b, "batch");
        if (n_graphs) *n_graphs = b->G;
        if (waves) *waves = b->last_waves;
        if (instances) *instances = b->last_instances;
        if (device_ms) *device_ms = b->last_ms;
    });
}

rmx_status rmx_batch_destroy(rmx_batch *b) {
    return guard([&] { delete b; });
}

rmx_status rmx_adjoint_forward(rmx_graph *g, const int32_t *part, double tau, double *L, double *p) {
    return guard([&] {
        need(g, "graph");
        need(part, "part");
        need(L, "L");
        g->adjoint(part, tau, L, p, nullptr, nullptr, nullptr);
    });
}

rmx_status rmx_adjoint_backward(rmx_graph *g, const int32_t *part, double tau, double *dL_dw, double *dL_dtau,
                                double *L) {
    return guard([&] {
        need(g, "graph");
        need(part, "part");
        if (!dL_dw && !dL_dtau) throw std::invalid_argument("dL_dw and dL_dtau are both NULL");
        g->adjoint(part, tau, L, nullptr, dL_dw, dL_dtau, nullptr);
    });
}

rmx_status rmx_coarsen(rmx_graph *g, const int32_t *part, int32_t *n_sn, int64_t *n_sn_links, int32_t *sn_of_mod,
                       int64_t *out_off, int32_t *out_dst, double *out_f, int64_t *in_off, int32_t *in_src,
                       double *in_f) {
    return guard([&] {
        need(g, "graph");
        need(part, "part");
        g->coarsen_hook(part, n_sn, n_sn_links, sn_of_mod, out_off, out_dst, out_f, in_off, in_src, in_f);
    });
}

rmx_status rmx_evaluate_moves(rmx_graph *g, const int32_t *part, const uint8_t *allow_new, int32_t *best_mod,
                              double *best_delta) {
    return guard([&] {
        need(g, "graph");
        need(part, "part");
        need(best_mod, "best_mod");
        need(best_delta, "best_delta");
        g->evaluate_hook(part, allow_new, best_mod, best_delta);
    });
}

rmx_status rmx_coarsen_engine(rmx_graph *g, const int32_t *part, const int32_t *part2, int32_t *n_sn,
                              int64_t *n_sn_links, int32_t *sn_of_mod, int64_t *out_off, int32_t *out_dst,
                              int64_t *out_fx, int64_t *in_off, int32_t *in_src, int64_t *in_fx, int64_t *sn_stat) {
    return guard([&] {
        need(g, "graph");
        need(part, "part");
        using fxp = rmx::fx_t *;
        g->coarsen_engine_hook(part, part2, n_sn, n_sn_links, sn_of_mod, out_off, out_dst,
                               reinterpret_cast<fxp>(out_fx), in_off, in_src, reinterpret_cast<fxp>(in_fx),
                               reinterpret_cast<fxp>(sn_stat));
    });
}

rmx_status rmx_evaluate_sn_moves(rmx_graph *g, const int32_t *part, int32_t n_sn, const int32_t *sn_part,
                                 const uint8_t *allow_new, int32_t *best_mod, double *best_delta) {
    return guard([&] {
        need(g, "graph");
        need(part, "part");
        need(sn_part, "sn_part");
        need(best_mod, "best_mod");
        need(best_delta, "best_delta");
        if (n_sn < 1) throw std::invalid_argument("n_sn must be positive");
        g->evaluate_sn_hook(part, n_sn, sn_part, allow_new, best_mod, best_delta);
    });
}

rmx_status rmx_optimize(rmx_graph *g, const rmx_opts *opts, int32_t *part_out, double *L_out, int32_t *n_modules) {
    return guard([&] {
        need(g, "graph");
        rmx_opts o;
        if (opts)
            o = *opts;
        else
            rmx_opts_default(&o);
        const double L = g->optimize(o, part_out, n_modules);
        if (L_out) *L_out = L;
    });
}

int32_t rmx_superstep_codelengths(const rmx_graph *g, double *bits, int32_t cap) {
    if (!g) return 0;
    const int32_t n = (int32_t)g->step_bits.size();
    for (int32_t i = 0; i < n && i < cap && bits; i++) bits[i] = g->step_bits[i];
    return n;
}

rmx_status rmx_write_outputs(rmx_graph *g, const int32_t *part, double L, const char *outdir, const char *name) {
    return guard([&] {
        need(g, "graph");
        need(part, "part");
        need(outdir, "outdir");
        need(name, "name");
        g->initiate();
        std::vector<int32_t> pv(part, part + g->N);
        for (int32_t m : pv)
            if ((uint32_t)m >= (uint32_t)g->N) throw std::invalid_argument("module id outside 0..N-1");
        std::vector<double> size(g->N);
        RMX_CUDA(cudaMemcpyAsync(size.data(), g->p, sizeof(double) * g->N, cudaMemcpyDeviceToHost, g->stream));
        RMX_CUDA(cudaStreamSynchronize(g->stream));
        std::vector<uint8_t> seen(g->N, 0);
        int32_t nm = 0;
        for (int32_t m : pv)
            if (!seen[m]) {
                seen[m] = 1;
                nm++;
            }
        const std::string base = std::string(outdir) + "/" + name;
        rmx::write_tree(base + ".tree", L / std::log(2.0), nm, pv, size, g->names);
        rmx::write_clu(base + ".clu", pv);
    });
}

rmx_status rmx_read_clu(const char *path, int32_t n_nodes, int32_t *part_out) {
    return guard([&] {
        need(path, "path");
        need(part_out, "part_out");
        if (n_nodes <= 0) throw std::invalid_argument("n_nodes must be positive");
        const std::vector<int32_t> part = rmx::read_clu(path, n_nodes);
        std::memcpy(part_out, part.data(), sizeof(int32_t) * part.size());
    });
}

rmx_status rmx_set_profiling(rmx_graph *g, int32_t on) {
    return guard([&] {
        need(g, "graph");
        g->timers.on = on != 0;
        g->timers.reset();
        g->prof = rmx_profile{};
        RMX_CUDA(cudaMemsetAsync(g->work.counters + rmx::kCntBins, 0, 3 * rmx::kEvalBins * sizeof(int64_t),
                                 g->stream));
        RMX_CUDA(cudaStreamSynchronize(g->stream));
    });
}

rmx_status rmx_get_profile(const rmx_graph *g, rmx_profile *out) {
    return guard([&] {
        need(g, "graph");
        need(out, "out");
        rmx_graph *h = const_cast<rmx_graph *>(g);
        if (h->timers.on) h->timers.resolve();
        *out = g->prof;
        for (int k = 0; k < RMX_K_COUNT; k++) {
            out->k[k].launches = g->timers.launches[k];
            out->k[k].ms = g->timers.ms[k];
            out->k[k].bytes = 0.0;
        }
        int64_t c[3 * rmx::kEvalBins];
        RMX_CUDA(cudaMemcpyAsync(c, g->work.counters + rmx::kCntBins, sizeof c, cudaMemcpyDeviceToHost, g->stream));
        RMX_CUDA(cudaStreamSynchronize(g->stream));
        out->links_evaluated = out->units_evaluated = out->candidates_evaluated = 0;
        for (int b = 0; b < rmx::kEvalBins; b++) {
            out->links_evaluated += c[3 * b];
            out->units_evaluated += c[3 * b + 1];
            out->candidates_evaluated += c[3 * b + 2];
            out->eval_bin_links[b] = c[3 * b];
            out->eval_bin_bytes[b] = g->timers.eval_bin_bytes[b];
        }
        out->k[RMX_K_EVAL].bytes = g->timers.eval_bytes;  // compulsory bytes per launch group (Timers)
        // The transposed solve, per sweep: link index, weight and the gathered
        // adjoint value (4 + 8 + 8 B per link); per node, the offsets, row sum,
        // right-hand side, teleport weight, dangling flag, the old value read
        // and the new one written and copied back (8+8+8+8+1+8+8+8+8 B).
        out->k[RMX_K_ADJOINT].bytes =
            (double)g->prof.adjoint_iters * (20.0 * (double)g->E + 65.0 * (double)g->N);
        for (int k = 0; k < 3; k++) out->level_ms[k] = g->timers.ms[rmx::kTimerLvNode + k];
        for (int k = 0; k < 6; k++) {
            out->eval_bin_ms[k] = g->timers.ms[rmx::kTimerBinReg + k];
            out->eval_bin_launches[k] = g->timers.launches[rmx::kTimerBinReg + k];
        }
        out->power_iters = g->power_iters;
        out->kernel_launches = (int64_t)__atomic_load_n(&rmx::g_kernel_launches, __ATOMIC_RELAXED);
    });
}

void *rmx_graph_stream(const rmx_graph *g) { return g ? (void *)g->stream : nullptr; }

rmx_status rmx_sync(rmx_graph *g) {
    return guard([&] {
        need(g, "graph");
        RMX_CUDA(cudaStreamSynchronize(g->stream));
    });
}

rmx_status rmx_get_tuning(rmx_tuning *out) {
    return guard([&] {
        need(out, "out");
        const rmx::EvalTuning t = rmx::eval_tuning();
        *out = rmx_tuning{};
        out->eval_mid_grid = t.mid;
        out->eval_block_grid = t.block;
        out->eval_large_grid = t.large;
        out->eval_warp_grid = t.warp;
        out->eval_reg_grid = t.reg;
        out->warp_max_degree = t.warp_max;
        out->mid_max_degree = t.mid_max;
        out->block_max_degree = t.block_max;
        out->large_max_degree = t.large_max;
        out->hub_partition_links = t.hub_part;
    });
}

rmx_status rmx_set_tuning(const rmx_tuning *t) {
    return guard([&] {
        need(t, "tuning");
        rmx::EvalTuning v;
        v.mid = t->eval_mid_grid;
        v.block = t->eval_block_grid;
        v.large = t->eval_large_grid;
        v.warp = t->eval_warp_grid;
        v.reg = t->eval_reg_grid;
        v.warp_max = t->warp_max_degree;
        v.mid_max = t->mid_max_degree;
        v.block_max = t->block_max_degree;
        v.large_max = t->large_max_degree;
        v.hub_part = t->hub_partition_links;
        rmx::set_eval_tuning(v);
    });
}

rmx_status rmx_release_device_cache(void) {
    return guard([&] { rmx::release_device_cache(); });
}

}  // extern "C"
