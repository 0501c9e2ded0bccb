// The ompRelaxmap command line on the B200 engine (OmpRelaxmap.cpp:41-252):
// same positional arguments, the same key stdout lines and the same .tree /
// .clu files, so scripts can drive either binary.
#include <sys/time.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/relaxmap_b200.h"

namespace {

double now_s() {
    struct timeval t;
    gettimeofday(&t, nullptr);
    return t.tv_sec + 1e-6 * t.tv_usec;
}

// Applies a launch tuning file (the JSON that relaxmap_b200.autotune writes):
// every grid cap ("eval_*_grid") and bin bound ("*_max_degree") found in it,
// the others keep their values. The values change run time only, never results.
bool apply_tuning_file(const std::string &path) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) {
        printf("cannot read the tuning file %s\n", path.c_str());
        return false;
    }
    std::string text;
    char buf[4096];
    size_t r;
    while ((r = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, r);
    fclose(f);
    rmx_tuning t;
    rmx_get_tuning(&t);
    struct Field {
        const char *name;
        int32_t *v;
    } fields[] = {{"\"eval_mid_grid\"", &t.eval_mid_grid},
                  {"\"eval_block_grid\"", &t.eval_block_grid},
                  {"\"eval_large_grid\"", &t.eval_large_grid},
                  {"\"eval_warp_grid\"", &t.eval_warp_grid},
                  {"\"eval_reg_grid\"", &t.eval_reg_grid},
                  {"\"warp_max_degree\"", &t.warp_max_degree},
                  {"\"mid_max_degree\"", &t.mid_max_degree},
                  {"\"block_max_degree\"", &t.block_max_degree},
                  {"\"large_max_degree\"", &t.large_max_degree},
                  {"\"hub_partition_links\"", &t.hub_partition_links}};
    for (const Field &fd : fields) {
        const size_t k = text.find(fd.name);
        if (k == std::string::npos) continue;
        const size_t colon = text.find(':', k);
        if (colon == std::string::npos) continue;
        char *end = nullptr;
        const long v = strtol(text.c_str() + colon + 1, &end, 10);
        if (end == text.c_str() + colon + 1) {
            printf("tuning file %s: %s has no integer value\n", path.c_str(), fd.name);
            return false;
        }
        *fd.v = (int32_t)std::max(-1L, std::min(v, 1L << 30));  // out-of-range values are rejected below
    }
    if (rmx_set_tuning(&t) != RMX_OK) {
        printf("tuning file %s: %s\n", path.c_str(), rmx_last_error());
        return false;
    }
    printf("Launch tuning from %s: grid caps (blocks per SM) mid %d, block %d, large %d, warp %d, register %d; "
           "bin bounds (links) warp %d, mid %d, block %d, large %d; hub partitions of %d links\n",
           path.c_str(), t.eval_mid_grid, t.eval_block_grid, t.eval_large_grid, t.eval_warp_grid, t.eval_reg_grid,
           t.warp_max_degree, t.mid_max_degree, t.block_max_degree, t.large_max_degree, t.hub_partition_links);
    return true;
}

}  // namespace

extern "C" int rmx_cli_main(int argc, char **argv) {
    if (argc < 10) {
        printf("Call: ./ompRelaxmap <seed> <network.net> <# threads> <# attempts> <threshold> <vThresh> <maxIter> "
               "<outDir> <prior/normal>  [selflinks] [--tuning=<file>]\n");
        return -1;
    }
    const std::string outDir = argv[8];
    rmx_opts o;
    rmx_opts_default(&o);
    o.max_iter = atoi(argv[7]);
    o.attempts = atoi(argv[4]);
    o.threads = atoi(argv[3]);
    o.seed = (uint32_t)strtoul(argv[1], nullptr, 10);
    const std::string infile = argv[2];
    // networkName keeps the leading '/' (OmpRelaxmap.cpp:59); without a '/' the
    // whole stem is used with one prepended.
    const size_t slash = infile.find_last_of('/');
    const size_t dot = infile.find_last_of('.');
    const size_t b = slash == std::string::npos ? 0 : slash;
    const size_t e = (dot == std::string::npos || dot < b) ? infile.size() : dot;
    std::string name = infile.substr(b, e - b);
    if (slash == std::string::npos) name = "/" + name;
    o.threshold = atof(argv[5]);
    o.vthresh = atof(argv[6]);
    printf("Threshold = %g, Vertex-Threshold = %g\n", o.threshold, o.vthresh);
    o.prior = std::string(argv[9]) == "prior";
    // options of this build (--tuning=<file>) may follow the positional
    // arguments; without them "selflinks" counts only as the single argument
    // after the ninth (argc == 11, OmpRelaxmap.cpp:75-77), and so it does here
    std::vector<std::string> extra;
    for (int i = 10; i < argc; i++) {
        const std::string a = argv[i];
        if (a.rfind("--tuning=", 0) == 0) {
            if (!apply_tuning_file(a.substr(9))) return -1;
        } else {
            extra.push_back(a);
        }
    }
    const bool selflinks = extra.size() == 1 && extra[0] == "selflinks";
    o.verbose = 1;

    const double all0 = now_s();
    rmx_graph *g = nullptr;
    printf("Reading network %s file\n", infile.c_str());
    rmx_status st = rmx_graph_load_file(infile.c_str(), o.threads > 0 ? o.threads : 1, &g);
    if (st != RMX_OK) {
        printf("%s\n", rmx_last_error());
        return -1;
    }
    int32_t N = 0;
    int64_t E = 0, nself = 0;
    rmx_graph_info(g, &N, &E, &nself);
    const double io1 = now_s();
    printf("done! (found %d nodes and %lld edges.)\n", N, (long long)E);
    printf("Time for reading input data : %g (sec)\n", io1 - all0);
    if (selflinks)
        printf("current version always excludes self links.\nignoring %lld self link(s).\n", (long long)nself);
    else
        printf("ignoring %lld self link(s).\n", (long long)nself);
    printf("DONE: Parsing the given network  ...\n");
    int32_t iters = 0;
    double L0 = 0;
    st = rmx_initiate(g, nullptr, nullptr, nullptr, nullptr, &iters, &L0);
    if (st != RMX_OK) {
        printf("%s\n", rmx_last_error());
        rmx_graph_destroy(g);
        return -1;
    }
    printf("Calculating flow done in %d iterations!\n", iters);
    printf("Initial Code Length: %g in %d modules.\n", L0 / std::log(2.0), N);
    printf("Now partition the network starts...\n");
    std::vector<int32_t> part(N);
    double L = 0;
    int32_t nmod = 0;
    st = rmx_optimize(g, &o, part.data(), &L, &nmod);
    if (st != RMX_OK) {
        printf("%s\n", rmx_last_error());
        rmx_graph_destroy(g);
        return -1;
    }
    const double t1 = now_s();
    printf("DONE: Code Length = %g in %d modules, with %d nodes.\n\n", L / std::log(2.0), nmod, N);
    printf("Overall Elapsed Time for Module Detection (w/o file IO): %g (sec)\n", t1 - io1);
    printf("Overall Elapsed Time for Module Detection (w/ file Reading): %g (sec)\n", t1 - all0);
    double Lc = 0;
    if (rmx_codelength(g, part.data(), &Lc) == RMX_OK) printf("\nComputed Code Length = %g\n", Lc / std::log(2.0));
    st = rmx_write_outputs(g, part.data(), L, outDir.c_str(), name.c_str());
    if (st != RMX_OK) printf("%s\n", rmx_last_error());
    rmx_graph_destroy(g);
    return 0;
}
