// The ompRelaxmap command line on the B200 engine (OmpRelaxmap.cpp:41-252):
// same positional arguments, the same key stdout lines and the same .tree /
// .clu files, so scripts can drive either binary.
#include <sys/time.h>

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

}  // namespace

extern "C" int rmx_cli_main(int argc, char **argv) {
    if (argc < 10) {
        printf("Call: ./ompRelaxmap <seed> <network.net> <# threads> <# attempts> <threshold> <vThresh> <maxIter> "
               "<outDir> <prior/normal>  [selflinks]\n");
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
    bool selflinks = argc == 11 && std::string(argv[10]) == "selflinks";
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
