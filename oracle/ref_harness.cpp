// Test-only harness over the reference implementation (oracle infrastructure).
//
// This file is ours; it is compiled together with the UNMODIFIED reference
// sources (Node.cpp, Module.cpp, FileIO.cpp, timing.cpp, OmpRelaxmap.cpp with
// main renamed) by oracle/Makefile into oracle/_ref/librmxref.so. It exposes
// a C ABI so the Python tests and bench.py --impl reference can drive the
// reference's own routines in-process and read results at full precision:
//   - loaders           FileIO.cpp:32-171 (Pajek), FileIO.cpp:177-265 (edge list)
//   - edge preparation  OmpRelaxmap.cpp:104-162
//   - initiate/flows    Module.cpp:210-333, 340-469
//   - code length       Module.cpp:2966-3002
//   - coarsening        Module.cpp:3008-3077 (convertModulesToSuperNodes)
//   - full optimiser    OmpRelaxmap.cpp:170-233 (main's superstep loop)
// Nothing on the product path links or loads this library.

#include <cstdio>
#include <cstring>
#include <ctime>
#include <iostream>
#include <map>
#include <string>
#include <vector>

#include "FileIO.h"
#include "Module.h"
#include "Node.h"

using namespace std;

// Driver functions defined in the reference's OmpRelaxmap.cpp.
void stochastic_greedy_partition(Network &network, int numTh, double threshold, double vThresh,
                                 int maxIter, bool prior, bool fineTune, bool fast);
void generate_sub_modules(Network &network, int numTh, double threshold, int maxIter);

namespace {

struct Quiet {  // silence the reference's progress printing while a call runs
    streambuf *old;
    Quiet() : old(cout.rdbuf(NULL)) {}
    ~Quiet() {
        cout.rdbuf(old);
        cout.clear();
    }
};

double now_s() {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

struct RefNet {
    Network net;
    MTRand *R;
    vector<double> nodeSize;
    vector<int> steps_unused;
    RefNet() : R(NULL) {}
    ~RefNet() { delete R; }
};

}  // namespace

extern "C" {

// Loader-equivalent construction from raw arrays: duplicate (src,dst) pairs are
// summed in input order exactly as the loaders do (FileIO.cpp:157, :220).
// node_w may be NULL (uniform weight 1, total = N as in FileIO.cpp:229).
void *rmxref_create(int N, long long E, const int *src, const int *dst, const double *w,
                    const double *node_w) {
    RefNet *h = new RefNet();
    Network &net = h->net;
    net.setNNode(N);
    net.modules = vector<Module>(N);
    net.nodes = vector<Node>(N);
    double tot = 0.0;
    for (int i = 0; i < N; i++) {
        net.nodes[i].setID(i);
        double nw = node_w ? node_w[i] : 1.0;
        net.nodes[i].setNodeWeight(nw);
        tot += nw;
    }
    net.setTotNodeWeights(node_w ? tot : (double)N);
    for (long long e = 0; e < E; e++) net.Edges[make_pair(src[e], dst[e])] += (w ? w[e] : 1.0);
    net.setNEdge(net.Edges.size());
    return h;
}

// Reference loaders (FileIO.cpp). is_pajek selects load_pajek_format_network.
void *rmxref_load_file(const char *path, int is_pajek) {
    RefNet *h = new RefNet();
    Quiet q;
    if (is_pajek)
        load_pajek_format_network(string(path), h->net);
    else
        load_linkList_format_network(string(path), h->net);
    return h;
}

void rmxref_destroy(void *p) { delete (RefNet *)p; }

int rmxref_nnode(void *p) { return ((RefNet *)p)->net.NNode(); }
double rmxref_tot_node_weights(void *p) { return ((RefNet *)p)->net.TotNodeWeights(); }

// Loader output before edge preparation: the summed edge map in key order.
long long rmxref_num_map_edges(void *p) { return (long long)((RefNet *)p)->net.Edges.size(); }
void rmxref_get_map_edges(void *p, int *src, int *dst, double *w) {
    RefNet *h = (RefNet *)p;
    long long k = 0;
    for (map<pair<int, int>, double>::iterator it = h->net.Edges.begin(); it != h->net.Edges.end(); ++it, ++k) {
        src[k] = it->first.first;
        dst[k] = it->first.second;
        w[k] = it->second;
    }
}
int rmxref_node_name(void *p, int i, char *buf, int cap) {
    string s = ((RefNet *)p)->net.nodes[i].Name();
    snprintf(buf, cap, "%s", s.c_str());
    return (int)s.size();
}
double rmxref_node_weight(void *p, int i) { return ((RefNet *)p)->net.nodes[i].NodeWeight(); }

// OmpRelaxmap.cpp:104-162: teleport weights, edge map -> outLinks (self-loops and
// non-positive weights dropped), Network::initiate, inLinks. Returns seconds.
double rmxref_prepare(void *p, int numTh) {
    RefNet *h = (RefNet *)p;
    Network &net = h->net;
    Quiet q;
    double t0 = now_s();
    int nNode = net.NNode();
    double tot = net.TotNodeWeights();
    for (int i = 0; i < nNode; i++) net.nodes[i].setTeleportWeight(net.nodes[i].NodeWeight() / tot);
    for (map<pair<int, int>, double>::iterator it = net.Edges.begin(); it != net.Edges.end(); ++it) {
        int from = it->first.first, to = it->first.second;
        double weight = it->second;
        if (weight > 0.0 && from != to) net.nodes[from].outLinks.push_back(make_pair(to, weight));
    }
    map<pair<int, int>, double>().swap(net.Edges);
    net.initiate(numTh);
    for (int i = 0; i < nNode; i++) {
        int n = net.nodes[i].outLinks.size();
        for (int j = 0; j < n; j++)
            net.nodes[net.nodes[i].outLinks[j].first].inLinks.push_back(make_pair(i, net.nodes[i].outLinks[j].second));
    }
    h->nodeSize.resize(nNode);
    for (int i = 0; i < nNode; i++) h->nodeSize[i] = net.nodes[i].Size();
    return now_s() - t0;
}

long long rmxref_num_links(void *p) {
    RefNet *h = (RefNet *)p;
    long long n = 0;
    for (int i = 0; i < h->net.NNode(); i++) n += h->net.nodes[i].outLinks.size();
    return n;
}

// Out-links (CSR by source, destinations ascending) with their current values
// (edge flows p_a * w_ab / sum_b w_ab after initiate).
void rmxref_get_links(void *p, long long *off, int *dst, double *f) {
    RefNet *h = (RefNet *)p;
    long long k = 0;
    off[0] = 0;
    for (int i = 0; i < h->net.NNode(); i++) {
        vector<pair<int, double> > &L = h->net.nodes[i].outLinks;
        for (size_t j = 0; j < L.size(); j++, k++) {
            dst[k] = L[j].first;
            f[k] = L[j].second;
        }
        off[i + 1] = k;
    }
}

// Per-node attributes after initiate: flow p, teleport weight tau, dangling
// size, singleton exit (Module.cpp:67-99), dangling flag.
void rmxref_get_nodes(void *p, double *size, double *tw, double *dsize, double *exitpr, char *dangling) {
    RefNet *h = (RefNet *)p;
    for (int i = 0; i < h->net.NNode(); i++) {
        Node &nd = h->net.nodes[i];
        size[i] = nd.Size();
        tw[i] = nd.TeleportWeight();
        dsize[i] = nd.DanglingSize();
        exitpr[i] = nd.ExitPr();
        dangling[i] = nd.IsDangling() ? 1 : 0;
    }
}

double rmxref_codelength(void *p) { return ((RefNet *)p)->net.CodeLength(); }
double rmxref_all_log_all(void *p) { return ((RefNet *)p)->net.AllLogAll(); }

// Replace the out-link flows (CSR order) and rebuild inLinks from them, so a
// coarsening can be compared bit-for-bit on identical input flows.
void rmxref_set_flows(void *p, const double *f) {
    RefNet *h = (RefNet *)p;
    Network &net = h->net;
    long long k = 0;
    for (int i = 0; i < net.NNode(); i++) {
        vector<pair<int, double> > &L = net.nodes[i].outLinks;
        for (size_t j = 0; j < L.size(); j++) L[j].second = f[k++];
        net.nodes[i].inLinks.clear();
    }
    for (int i = 0; i < net.NNode(); i++) {
        vector<pair<int, double> > &L = net.nodes[i].outLinks;
        for (size_t j = 0; j < L.size(); j++) net.nodes[L[j].first].inLinks.push_back(make_pair(i, L[j].second));
    }
}

// Install a partition (module index per node, each in [0,N)). Module sums are
// formed in node order; the module exit uses the calculateCodeLength formula
// (Module.cpp:2978-2991). Member lists are rebuilt by the reference's own
// updateMembersInModule (Module.cpp:2881-2902).
void rmxref_set_partition(void *p, const int *part) {
    RefNet *h = (RefNet *)p;
    Network &net = h->net;
    int N = net.NNode();
    vector<double> P(N, 0.0), TW(N, 0.0), D(N, 0.0), OUT(N, 0.0);
    vector<int> cnt(N, 0);
    for (int i = 0; i < N; i++) {
        Node &nd = net.nodes[i];
        nd.setModIdx(part[i]);
        int m = part[i];
        P[m] += nd.Size();
        TW[m] += nd.TeleportWeight();
        D[m] += nd.DanglingSize();
        cnt[m]++;
    }
    for (int i = 0; i < N; i++) {
        Node &nd = net.nodes[i];
        for (size_t j = 0; j < nd.outLinks.size(); j++)
            if (part[nd.outLinks[j].first] != part[i]) OUT[part[i]] += nd.outLinks[j].second;
    }
    int nMod = 0;
    net.emptyModules.clear();
    for (int m = 0; m < N; m++) {
        Module &M = net.modules[m];
        M.setIndex(m);
        M.setSumPr(P[m]);
        M.setSumTPWeight(TW[m]);
        M.setSumDangling(D[m]);
        M.setNumMembers(cnt[m]);
        double ex = 0.0;
        if (cnt[m] > 0) {
            ex = Network::alpha * (1.0 - TW[m]) * P[m] + Network::beta * (OUT[m] + (1.0 - TW[m]) * D[m]);
            nMod++;
        } else {
            net.emptyModules.push_back(m);
        }
        M.setExitPr(ex);
        M.setStayPr(ex + P[m]);
    }
    net.setNModule(nMod);
    net.setNEmptyMod(N - nMod);
    net.updateMembersInModule();
    net.calibrate(1);
}

double rmxref_calc_codelength(void *p) { return ((RefNet *)p)->net.calculateCodeLength(); }
double rmxref_sum_exit(void *p) { return ((RefNet *)p)->net.SumAllExitPr(); }

// convertModulesToSuperNodes (Module.cpp:3008-3077) on the installed partition.
int rmxref_convert(void *p) {
    RefNet *h = (RefNet *)p;
    Quiet q;
    h->net.convertModulesToSuperNodes(1);
    return (int)h->net.superNodes.size();
}
long long rmxref_sn_num_links(void *p) {
    RefNet *h = (RefNet *)p;
    long long n = 0;
    for (size_t i = 0; i < h->net.superNodes.size(); i++) n += h->net.superNodes[i].outLinks.size();
    return n;
}
void rmxref_sn_get(void *p, int *modidx, double *size, double *exitpr, double *tw, double *dsize, int *nmembers,
                   long long *out_off, int *out_dst, double *out_w, long long *in_off, int *in_src, double *in_w) {
    RefNet *h = (RefNet *)p;
    vector<SuperNode> &S = h->net.superNodes;
    long long ko = 0, ki = 0;
    out_off[0] = 0;
    in_off[0] = 0;
    for (size_t i = 0; i < S.size(); i++) {
        modidx[i] = S[i].ModIdx();
        size[i] = S[i].Size();
        exitpr[i] = S[i].ExitPr();
        tw[i] = S[i].TeleportWeight();
        dsize[i] = S[i].DanglingSize();
        nmembers[i] = (int)S[i].members.size();
        for (size_t j = 0; j < S[i].outLinks.size(); j++, ko++) {
            out_dst[ko] = S[i].outLinks[j].first;
            out_w[ko] = S[i].outLinks[j].second;
        }
        for (size_t j = 0; j < S[i].inLinks.size(); j++, ki++) {
            in_src[ki] = S[i].inLinks[j].first;
            in_w[ki] = S[i].inLinks[j].second;
        }
        out_off[i + 1] = ko;
        in_off[i + 1] = ki;
    }
}

// The first loop of stochastic_greedy_partition at one thread
// (OmpRelaxmap.cpp:276-339): Network::prioritize_move / Network::move sweeps
// from the singleton state after initiate. Returns the incremental code length
// (nats) and the module per node.
double rmxref_node_sweeps(void *p, unsigned seed, int prior, double vthresh_arg, double threshold, int maxIter,
                          int *part_out, int *n_sweeps) {
    RefNet *h = (RefNet *)p;
    Network &net = h->net;
    Quiet q;
    delete h->R;
    h->R = new MTRand(seed);
    net.R = h->R;
    double vThresh = -vthresh_arg;
    int n = net.NNode();
    vector<char>(n).swap(net.isActives);
    vector<int>(n).swap(net.activeNodes);
    for (int i = 0; i < n; i++) {
        net.activeNodes[i] = i;
        net.isActives[i] = 0;
    }
    int iter = 0;
    bool stop = false;
    while (!stop && iter < maxIter) {
        double oldL = net.CodeLength();
        if (prior)
            net.prioritize_move(vThresh);
        else
            net.move();
        iter++;
        if (oldL - net.CodeLength() >= 0 && (oldL - net.CodeLength()) / log(2.0) < threshold) stop = true;
    }
    *n_sweeps = iter;
    for (int i = 0; i < n; i++) part_out[i] = net.nodes[i].ModIdx();
    return net.CodeLength();
}

// generate_sub_modules (OmpRelaxmap.cpp:502-638) on the installed partition:
// returns the number of sub-module super-nodes and writes each node's
// sub-module index (ndToSubMod) and each super-node's parent module.
int rmxref_coarse_tune(void *p, int numTh, double threshold, int maxIter, int *sub_of_node, int *sn_parent) {
    RefNet *h = (RefNet *)p;
    Network &net = h->net;
    Quiet q;
    generate_sub_modules(net, numTh, threshold, maxIter);
    for (int i = 0; i < net.NNode(); i++) sub_of_node[i] = net.ndToSubMod[i];
    for (size_t s = 0; s < net.superNodes.size(); s++) sn_parent[s] = net.superNodes[s].ModIdx();
    return (int)net.superNodes.size();
}

// The reference's superstep loop (OmpRelaxmap.cpp:170-233) on a prepared network.
// vthresh_arg is the CLI value (negated internally as at OmpRelaxmap.cpp:66).
// Writes the final module index per node, the incremental code length and the
// from-scratch one (both in bits), the superstep code lengths (bits, up to
// max_steps) and returns the elapsed seconds of the loop.
double rmxref_partition(void *p, unsigned seed, int numTh, double threshold, double vthresh_arg, int maxIter,
                        int prior, int *part_out, double *L_bits, double *L_computed_bits, int *n_modules,
                        double *step_L_bits, int max_steps, int *n_steps) {
    RefNet *h = (RefNet *)p;
    Network &net = h->net;
    Quiet q;
    delete h->R;
    h->R = new MTRand(seed);
    net.R = h->R;
    double vThresh = -vthresh_arg;
    double t0 = now_s();
    bool fineTune = true, fast = false;
    int step = 1, ns = 0;
    double oldL = net.CodeLength();
    stochastic_greedy_partition(net, numTh, threshold, vThresh, maxIter, prior != 0, fineTune, fast);
    if (ns < max_steps) step_L_bits[ns] = net.CodeLength() / log(2.0);
    ns++;
    bool nextIter = (oldL - net.CodeLength()) / log(2.0) >= threshold;
    while (nextIter) {
        oldL = net.CodeLength();
        stochastic_greedy_partition(net, numTh, threshold, vThresh, maxIter, prior != 0, fineTune, fast);
        step++;
        if (ns < max_steps) step_L_bits[ns] = net.CodeLength() / log(2.0);
        ns++;
        if ((oldL - net.CodeLength()) / log(2.0) < threshold) nextIter = false;
        fineTune = !fineTune;
        if (nextIter && !fineTune) generate_sub_modules(net, numTh, threshold, maxIter);
    }
    double t1 = now_s();
    *n_steps = ns;
    *L_bits = net.CodeLength() / log(2.0);
    *n_modules = net.NModule();
    *L_computed_bits = net.calculateCodeLength() / log(2.0);
    for (int i = 0; i < net.NNode(); i++) part_out[i] = net.nodes[i].ModIdx();
    return t1 - t0;
}

}  // extern "C"
