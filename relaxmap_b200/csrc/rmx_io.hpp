// Host-side input parsing and output writing with the reference's rules.
#pragma once
#include <stdexcept>
#include <string>
#include <vector>

namespace rmx {

struct IoError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct FormatError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// What a reference loader leaves behind, as raw (unsummed) edges in file
// order: the device build sums duplicates in that order.
struct ParsedGraph {
    int32_t n = 0;
    std::vector<int32_t> src, dst;
    std::vector<double> w;
    std::vector<double> node_w;  // empty: uniform (edge-list files)
    std::vector<std::string> names;
    int64_t n_self = 0;          // self-link pairs with positive summed weight
    int64_t n_lines = 0;
};

// load_linkList_format_network (FileIO.cpp:177-265).
ParsedGraph parse_edge_list(const std::string &path, int threads);
// load_pajek_format_network (FileIO.cpp:32-171).
ParsedGraph parse_pajek(const std::string &path, int threads = 1);
// Choose by extension as main does (OmpRelaxmap.cpp:60, :93-98).
ParsedGraph parse_file(const std::string &path, int threads);

// .tree (print_twoLevel_Cluster, OmpRelaxmap.cpp:790-812) and .clu
// (OmpRelaxmap.cpp:240-249).
void write_tree(const std::string &file, double L_bits, int32_t n_modules, const std::vector<int32_t> &part,
                const std::vector<double> &size, const std::vector<std::string> &names);
void write_clu(const std::string &file, const std::vector<int32_t> &part);

}  // namespace rmx
