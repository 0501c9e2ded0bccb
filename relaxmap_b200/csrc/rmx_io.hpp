// Host-side input parsing and output writing with the reference's rules.
#pragma once
#include <cstdint>
#include <exception>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

namespace rmx {

// job(t) for t < T on T host threads (inline for T == 1); the first exception
// a job throws (or a failed thread start) is rethrown after every started
// thread has joined.
template <typename Job>
void run_parallel(int T, Job &&job) {
    if (T <= 1) {
        job(0);
        return;
    }
    std::exception_ptr err;
    std::mutex err_mu;
    auto guarded = [&](int t) {
        try {
            job(t);
        } catch (...) {
            std::lock_guard<std::mutex> lk(err_mu);
            if (!err) err = std::current_exception();
        }
    };
    std::vector<std::thread> pool;
    try {
        for (int t = 0; t < T; t++) pool.emplace_back(guarded, t);
    } catch (...) {
        std::lock_guard<std::mutex> lk(err_mu);
        if (!err) err = std::current_exception();
    }
    for (auto &th : pool) th.join();
    if (err) std::rethrow_exception(err);
}

struct IoError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct FormatError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// std::allocator whose default construction of trivial elements leaves them
// uninitialised: resize() of an array that parser threads then fill touches
// no page itself, so the pages are first touched by those threads, in
// parallel, instead of being zeroed by one.
template <typename T>
struct NoInitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <typename U>
    NoInitAlloc(const NoInitAlloc<U> &) noexcept {}
    template <typename U>
    void construct(U *p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new (static_cast<void *>(p)) U;
    }
    template <typename U, typename... Args>
    void construct(U *p, Args &&...args) {
        ::new (static_cast<void *>(p)) U(std::forward<Args>(args)...);
    }
};
template <typename T>
using HostVec = std::vector<T, NoInitAlloc<T>>;

// What a reference loader leaves behind, as raw (unsummed) edges in file
// order: the device build sums duplicates in that order.
struct ParsedGraph {
    int32_t n = 0;
    HostVec<int32_t> src, dst;
    HostVec<double> w;
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
// A .clu file as write_clu writes it ("*Vertices N", then N labels = module
// index + 1; CRLF or LF): the module index of each of the n nodes. A vertex
// count other than n, a label that is not an integer in 1..n, or a missing
// label is a FormatError; an unreadable file an IoError.
std::vector<int32_t> read_clu(const std::string &file, int32_t n);

}  // namespace rmx
