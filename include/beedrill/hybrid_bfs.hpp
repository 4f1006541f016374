// beedrill/hybrid_bfs.hpp -- C++ facade over the C ABI, keeping the public
// surface of the reference's hybrid_bfs class (hybrid_bfs.h:11-47) and the
// graph / edge-list calls its driver makes (hybrid_bfs_main.cc:164-246).
//
// Differences from the reference, by design:
//   * errors throw beedrill::error (carrying the bd_status) instead of
//     assert() / exit(1);
//   * the graph and BFS state live in HBM; results are copied to the host
//     only when asked for (depths(), parents(), check(), print_tree()).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "beedrill_b200.h"

namespace beedrill {

class error : public std::runtime_error {
public:
    error(bd_status s, const std::string &what)
        : std::runtime_error(what + ": " + bd_status_string(s)), status(s) {}
    bd_status status;
};

inline void throw_if(bd_status s, const char *what)
{
    if (s != BD_OK) { throw error(s, what); }
}

// A trained direction policy as the trainer (beedrill_b200/policy.py) writes
// it: a JSON object with the float arrays "params" (BD_POLICY_PARAMS),
// "mean", "inv_std", optionally "lo" and "hi" (BD_POLICY_FEATURES each), and
// the number "margin".  No counterpart in the reference.
struct policy {
    std::vector<float> params, mean, inv_std, lo, hi;
    float margin = 0.f;
};

namespace detail {
// The numbers of the JSON array stored under "key" (empty if absent).
inline std::vector<float> json_array(const std::string &text, const char *key)
{
    std::vector<float> out;
    const std::string k = std::string("\"") + key + "\"";
    size_t at = text.find(k);
    if (at == std::string::npos) { return out; }
    at = text.find_first_not_of(" \t\r\n:", at + k.size());
    if (at == std::string::npos || text[at] != '[') { return out; }
    const char *p = text.c_str() + at + 1;
    while (*p && *p != ']') {
        char *end = nullptr;
        const double v = strtod(p, &end);
        if (end == p) { throw error(BD_ERR_FORMAT, std::string("policy array ") + key); }
        out.push_back((float)v);
        p = end;
        while (*p == ',' || *p == ' ' || *p == '\n' || *p == '\r' || *p == '\t') { ++p; }
    }
    return out;
}
}  // namespace detail

inline policy load_policy(const std::string &path)
{
    FILE *fp = fopen(path.c_str(), "rb");
    if (!fp) { throw error(BD_ERR_IO, "policy file " + path); }
    std::string text;
    char buf[65536];
    size_t got;
    while ((got = fread(buf, 1, sizeof(buf), fp)) > 0) { text.append(buf, got); }
    fclose(fp);
    policy pol;
    pol.params = detail::json_array(text, "params");
    pol.mean = detail::json_array(text, "mean");
    pol.inv_std = detail::json_array(text, "inv_std");
    pol.lo = detail::json_array(text, "lo");
    pol.hi = detail::json_array(text, "hi");
    const size_t at = text.find("\"margin\"");
    if (at != std::string::npos) {
        const size_t colon = text.find(':', at);
        if (colon != std::string::npos) { pol.margin = strtof(text.c_str() + colon + 1, nullptr); }
    }
    const bool bounded = !pol.lo.empty() || !pol.hi.empty();
    if (pol.params.size() != BD_POLICY_PARAMS || pol.mean.size() != BD_POLICY_FEATURES ||
        pol.inv_std.size() != BD_POLICY_FEATURES ||
        (bounded && (pol.lo.size() != BD_POLICY_FEATURES || pol.hi.size() != BD_POLICY_FEATURES))) {
        throw error(BD_ERR_FORMAT, "policy file " + path);
    }
    return pol;
}

// Launch parameters chosen by the autotuner (beedrill_b200/autotune.py) for
// this GPU, read from its JSON file: the entry tuned at the graph scale
// nearest log2(n).  No counterpart in the reference.
struct tuning {
    std::map<std::string, double> single, batched;
    // Fills the fields an application left at 0 (library default) with the
    // tuned values; the batched rule's alpha is taken whenever it is tuned.
    void apply(bd_bfs_opts *o) const
    {
        set(single, "block_size", &o->block_size);
        set(single, "large_degree", &o->large_degree);
        set(single, "chunk_edges", &o->chunk_edges);
        set(single, "bu_prefix", &o->bu_prefix);
        set(single, "bu_words", &o->bu_words);
        set(single, "bu_sparse_words", &o->bu_sparse_words);
    }
    void apply(bd_msbfs_opts *o) const
    {
        auto a = batched.find("alpha");
        if (a != batched.end()) { o->alpha = (int64_t)a->second; }
        set(batched, "block_size", &o->block_size);
        set(batched, "large_degree", &o->large_degree);
        set(batched, "chunk_edges", &o->chunk_edges);
        set(batched, "pull_prefix", &o->pull_prefix);
        set(batched, "heavy_degree", &o->heavy_degree);
        set(batched, "heavy_chunk", &o->heavy_chunk);
    }

private:
    static void set(const std::map<std::string, double> &m, const char *k, int32_t *f)
    {
        auto it = m.find(k);
        if (it != m.end() && *f == 0) { *f = (int32_t)it->second; }
    }
};

namespace detail {
// A small JSON reader for the tuning file (objects, arrays, numbers,
// strings, true / false / null).
struct jvalue {
    enum kind_t { NUL, NUM, STR, ARR, OBJ, BOOL } kind = NUL;
    double num = 0;
    std::string str;
    std::vector<jvalue> arr;
    std::vector<std::pair<std::string, jvalue>> obj;
    const jvalue *get(const std::string &k) const
    {
        for (const auto &kv : obj) {
            if (kv.first == k) { return &kv.second; }
        }
        return nullptr;
    }
};

struct jparser {
    const char *p;
    void ws()
    {
        while (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t') { ++p; }
    }
    [[noreturn]] void fail() { throw error(BD_ERR_FORMAT, "tuning file"); }
    std::string string()
    {
        if (*p != '"') { fail(); }
        std::string out;
        for (++p; *p && *p != '"'; ++p) {
            if (*p == '\\' && p[1]) { ++p; }
            out += *p;
        }
        if (*p != '"') { fail(); }
        ++p;
        return out;
    }
    jvalue value()
    {
        ws();
        jvalue v;
        if (*p == '{') {
            v.kind = jvalue::OBJ;
            ++p;
            ws();
            while (*p != '}') {
                ws();
                std::string k = string();
                ws();
                if (*p != ':') { fail(); }
                ++p;
                v.obj.emplace_back(k, value());
                ws();
                if (*p == ',') { ++p; } else if (*p != '}') { fail(); }
            }
            ++p;
        } else if (*p == '[') {
            v.kind = jvalue::ARR;
            ++p;
            ws();
            while (*p != ']') {
                v.arr.push_back(value());
                ws();
                if (*p == ',') { ++p; } else if (*p != ']') { fail(); }
            }
            ++p;
        } else if (*p == '"') {
            v.kind = jvalue::STR;
            v.str = string();
        } else if (!strncmp(p, "true", 4) || !strncmp(p, "false", 5)) {
            v.kind = jvalue::BOOL;
            v.num = *p == 't';
            p += *p == 't' ? 4 : 5;
        } else if (!strncmp(p, "null", 4)) {
            p += 4;
        } else {
            char *end = nullptr;
            v.num = strtod(p, &end);
            if (end == p) { fail(); }
            v.kind = jvalue::NUM;
            p = end;
        }
        return v;
    }
};

inline void numbers_of(const jvalue *o, std::map<std::string, double> *out)
{
    if (!o || o->kind != jvalue::OBJ) { return; }
    for (const auto &kv : o->obj) {
        if (kv.second.kind == jvalue::NUM) { (*out)[kv.first] = kv.second.num; }
    }
}
}  // namespace detail

// Reads the autotuner's file; the entry of the scale nearest log2(n) (ties
// go to the larger scale), or the file's default entry.
inline tuning load_tuning(const std::string &path, long num_vertices)
{
    FILE *fp = fopen(path.c_str(), "rb");
    if (!fp) { throw error(BD_ERR_IO, "tuning file " + path); }
    std::string text;
    char buf[65536];
    size_t got;
    while ((got = fread(buf, 1, sizeof(buf), fp)) > 0) { text.append(buf, got); }
    fclose(fp);
    detail::jparser jp{text.c_str()};
    const detail::jvalue root = jp.value();
    const detail::jvalue *entry = &root;
    const detail::jvalue *by = root.get("by_scale");
    if (by && by->kind == detail::jvalue::OBJ && !by->obj.empty() && num_vertices > 0) {
        const double scale = std::log2((double)std::max(num_vertices, 2L));
        double best = 1e300;
        int best_key = 0;
        for (const auto &kv : by->obj) {
            const int key = atoi(kv.first.c_str());
            const double d = std::fabs(key - scale);
            if (d < best || (d == best && key > best_key)) {
                best = d;
                best_key = key;
                entry = &kv.second;
            }
        }
    }
    tuning t;
    detail::numbers_of(entry->get("single"), &t.single);
    detail::numbers_of(entry->get("batched"), &t.batched);
    return t;
}

// The graph (graph_base.h): a CSR in HBM.
class graph {
public:
    static graph from_el64(const std::string &path, int32_t order = BD_ORDER_INSERTION)
    {
        bd_graph *h = nullptr;
        throw_if(bd_graph_from_el64(path.c_str(), order, &h), "load_binary");
        return graph(h);
    }
    static graph rmat(int32_t scale, int64_t edge_factor = 16, uint64_t seed = 0,
                      double a = 0.57, double b = 0.19, double c = 0.19, double d = 0.05,
                      int32_t order = BD_ORDER_INSERTION)
    {
        bd_graph *h = nullptr;
        throw_if(bd_graph_rmat(scale, edge_factor, a, b, c, d, seed, order, &h), "rmat");
        return graph(h);
    }
    explicit graph(bd_graph *h) : h_(h) {}
    graph(graph &&o) noexcept : h_(std::exchange(o.h_, nullptr)) {}
    graph &operator=(graph &&o) noexcept
    {
        std::swap(h_, o.h_);
        return *this;
    }
    graph(const graph &) = delete;
    graph &operator=(const graph &) = delete;
    ~graph()
    {
        if (h_) { bd_graph_destroy(h_); }
    }

    long num_vertices() const
    {
        int64_t n = 0;
        throw_if(bd_graph_info(h_, &n, nullptr), "num_vertices");
        return (long)n;
    }
    long num_edges() const
    {
        int64_t m = 0;
        throw_if(bd_graph_info(h_, nullptr, &m), "num_edges");
        return (long)m;
    }
    // graph::check (graph_base.h:110-134)
    bool check() const
    {
        int32_t ok = 0;
        throw_if(bd_graph_check(h_, &ok), "check_graph");
        return ok != 0;
    }
    // hybrid_bfs::check (hybrid_bfs.cc:281-379) of any parent array (n entries,
    // the reference's encoding), on the device; *bad_vertex gets the lowest
    // failing vertex or -1.
    bool check_parents(int64_t source, const std::vector<int64_t> &parent,
                       int64_t *bad_vertex = nullptr) const
    {
        if ((long)parent.size() != num_vertices()) {
            throw error(BD_ERR_INVALID, "check_parents: parent array size");
        }
        int32_t ok = 0;
        int64_t bad = -1;
        throw_if(bd_graph_check_parents(h_, source, parent.data(), &ok, &bad), "check_parents");
        if (bad_vertex) { *bad_vertex = bad; }
        return ok != 0;
    }
    // pick_random_vertex with lcg(seed) (hybrid_bfs_main.cc:136-144)
    std::vector<int64_t> pick_roots(uint64_t seed, int64_t k) const
    {
        std::vector<int64_t> r(k);
        throw_if(bd_graph_pick_roots(h_, seed, k, r.data()), "pick_roots");
        return r;
    }
    void csr(std::vector<int64_t> &offsets, std::vector<uint32_t> &adjacency) const
    {
        offsets.resize(num_vertices() + 1);
        throw_if(bd_graph_copy_csr(h_, offsets.data(), nullptr), "csr");
        adjacency.resize(offsets.back());
        throw_if(bd_graph_copy_csr(h_, offsets.data(), adjacency.data()), "csr");
    }
    void write_el64(const std::string &path) const
    {
        throw_if(bd_graph_write_el64(h_, path.c_str()), "write_el64");
    }
    bd_graph *handle() const { return h_; }

private:
    bd_graph *h_ = nullptr;
};

namespace detail {
// hybrid_bfs::print_tree's text (hybrid_bfs.cc:381-399): for each vertex
// with a parent, the vertex and its ancestors up to the root,
// "%4li <- %4li <- ...".  A chain that meets a negative or out-of-range
// entry stops there (the reference would index with it); a chain that climbs
// n times without reaching a root is a cycle (the reference would loop
// forever), and its line ends with " <- (cycle)".
inline void print_tree(const std::vector<int64_t> &p, FILE *out)
{
    const long n = (long)p.size();
    for (long v = 0; v < n; ++v) {
        long parent = (long)p[v];
        if (parent < 0) { continue; }
        fprintf(out, "%4li", v);
        bool ended = false;
        for (long climb = 0; climb <= n && !ended; ++climb) {
            fprintf(out, " <- %4li", parent);
            if (parent < 0 || parent >= n || parent == p[parent]) {
                ended = true;
            } else {
                parent = (long)p[parent];
            }
        }
        if (!ended) { fprintf(out, " <- (cycle)"); }
        fprintf(out, "\n");
    }
    fflush(out);
}

// components::dump's text (components.cc:120-152): for each label in
// ascending order, "Component <label>: " and its vertices as ranges
// ("a-b" or "a"), comma separated, then a newline.  The reference ends a
// line only after a range that closed before the last vertex, so a label
// whose vertices form one range ending at vertex n-1 gets no newline (with
// minimum-id labels, that is the last line when vertex n-1's component is
// one contiguous run).  Labels must lie in [0, n).
inline void print_components(const std::vector<int64_t> &c, FILE *out)
{
    std::vector<std::vector<int64_t>> members(c.size());
    for (size_t v = 0; v < c.size(); ++v) { members[(size_t)c[v]].push_back((int64_t)v); }
    const int64_t last_vertex = (int64_t)c.size() - 1;
    for (size_t l = 0; l < members.size(); ++l) {
        const std::vector<int64_t> &m = members[l];
        if (m.empty()) { continue; }
        fprintf(out, "Component %zu: ", l);
        bool closed_early = false;  // a range ended before the last vertex
        for (size_t i = 0; i < m.size();) {
            size_t j = i;
            while (j + 1 < m.size() && m[j + 1] == m[j] + 1) { ++j; }
            if (i) { fprintf(out, ", "); }
            if (j == i) {
                fprintf(out, "%li", (long)m[i]);
            } else {
                fprintf(out, "%li-%li", (long)m[i], (long)m[j]);
            }
            if (m[j] != last_vertex) { closed_early = true; }
            i = j + 1;
        }
        if (closed_early) { fprintf(out, "\n"); }
    }
    fflush(out);
}
}  // namespace detail

// hybrid_bfs (hybrid_bfs.h:11-47).
class hybrid_bfs {
public:
    explicit hybrid_bfs(graph &g, const bd_bfs_opts *opts = nullptr) : g_(g)
    {
        throw_if(bd_bfs_create(g.handle(), opts, &h_), "hybrid_bfs");
    }
    hybrid_bfs(const hybrid_bfs &) = delete;
    hybrid_bfs &operator=(const hybrid_bfs &) = delete;
    ~hybrid_bfs()
    {
        if (h_) { bd_bfs_destroy(h_); }
    }

    void clear() { throw_if(bd_bfs_clear(h_), "clear"); }
    void run_beamer(long source, long alpha, long beta)
    {
        throw_if(bd_bfs_run_beamer(h_, source, alpha, beta, &stats_), "run_beamer");
    }
    void run_with_migrating_threads(long source)
    {
        throw_if(bd_bfs_run_top_down(h_, source, &stats_), "run_with_migrating_threads");
    }
    void run_with_remote_writes(long source)
    {
        throw_if(bd_bfs_run_top_down(h_, source, &stats_), "run_with_remote_writes");
    }
    void run_with_remote_writes_hybrid(long source, long alpha, long beta)
    {
        throw_if(bd_bfs_run_beamer(h_, source, alpha, beta, &stats_),
                 "run_with_remote_writes_hybrid");
    }
    void run_top_down(long source) { throw_if(bd_bfs_run_top_down(h_, source, &stats_), "top_down"); }
    void run_bottom_up(long source)
    {
        throw_if(bd_bfs_run_bottom_up(h_, source, &stats_), "bottom_up");
    }
    // Runs the policy the handle was created with (beamer / learned / ...).
    void run(long source) { throw_if(bd_bfs_run(h_, source, &stats_), "run"); }
    // The network BD_ALG_LEARNED consults (Beamer decides without one).
    void set_policy(const policy &p)
    {
        throw_if(bd_bfs_set_policy(h_, p.params.data(), p.mean.data(), p.inv_std.data(),
                                   p.lo.empty() ? nullptr : p.lo.data(),
                                   p.hi.empty() ? nullptr : p.hi.data(), p.margin),
                 "set_policy");
    }

    bool check(long source)
    {
        int32_t ok = 0;
        throw_if(bd_bfs_check(h_, source, &ok), "check");
        return ok != 0;
    }
    long count_num_traversed_edges()
    {
        int64_t m = 0;
        throw_if(bd_bfs_count_traversed_edges(h_, &m), "count_num_traversed_edges");
        return (long)m;
    }
    // print_tree (hybrid_bfs.cc:381-399)
    void print_tree() { detail::print_tree(parents(), stdout); }
    std::vector<int32_t> depths()
    {
        std::vector<int32_t> d(g_.num_vertices());
        throw_if(bd_bfs_get_depths(h_, d.data()), "depths");
        return d;
    }
    std::vector<int64_t> parents()
    {
        std::vector<int64_t> p(g_.num_vertices());
        throw_if(bd_bfs_get_parents(h_, p.data()), "parents");
        return p;
    }
    std::vector<bd_step> steps()
    {
        int64_t count = 0;
        throw_if(bd_bfs_get_steps(h_, nullptr, 0, &count), "steps");
        std::vector<bd_step> s(count);
        throw_if(bd_bfs_get_steps(h_, s.data(), count, &count), "steps");
        return s;
    }
    const bd_run_stats &last_stats() const { return stats_; }
    bd_bfs *handle() const { return h_; }

private:
    graph &g_;
    bd_bfs *h_ = nullptr;
    bd_run_stats stats_{};
};

// Many roots per pass over the graph (64 per group, all groups of a call as
// one captured CUDA graph).  Per root, the results read like hybrid_bfs's.
// No counterpart in the reference, whose driver runs its roots one by one
// (hybrid_bfs_main.cc:252-302).
class batched_bfs {
public:
    batched_bfs(graph &g, int32_t max_roots, const bd_msbfs_opts *opts = nullptr) : g_(g)
    {
        throw_if(bd_msbfs_create(g.handle(), max_roots, opts, &h_), "batched_bfs");
    }
    batched_bfs(const batched_bfs &) = delete;
    batched_bfs &operator=(const batched_bfs &) = delete;
    ~batched_bfs()
    {
        if (h_) { bd_msbfs_destroy(h_); }
    }
    void run(const std::vector<int64_t> &sources)
    {
        throw_if(bd_msbfs_run(h_, sources.data(), (int32_t)sources.size(), &stats_), "run");
    }
    void set_policy(const policy &p)
    {
        throw_if(bd_msbfs_set_policy(h_, p.params.data(), p.mean.data(), p.inv_std.data(),
                                     p.lo.empty() ? nullptr : p.lo.data(),
                                     p.hi.empty() ? nullptr : p.hi.data(), p.margin),
                 "set_policy");
    }
    long count_num_traversed_edges(int32_t i)
    {
        int64_t m = 0;
        throw_if(bd_msbfs_count_traversed_edges(h_, i, &m, nullptr), "count_num_traversed_edges");
        return (long)m;
    }
    std::vector<int32_t> depths(int32_t i)
    {
        std::vector<int32_t> d(g_.num_vertices());
        throw_if(bd_msbfs_get_depths(h_, i, d.data()), "depths");
        return d;
    }
    std::vector<int64_t> parents(int32_t i)
    {
        std::vector<int64_t> p(g_.num_vertices());
        throw_if(bd_msbfs_get_parents(h_, i, p.data()), "parents");
        return p;
    }
    // Root i's parent_ in device memory (opts.materialize handles only).
    const int64_t *device_parents(int32_t i)
    {
        const int64_t *p = nullptr;
        throw_if(bd_msbfs_device_results(h_, i, nullptr, &p), "device_parents");
        return p;
    }
    bool check(int32_t i)
    {
        int32_t ok = 0;
        throw_if(bd_msbfs_check(h_, i, &ok), "check");
        return ok != 0;
    }
    std::vector<bd_step> steps()
    {
        int64_t count = 0;
        throw_if(bd_msbfs_get_steps(h_, nullptr, 0, &count), "steps");
        std::vector<bd_step> s(count);
        throw_if(bd_msbfs_get_steps(h_, s.data(), count, &count), "steps");
        return s;
    }
    const bd_run_stats &last_stats() const { return stats_; }
    bd_msbfs *handle() const { return h_; }

private:
    graph &g_;
    bd_msbfs *h_ = nullptr;
    bd_run_stats stats_{};
};

// The reference's `components` class (components.h:6-33): run() labels
// every vertex with the smallest id of its component.
class components {
public:
    using stats = bd_components_stats;
    explicit components(graph &g) : g_(g)
    {
        throw_if(bd_components_create(g.handle(), &h_), "components");
    }
    components(const components &) = delete;
    components &operator=(const components &) = delete;
    ~components()
    {
        if (h_) { bd_components_destroy(h_); }
    }
    void clear() { throw_if(bd_components_clear(h_), "clear"); }
    stats run()
    {
        throw_if(bd_components_run(h_, &stats_), "run");
        return stats_;
    }
    bool check()
    {
        int32_t ok = 0;
        throw_if(bd_components_check(h_, &ok), "check");
        return ok != 0;
    }
    // component_ and component_size_ (components.h:13-15)
    std::vector<int64_t> component()
    {
        std::vector<int64_t> c(g_.num_vertices());
        throw_if(bd_components_get_labels(h_, c.data()), "component");
        return c;
    }
    std::vector<int64_t> component_size()
    {
        std::vector<int64_t> s(g_.num_vertices());
        throw_if(bd_components_get_sizes(h_, s.data()), "component_size");
        return s;
    }
    // components::dump (components.cc:120-152): per label, its vertices as ranges.
    void dump() { detail::print_components(component(), stdout); }
    const stats &last_stats() const { return stats_; }
    bd_components *handle() const { return h_; }

private:
    graph &g_;
    bd_components *h_ = nullptr;
    stats stats_{};
};

}  // namespace beedrill
