// louvain_b200.hpp -- C++ drop-in for the reference's host API, over the C ABI in louvain_b200.h.
//
// The reference's callers write (main.cu:16-33):
//     GraphHost g("graph.edge", false, 0);
//     Community C = ModularityAlgorithms::Louvain(g, SORT);
//     C.n_of_best_communities; C.modularity; C.best_communities;
// Including this header instead of modularityAlgorithms.h keeps that code compiling and
// running on the B200 engine: same names, same argument meaning, same result fields
// (graphHost.cuh:7-18, community.h:15-26, modularityAlgorithms.h:7-82, constants.h:13).
// Differences a caller can see: best_communities is a host std::vector (the reference keeps a
// thrust::device_vector), and failures throw louvain::Error with the engine's message instead
// of exiting the process (graph.cu:52-55) or surfacing as std::bad_alloc.
//
// Define LOUVAIN_B200_NO_GLOBAL_NAMES to keep everything inside namespace louvain.
#pragma once

#include <algorithm>
#include <cstdint>
#include <fstream>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "louvain_b200.h"

namespace louvain {

enum MODE { HASH = LV_MODE_HASH, SORT = LV_MODE_SORT, ADAPTIVE_SPEED = LV_MODE_ADAPTIVE_SPEED,
            ADAPTIVE_MEMORY = LV_MODE_ADAPTIVE_MEMORY };

struct Error : std::runtime_error {
  lv_status status;
  Error(lv_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

// graphHost.cuh:7-18 / graph.cu:17-87: reads `a b` pairs after `skip_line` header lines,
// keeps each undirected pair once, emits both directions with weight 1, shifts IDs by the
// smallest one. The CSR form the engine consumes is built alongside.
struct GraphHost {
  unsigned int n_nodes = 0;
  unsigned long n_links = 0;
  double total_weight = 0;
  unsigned int min_id = 0;
  std::vector<unsigned int> edge_source, edge_destination;
  std::vector<unsigned> weights;
  std::vector<int64_t> row_ptr;  // CSR of the symmetric graph (IDs shifted by min_id)
  std::vector<int32_t> col;

  GraphHost(const std::string& name, bool weighted, int skip_line) {
    if (weighted) throw Error(LV_ERR_ARGUMENT, "weighted edge lists are not parsed (graph.cu:32-34)");
    std::ifstream f(name);
    if (!f) throw Error(LV_ERR_ARGUMENT, "cannot open " + name);
    std::string ignore;
    for (int i = 0; i < skip_line; i++) std::getline(f, ignore);
    std::set<int> nodes;
    std::set<std::pair<int, int>> edges;
    int a, b;
    while (f >> a >> b) {
      nodes.insert(a);
      nodes.insert(b);
      edges.insert(a > b ? std::make_pair(b, a) : std::make_pair(a, b));
    }
    if (nodes.empty()) throw Error(LV_ERR_INPUT, "Error during parsing: no node found");
    n_links = edges.size();
    n_nodes = (unsigned)nodes.size();
    min_id = (unsigned)*nodes.begin();
    if ((long long)*nodes.rbegin() - (long long)min_id + 1 != (long long)n_nodes)
      throw Error(LV_ERR_INPUT, "vertex IDs must be contiguous (the reference indexes by id - min_id)");
    total_weight = (double)n_links;
    edge_source.reserve(2 * n_links);
    edge_destination.reserve(2 * n_links);
    std::vector<int64_t> deg(n_nodes + 1, 0);
    for (const auto& e : edges) {  // both directions, a self-loop pair included (graph.cu:68-79)
      const unsigned u = (unsigned)e.first - min_id, v = (unsigned)e.second - min_id;
      edge_source.push_back(u); edge_destination.push_back(v);
      edge_source.push_back(v); edge_destination.push_back(u);
      deg[u + 1]++;
      deg[v + 1]++;
    }
    weights.assign(edge_source.size(), 1u);
    // CSR of exactly those entries, rows sorted by destination as GraphDevice's
    // sort_by_key leaves them (graph.cuh:60-64)
    row_ptr.assign(n_nodes + 1, 0);
    for (unsigned i = 0; i < n_nodes; i++) row_ptr[i + 1] = row_ptr[i] + deg[i + 1];
    col.assign((size_t)row_ptr[n_nodes], 0);
    std::vector<int64_t> cur(row_ptr.begin(), row_ptr.end() - 1);
    for (size_t i = 0; i < edge_source.size(); i++)
      col[(size_t)cur[edge_source[i]]++] = (int32_t)edge_destination[i];
    for (unsigned i = 0; i < n_nodes; i++)
      std::sort(col.begin() + row_ptr[i], col.begin() + row_ptr[i + 1]);
  }

  // A graph already in symmetric CSR form (unit weights).
  GraphHost(std::vector<int64_t> rp, std::vector<int32_t> c)
      : row_ptr(std::move(rp)), col(std::move(c)) {
    n_nodes = (unsigned)(row_ptr.size() - 1);
    n_links = (unsigned long)(col.size() / 2);
    total_weight = (double)n_links;
  }
};

// community.h:15-26: the fields a caller reads after a run.
struct Community {
  std::vector<unsigned int> best_communities;
  unsigned int n_of_best_communities = 0;
  double modularity = -0.5;
  lv_stats stats{};
};

class Engine {
 public:
  explicit Engine(MODE mode, int device = 0, double threshold = 0.001) {
    lv_config c;
    lv_config_default(&c);
    c.mode = (int32_t)mode;
    c.threshold = threshold;
    lv_context* ctx = nullptr;
    const lv_status s = lv_create(device, &c, &ctx);
    if (s != LV_OK) throw Error(s, std::string("lv_create: ") + lv_status_string(s));
    ctx_.reset(ctx);
  }
  // Any configuration (e.g. refine = 1 for the Leiden-style refinement); start from
  // lv_config_default.
  explicit Engine(const lv_config& cfg, int device = 0) {
    lv_context* ctx = nullptr;
    const lv_status s = lv_create(device, &cfg, &ctx);
    if (s != LV_OK) throw Error(s, std::string("lv_create: ") + lv_status_string(s));
    ctx_.reset(ctx);
  }
  Community run(const GraphHost& g) {
    Community C;
    std::vector<int32_t> out(g.n_nodes);
    double q = 0;
    const lv_status s = lv_run_csr(ctx_.get(), g.n_nodes, g.row_ptr.data(), g.col.data(), nullptr,
                                   LV_MEM_HOST, out.data(), LV_MEM_HOST, &q, &C.stats);
    if (s != LV_OK) throw Error(s, lv_last_error(ctx_.get()));
    C.best_communities.assign(out.begin(), out.end());
    C.n_of_best_communities = (unsigned)C.stats.n_communities;
    C.modularity = q;
    return C;
  }

 private:
  struct Del {
    void operator()(lv_context* c) const { lv_destroy(c); }
  };
  std::unique_ptr<lv_context, Del> ctx_;
};

// modularityAlgorithms.h:7-82
struct ModularityAlgorithms {
  static Community Louvain(GraphHost& graph, MODE fastLocalMoveEnable) {
    Engine e(fastLocalMoveEnable);
    return e.run(graph);
  }
};

}  // namespace louvain

#ifndef LOUVAIN_B200_NO_GLOBAL_NAMES
using louvain::ADAPTIVE_MEMORY;
using louvain::ADAPTIVE_SPEED;
using louvain::Community;
using louvain::GraphHost;
using louvain::HASH;
using louvain::MODE;
using louvain::ModularityAlgorithms;
using louvain::SORT;
#endif
