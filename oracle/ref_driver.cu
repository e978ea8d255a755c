// ref_driver.cu -- TEST INFRASTRUCTURE. Drives the reference's own CUDA pipeline
// (ModularityAlgorithms::Louvain, modularityAlgorithms.h:8-10) on one input and writes
// its result, so golden vectors come from the reference itself. Built by `make ref` from
// the reference's unmodified sources (see Makefile); never linked into the product.
//
// usage: ref_louvain <input> <SORT|HASH> <out.bin> [edges|csr]
//   edges : text edge list parsed by the reference's GraphHost (graph.cu:17-87)
//   csr   : binary CSR (int64 n, int64 E, int64 row_ptr[n+1], int32 col[E]) loaded
//           straight into GraphHost's fields, skipping the std::set parser for large
//           graphs; the parser runs outside the reference's timed window either way.
// out.bin: uint32 n0, uint32 n_of_best_communities, double modularity,
//          float elapsed_ms (the reference's own cudaEvent window), uint32 best[n0]
#include "modularityAlgorithms.h"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

static bool load_csr(const char* path, GraphHost& g) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  int64_t n = 0, E = 0;
  if (std::fread(&n, 8, 1, f) != 1 || std::fread(&E, 8, 1, f) != 1) { std::fclose(f); return false; }
  std::vector<int64_t> row(n + 1);
  std::vector<int32_t> col(E);
  bool ok = std::fread(row.data(), 8, n + 1, f) == (size_t)(n + 1) &&
            std::fread(col.data(), 4, E, f) == (size_t)E;
  std::fclose(f);
  if (!ok) return false;
  g.n_nodes = (unsigned)n;
  g.n_links = (unsigned long)(E / 2);
  g.total_weight = (double)(E / 2);
  g.min_id = 0;
  g.edge_source = thrust::host_vector<unsigned int>(E);
  g.edge_destination = thrust::host_vector<unsigned int>(E);
  g.weights = thrust::host_vector<unsigned>(E);
  for (int64_t v = 0; v < n; v++)
    for (int64_t e = row[v]; e < row[v + 1]; e++) {
      g.edge_source[e] = (unsigned)v;
      g.edge_destination[e] = (unsigned)col[e];
      g.weights[e] = 1;
    }
  return true;
}

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s <input> <SORT|HASH> <out.bin> [edges|csr]\n", argv[0]);
    return 2;
  }
  const std::string mode_s = argv[2];
  MODE mode = mode_s == "HASH" ? HASH : SORT;
  const bool csr = argc > 4 && std::string(argv[4]) == "csr";
  std::string input = argv[1];
  std::string stub;
  if (csr) {
    // GraphHost's only constructor parses a file; give it a one-edge stub and then
    // replace every field with the binary CSR.
    stub = std::string(argv[3]) + ".stub.edge";
    std::ofstream(stub) << "0 1\n";
    input = stub;
  }
  GraphHost g(input, false, 0);
  if (csr && !load_csr(argv[1], g)) {
    std::fprintf(stderr, "cannot read %s\n", argv[1]);
    return 3;
  }
  if (csr) std::remove(stub.c_str());

  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventRecord(t0);
  Community C = ModularityAlgorithms::Louvain(g, mode);
  cudaEventRecord(t1);
  cudaEventSynchronize(t1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    std::fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(err));
    return 4;
  }
  thrust::host_vector<unsigned> best = C.best_communities;
  FILE* f = std::fopen(argv[3], "wb");
  if (!f) return 5;
  unsigned n0 = (unsigned)best.size();
  unsigned nb = C.n_of_best_communities;
  double q = C.modularity;
  std::fwrite(&n0, 4, 1, f);
  std::fwrite(&nb, 4, 1, f);
  std::fwrite(&q, 8, 1, f);
  std::fwrite(&ms, 4, 1, f);
  std::fwrite(best.data(), 4, n0, f);
  std::fclose(f);
  std::printf("RESULT n0=%u n_best=%u Q=%.17g ms_total=%.3f\n", n0, nb, q, ms);
  return 0;
}
