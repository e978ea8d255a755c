// A caller written against the reference's own API (main.cu:16-33), compiled against
// include/louvain_b200.hpp and linked with liblouvain_b200.so. Used by the GPU tests.
//
// usage: facade_main <edge list> <SORT|HASH> <out.bin>
// prints "<n_of_best_communities> <modularity>" and writes best_communities (u32) to out.bin
#include <cstdio>
#include <string>

#include "louvain_b200.hpp"

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s <edge list> <SORT|HASH> <out.bin>\n", argv[0]);
    return 2;
  }
  try {
    GraphHost g(argv[1], false, 0);
    Community C = ModularityAlgorithms::Louvain(g, std::string(argv[2]) == "HASH" ? HASH : SORT);
    std::printf("%u %.17g\n", C.n_of_best_communities, C.modularity);
    std::FILE* f = std::fopen(argv[3], "wb");
    if (!f) return 3;
    std::fwrite(C.best_communities.data(), 4, C.best_communities.size(), f);
    std::fclose(f);
  } catch (const louvain::Error& e) {
    std::fprintf(stderr, "louvain error %d: %s\n", (int)e.status, e.what());
    return 1;
  }
  return 0;
}
