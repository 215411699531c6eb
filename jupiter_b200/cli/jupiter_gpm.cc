// jupiter_gpm -- command-line front end over libjgpm's C-ABI.
//
// Mirrors the reference CLI (src/main.cc:7-47): `jupiter_gpm <graph_prefix> [pattern(P1)]
// [rounds(1)]`, loading the reference's on-disk CSR, orienting it for the clique patterns
// P13..P16 (src/main.cc:29-33) and printing the reference's result line
// `gpu count:<n>  runtime:<s>s` (src/jupiter_gpm.cu:908).  Extra, optional flags:
//   --induced        vertex-induced counts for the 4-vertex patterns
//   --stats          also print the canonical plan's set-op elements
//   --device <id>    GPU to use
// Errors print jgpm_last_error() and exit with status 1 (the library itself never exits).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "jgpm.h"

static int fail(const char* what, int rc) {
  std::fprintf(stderr, "jupiter_gpm: %s failed (status %d): %s\n", what, rc, jgpm_last_error());
  return 1;
}

int main(int argc, char** argv) {
  std::string prefix, pattern = "P1";
  int rounds = 1, induced = 0, device = 0, positional = 0;
  unsigned flags = 0;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a == "--induced") induced = 1;
    else if (a == "--stats") flags |= JGPM_COUNT_STATS;
    else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
    else if (positional == 0) { prefix = a; ++positional; }
    else if (positional == 1) { pattern = a; ++positional; }
    else if (positional == 2) { rounds = std::atoi(a.c_str()); ++positional; }
  }
  if (prefix.empty()) {
    std::printf("Usage: %s <graph> [pattern(P1)] [round(1)] [--induced] [--stats] [--device d]\n",
                argv[0]);
    std::printf("Example: %s /graph_inputs/mico/graph P1\n", argv[0]);
    return 1;
  }
  int rc = jgpm_set_device(device);
  if (rc) return fail("jgpm_set_device", rc);
  const bool use_dag = pattern == "P13" || pattern == "P14" || pattern == "P15" ||
                       pattern == "P16";
  jgpm_graph* g = nullptr;
  rc = jgpm_graph_load(prefix.c_str(), use_dag ? 1 : 0, &g);
  if (rc) return fail("jgpm_graph_load", rc);
  jgpm_graph_info info;
  jgpm_graph_get_info(g, &info);
  std::printf("|V| %d |E| %lld max degree %d\n", info.num_vertices, (long long)info.num_arcs,
              info.max_degree);
  uint64_t count = 0;
  jgpm_stats st;
  std::memset(&st, 0, sizeof(st));
  rc = jgpm_count_ex(g, pattern.c_str(), induced, rounds, flags, &count, &st);
  if (rc) {
    jgpm_graph_free(g);
    return fail("jgpm_count", rc);
  }
  std::printf("=====================gpu count:%llu  runtime:%.6fs\n", (unsigned long long)count,
              st.kernel_ms / 1e3);
  if (flags & JGPM_COUNT_STATS)
    std::printf("set-op elements:%llu\n", (unsigned long long)st.setop_elements);
  jgpm_graph_free(g);
  return 0;
}
