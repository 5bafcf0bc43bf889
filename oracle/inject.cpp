// ORACLE — test infrastructure only.
// A "variant body" for the reference's unchanged OpenMP harness (REF_HEADER):
// instead of computing, it loads the values to check from the raw int32 file
// named by $I2_RESULT. The harness's own main() then reads the graph, calls
// this body, and runs the reference's own verifier on those values, printing
// "verification passed" or exiting with an error. This lets the tests check
// any output (the GPU engine's or the oracle's) with the reference's checker.
#include <cstdio>
#include <cstdlib>
typedef int data_type;
#include REF_HEADER

static void i2_load(data_type* out, int n) {
  const char* path = std::getenv("I2_RESULT");
  FILE* f = path ? std::fopen(path, "rb") : nullptr;
  if (!f || std::fread(out, sizeof(data_type), n, f) != (size_t)n) {
    std::fprintf(stderr, "ERROR: cannot load I2_RESULT\n");
    std::exit(-2);
  }
  std::fclose(f);
}

#if defined(INJECT_BFS_VERTEX)
static double CPUbfs_vertex(const int, const ECLgraph& g, data_type* dist) { i2_load(dist, g.nodes); return 0.0; }
#elif defined(INJECT_SSSP_VERTEX)
static double CPUsssp_vertex(const int, const ECLgraph& g, data_type* dist) { i2_load(dist, g.nodes); return 0.0; }
#elif defined(INJECT_SSSP_EDGE)
static double CPUsssp_edge(const int, const ECLgraph& g, data_type* const dist, const int* const) { i2_load(dist, g.nodes); return 0.0; }
#elif defined(INJECT_CC_VERTEX)
static double CPUcc_vertex(const ECLgraph g, data_type* label) { i2_load(label, g.nodes); return 0.0; }
#endif
