// Shared part of the drop-in variant bodies in this directory.
//
// Each shim_*.cu file takes the place of one codes/cuda/<alg>-cuda/*.cu variant
// file of the Indigo2 suite: it defines the typedefs the harness expects,
// includes the unchanged harness header (include/<alg>_<kind>_cuda.h, which
// supplies main(), the ECLgraph reader, timing and the serial verifier) and
// implements the harness's GPU<alg>_<kind>() entry point on top of the C ABI
// of libi2b200 (include/i2b200.h). The harness passes the graph with device
// pointers (its d_g) and a host result array; the shim wraps the device arrays
// without copying them and returns the engine's device time in seconds. Only
// the SSSP harnesses upload the weights (include/sssp_vertex_cuda.h:122-125);
// in the BFS and CC harnesses d_g.eweight is still the host array from the file
// reader, so those shims pass no weights (MIS needs none).
//
// $I2_VARIANT selects the style: a variant name (vp_thread, vp_warp, vp_cta,
// vp_block, pull_frontier, pull_topo, edge_topo, push_topo), "heuristic"
// (default) or "learned"; $I2_LOOP=host selects the host-driven loop.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "i2b200.h"

static int i2shim_variant(int fallback) {
  const char* v = std::getenv("I2_VARIANT");
  if (!v || !*v) return fallback;
  if (!std::strcmp(v, "heuristic")) return I2_AUTO_HEURISTIC;
  if (!std::strcmp(v, "learned")) return I2_AUTO_LEARNED;
  for (int k = 0; k < I2_NUM_VARIANTS; ++k)
    if (!std::strcmp(v, i2_variant_name(k))) return k;
  return std::atoi(v);
}

static void i2shim_fail(const char* what, int st) {
  std::fprintf(stderr, "ERROR: i2b200 %s: %s\n", what, i2_status_string(st));
  std::exit(-1);
}

// algo: I2_BFS / I2_SSSP / I2_CC / I2_MIS. The CSR arrays in g are device pointers.
static double i2shim_run(int algo, int src, int nodes, int edges, int* nindex, int* nlist, int* eweight, int* out,
                         int fallback_variant) {
  i2_eclgraph d = {nodes, edges, nindex, nlist, eweight};
  i2_graph* h = nullptr;
  int st = i2_graph_wrap_device(&d, &h);
  if (st != I2_OK) i2shim_fail("graph", st);
  const char* loop = std::getenv("I2_LOOP");
  i2_opts o = {i2shim_variant(fallback_variant), (loop && !std::strcmp(loop, "host")) ? I2_LOOP_HOST : I2_LOOP_GRAPH,
               0, 0, nullptr};
  i2_report r;
  std::memset(&r, 0, sizeof(r));
  if (algo == I2_BFS) st = i2_bfs(h, src, out, &o, &r);
  else if (algo == I2_SSSP) st = i2_sssp(h, src, out, &o, &r);
  else if (algo == I2_CC) st = i2_cc(h, out, &o, &r);
  else st = i2_mis(h, out, &o, &r);
  i2_graph_free(h);
  if (st != I2_OK) i2shim_fail("run", st);
  std::printf("iterations: %d\n", r.iterations);
  return r.seconds;
}
