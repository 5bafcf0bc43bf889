// ORACLE — test infrastructure only.
// The harness headers declare the variant's host driver and call it from main();
// ref_serial.cpp only needs the serial checker, so it defines an unused body.
#if defined(REF_STUB_BFS_VERTEX)
static double CPUbfs_vertex(const int, const ECLgraph&, data_type*) { return 0.0; }
#elif defined(REF_STUB_SSSP_VERTEX)
static double CPUsssp_vertex(const int, const ECLgraph&, data_type*) { return 0.0; }
#elif defined(REF_STUB_SSSP_EDGE)
static double CPUsssp_edge(const int, const ECLgraph&, data_type* const, const int* const) { return 0.0; }
#endif
