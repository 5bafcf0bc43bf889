// Resident traversal kernels: relax_resident<ALG, style> runs every iteration
// of a traversal in one cooperative launch (relax.cuh). They are instantiated
// in a translation unit of their own so that they compile in parallel with
// engine.cu.
#include "engine.h"
#include "mlp.cuh"
#include "relax.cuh"
#include "iteration.cuh"

namespace i2 {

template <int ALG>
static KernelFn resident_fn(int v, bool wide) {
  switch (v) {
    case kVPThread: return relax_resident<ALG, kVPThread>;
    case kVPWarp: return relax_resident<ALG, kVPWarp>;
    case kVPCta: return relax_resident<ALG, kVPCta>;
    case kVPBlock: return relax_resident<ALG, kVPBlock>;
    case kPullFrontier: return relax_resident<ALG, kPullFrontier>;
    case kPullTopo: return relax_resident<ALG, kPullTopo>;
    case kEdgeTopo: return relax_resident<ALG, kEdgeTopo>;
    case kPushTopo: return relax_resident<ALG, kPushTopo>;
    case kUnionFind:
      if constexpr (ALG == kCC) return relax_resident<ALG, kUnionFind>;
      return nullptr;
  }
  // per-iteration pick
  return wide ? relax_resident<ALG, -1, false, I2_EB_MIN_BLOCKS> : relax_resident<ALG, -1>;
}

// Kernel of a resident traversal: fixed style v (mode 0) or the per-iteration
// pick (v < 0; `wide`: the form compiled for more resident blocks).
KernelFn resident_kernel(int algo, int v, bool near_far, bool wide) {
  if (algo == kMIS) return relax_resident<kMIS, kVPWarp>;  // one style
  if (near_far && algo == kSSSP && v == kVPCta) return relax_resident<kSSSP, kVPCta, true>;
  if (algo == kBFS) return resident_fn<kBFS>(v, wide);
  if (algo == kSSSP) return resident_fn<kSSSP>(v, wide);
  return resident_fn<kCC>(v, wide);
}

}  // namespace i2
