// Persistent Newton-Raphson kernel (one CTA per lane tile); see persistent.cu.
#pragma once

#include "kernels.cuh"

namespace olfb200 {

// lanesPerTile in {1, 2, 4, 8}; threads <= 512 (a multiple of 32).
void launchPersistent(const DevNet& net, const DevBatch& b, const DevRl& rl, const Settings& cfg,
                      const PersistentPlan& plan, int lanesPerTile, int threads, bool fp32, cudaStream_t st);

}  // namespace olfb200
