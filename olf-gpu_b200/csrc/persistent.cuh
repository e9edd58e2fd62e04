// Persistent Newton-Raphson kernel (one CTA per lane tile); see persistent.cu.
#pragma once

#include "kernels.cuh"

namespace olfb200 {

// One grid's batch inside a multi-grid launch: its network, lanes, settings, plan and first CTA index.
struct MultiItem {
    DevNet net;
    DevBatch b;
    DevRl rl;
    Settings cfg;
    PersistentPlan plan;
    int tileBegin;
};

// One persistent launch over nItems grids (itemsDevice in device memory, tileBegin ascending, totalTiles CTAs).
void launchMulti(const MultiItem* itemsDevice, int nItems, int totalTiles, int lanesPerTile, int threads, bool fp32,
                 cudaStream_t st);

// lanesPerTile in {1, 2, 4, 8}; threads <= 512 (a multiple of 32).
void launchPersistent(const DevNet& net, const DevBatch& b, const DevRl& rl, const Settings& cfg,
                      const PersistentPlan& plan, int lanesPerTile, int threads, bool fp32, cudaStream_t st);

}  // namespace olfb200
