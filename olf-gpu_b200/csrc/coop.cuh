// Cooperative level sweeps (one launch per factorization / per solve); see coop.cu.
#pragma once

#include "kernels.cuh"

namespace olfb200 {

// The level structure of the factorization and of the two solves, on the device, with each level's split factor.
struct CoopPlan {
    int nLevels, nFwd, nBwd;
    const int* levelPtr;
    const int* levelSplit;
    const int* fwdPtr;
    const int* fwdPos;
    const int* fwdSplit;
    const int* bwdPtr;
    const int* bwdPos;
    const int* bwdSplit;
};

// Both return the launch's status (a cooperative launch that cannot have all its CTAs resident is refused, never
// run partially).
cudaError_t launchFactorCoop(const DevNet& net, const DevBatch& b, const CoopPlan& cp, bool fp32, cudaStream_t st);
cudaError_t launchSolveCoop(const DevNet& net, const DevBatch& b, const CoopPlan& cp, bool fp32, bool fromResidual,
                            cudaStream_t st);

}  // namespace olfb200
