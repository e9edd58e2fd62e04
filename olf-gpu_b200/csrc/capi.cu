// C ABI of the engine (declared in include/olfgpu_b200.h).  Every entry point catches every exception and reports
// it through olfgpu_last_error(), the way the reference's JNI layer turns native failures into RuntimeExceptions.
#include "../../include/olfgpu_b200.h"

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "engine.hpp"

using namespace olfb200;

namespace {

thread_local std::string lastError;

template <typename F>
int guarded(F&& f) {
    try {
        lastError.clear();
        f();
        return 0;
    } catch (const std::exception& e) {
        lastError = e.what();
    } catch (...) {
        lastError = "unknown native error";
    }
    return -1;
}

using StructurePtr = std::shared_ptr<NetStructure>;

StructurePtr& structureOf(int64_t h) {
    auto* p = reinterpret_cast<StructurePtr*>(h);
    if (!p || !*p) throw std::runtime_error("invalid structure handle");
    return *p;
}

BatchContext& contextOf(int64_t h) {
    auto* p = reinterpret_cast<BatchContext*>(h);
    if (!p) throw std::runtime_error("invalid batch solver context");
    return *p;
}

MultiContext& multiOf(int64_t h) {
    auto* p = reinterpret_cast<MultiContext*>(h);
    if (!p) throw std::runtime_error("invalid multi-grid context");
    return *p;
}

SolveRequest requestOf(const double* x0Base, const double* x0Full, const double* targetBase, const int* baseRowMode,
                       int nRowModeEntries, const int* rowModeEntries, int nScenarios, int nElements,
                       const unsigned char* disabled, int nTargetOverrides, const int* targetOverrideIndex,
                       const double* targetOverrideValue, int maxIter, double tol, double reactiveLimitTol,
                       int maxOuter, int maxPqPvSwitch) {
    if (nRowModeEntries < 0 || nTargetOverrides < 0 || nElements < 0) throw std::runtime_error("negative count");
    if ((nRowModeEntries && !rowModeEntries) || (nTargetOverrides && (!targetOverrideIndex || !targetOverrideValue))) {
        throw std::runtime_error("null array with a non-zero count");
    }
    SolveRequest r;
    r.x0Base = x0Base;
    r.x0Full = x0Full;
    r.targetBase = targetBase;
    r.baseRowMode = baseRowMode;
    r.nRowModeEntries = nRowModeEntries;
    r.rowModeEntries = rowModeEntries;
    r.nScenarios = nScenarios;
    r.nElements = nElements;
    r.disabled = disabled;
    r.nTargetOverrides = nTargetOverrides;
    r.targetOverrideIndex = targetOverrideIndex;
    r.targetOverrideValue = targetOverrideValue;
    r.maxIter = maxIter;
    r.tol = tol;
    r.reactiveLimitTol = reactiveLimitTol;
    r.maxOuter = maxOuter;
    r.maxPqPvSwitch = maxPqPvSwitch;
    return r;
}

}  // namespace

extern "C" const char* olfgpu_last_error(void) { return lastError.c_str(); }

extern "C" int olfgpu_create_structure(int n, int nCb, const double* cbParams, const int* cbIndices, int nOb,
                                       const double* obParams, const int* obIndices, int nSh, const double* shParams,
                                       const int* shIndices, int nIdentityRows, const int* identityRows, int ordering,
                                       int64_t* structureOut) {
    return guarded([&] {
        if (!structureOut) throw std::runtime_error("null output handle");
        *structureOut = 0;
        if ((nCb && (!cbParams || !cbIndices)) || (nOb && (!obParams || !obIndices)) || (nSh && (!shParams || !shIndices)) ||
            (nIdentityRows && !identityRows)) {
            throw std::runtime_error("null family array with a non-zero count");
        }
        auto s = std::make_shared<NetStructure>();
        s->host = buildStructure(n, nCb, cbParams, cbIndices, nOb, obParams, obIndices, nSh, shParams, shIndices,
                                 nIdentityRows, identityRows, ordering);
        *structureOut = reinterpret_cast<int64_t>(new StructurePtr(s));
    });
}

extern "C" int olfgpu_destroy_structure(int64_t structure) {
    return guarded([&] { delete reinterpret_cast<StructurePtr*>(structure); });
}

extern "C" int olfgpu_structure_info(int64_t structure, int* info, int64_t* blockOps) {
    return guarded([&] {
        const Structure& s = structureOf(structure)->host;
        const BlockPlan& p = s.plan;
        if (info) {
            info[0] = s.n;
            info[1] = s.nnz;
            info[2] = s.nb;
            info[3] = p.nU + p.nL;
            info[4] = static_cast<int>(p.levelPtr.size()) - 1;
            info[5] = static_cast<int>(p.fwdLevelPtr.size()) - 1;
            info[6] = static_cast<int>(p.bwdLevelPtr.size()) - 1;
            info[7] = s.nElements;
            info[8] = static_cast<int>(p.aCol.size());
        }
        if (blockOps) *blockOps = p.blockOps;
    });
}

extern "C" int olfgpu_structure_export(int64_t structure, int* rowMap, int* rowPtr, int* colIdx, int* diagPos,
                                       int* cbDest, int* obDest, int* shDest) {
    return guarded([&] {
        const Structure& s = structureOf(structure)->host;
        auto put = [](int* dst, const std::vector<int>& v) {
            if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(int));
        };
        put(rowMap, s.rowMap);
        put(rowPtr, s.rowPtr);
        put(colIdx, s.colIdx);
        put(diagPos, s.diagPos);
        put(cbDest, s.cbDest);
        put(obDest, s.obDest);
        put(shDest, s.shDest);
    });
}

extern "C" int olfgpu_structure_levels(int64_t structure, int* factorLevelPtr, int* forwardLevelPtr,
                                       int* backwardLevelPtr, int64_t* levelOps) {
    return guarded([&] {
        const BlockPlan& p = structureOf(structure)->host.plan;
        auto put = [](int* dst, const std::vector<int>& v) {
            if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(int));
        };
        put(factorLevelPtr, p.levelPtr);
        put(forwardLevelPtr, p.fwdLevelPtr);
        put(backwardLevelPtr, p.bwdLevelPtr);
        if (levelOps) {
            const int nl = static_cast<int>(p.levelPtr.size()) - 1;
            for (int l = 0; l < nl; l++) {
                int64_t ops = 0;
                for (int k = p.levelPtr[l]; k < p.levelPtr[l + 1]; k++) {
                    const int t = p.levelTask[k];
                    ops += p.opPtr[t + 1] - p.opPtr[t];
                }
                levelOps[l] = ops;
            }
        }
    });
}

extern "C" int olfgpu_recommend_batch_size(int64_t structure, int maxCap, int mode, int* batchOut) {
    return guarded([&] {
        if (!batchOut) throw std::runtime_error("null output");
        const Structure& s = structureOf(structure)->host;
        const BlockPlan& p = s.plan;
        // what one lane of a context takes: state vectors, the Jacobian, the factors in the mode's precision
        const double lu = static_cast<double>(p.nU + p.nL) * 4 * (mode == MODE_BATCHED_LU ? 8 + 4 : 8);
        const double perLane = 8.0 * s.n * 7 + s.n + static_cast<double>(p.aCol.size()) * 32 + lu + 8.0 * s.nb * 2 * 3;
        size_t freeB = 0, totalB = 0;
        OLF_CUDA(cudaMemGetInfo(&freeB, &totalB));
        const double budget = 0.7 * static_cast<double>(freeB);
        long fit = perLane > 0 ? static_cast<long>(budget / perLane) : maxCap;
        *batchOut = static_cast<int>(std::max<long>(1, std::min<long>(maxCap, fit)));
    });
}

extern "C" int olfgpu_create_batch_context(int64_t structure, int nScenarios, int mode, int nRl, const int* rlVoltageRow,
                                           const double* rlMinQ, const double* rlMaxQ, const double* rlLoadQ,
                                           const double* rlTargetV, const double* rlNomV, const int* rlPRow,
                                           const double* rlStaticP, const int* rlIdRank, int64_t* contextOut) {
    return guarded([&] {
        if (!contextOut) throw std::runtime_error("null output handle");
        *contextOut = 0;
        if (nRl < 0) throw std::runtime_error("negative reactive-limit entry count");
        if (nRl > 0 && (!rlVoltageRow || !rlMinQ || !rlMaxQ || !rlLoadQ || !rlTargetV || !rlNomV || !rlPRow ||
                        !rlStaticP || !rlIdRank)) {
            throw std::runtime_error("reactive-limit entries installed without their arrays or the forced-PV keys");
        }
        BatchContext* c = createContext(structureOf(structure), nScenarios, mode, nRl, rlVoltageRow, rlMinQ, rlMaxQ,
                                        rlLoadQ, rlTargetV, rlNomV, rlPRow, rlStaticP, rlIdRank);
        *contextOut = reinterpret_cast<int64_t>(c);
    });
}

extern "C" int olfgpu_destroy_batch_context(int64_t context) {
    return guarded([&] { delete reinterpret_cast<BatchContext*>(context); });
}

extern "C" int olfgpu_set_linear_solver_settings(int64_t context, int precision, int refinementSteps) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        if (precision != 0 && precision != 1) throw std::runtime_error("precision must be 0 (FP64) or 1 (mixed)");
        if (refinementSteps < 0 || refinementSteps > 8) throw std::runtime_error("refinementSteps must be in [0, 8]");
        c.precision = precision;
        c.refinementSteps = refinementSteps;
    });
}

extern "C" int olfgpu_set_schedule(int64_t context, int schedule, int lanesPerTile, int threads) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        if (schedule == -1) {
            c.autotunePending = true;
            return;
        }
        if (schedule != SCHEDULE_LEVELS && schedule != SCHEDULE_PERSISTENT && schedule != SCHEDULE_COOP &&
            schedule != SCHEDULE_LEVELS_SHARED && schedule != SCHEDULE_LEVELS_SHARED_ALL) {
            throw std::runtime_error("unknown schedule");
        }
        c.regionFactor = schedule == SCHEDULE_LEVELS_SHARED || schedule == SCHEDULE_LEVELS_SHARED_ALL;
        c.regionSolve = schedule == SCHEDULE_LEVELS_SHARED_ALL;
        if (c.regionFactor) schedule = SCHEDULE_LEVELS;
        if (schedule == SCHEDULE_COOP) {
            // cooperative sweeps have no tile parameters
        } else if (schedule == SCHEDULE_LEVELS) {
            if (lanesPerTile != 0 && lanesPerTile != 1 && lanesPerTile != 2 && lanesPerTile != 4) {
                throw std::runtime_error("level schedule: lanesPerTile of the narrow levels must be 0, 1, 2 or 4");
            }
            c.narrowLanes = lanesPerTile;
        } else {
            if (lanesPerTile != 1 && lanesPerTile != 2 && lanesPerTile != 4 && lanesPerTile != 8) {
                throw std::runtime_error("lanesPerTile must be 1, 2, 4 or 8");
            }
            if (threads != 256 && threads != 512) throw std::runtime_error("threads must be 256 or 512");
            c.lanesPerTile = lanesPerTile;
            c.threads = threads;
        }
        c.schedule = schedule;
        c.autotunePending = false;
    });
}

extern "C" int olfgpu_get_schedule(int64_t context, int* schedule, int* lanesPerTile, int* threads, int maxResults,
                                   double* results, int* nResults) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        if (schedule) {
            *schedule = c.schedule != SCHEDULE_LEVELS ? c.schedule
                        : c.regionSolve              ? SCHEDULE_LEVELS_SHARED_ALL
                        : c.regionFactor             ? SCHEDULE_LEVELS_SHARED
                                                     : SCHEDULE_LEVELS;
        }
        if (lanesPerTile) *lanesPerTile = c.schedule == SCHEDULE_LEVELS ? c.narrowLanes : c.lanesPerTile;
        // range kernels run 256 threads, as does the shared-memory factorization
        if (threads) *threads = c.schedule == SCHEDULE_LEVELS ? 256 : c.threads;
        const int k = std::min<int>(maxResults, static_cast<int>(c.tuning.size()));
        for (int i = 0; results && i < k; i++) {
            results[4 * i] = c.tuning[i].schedule;
            results[4 * i + 1] = c.tuning[i].lanesPerTile;
            results[4 * i + 2] = c.tuning[i].threads;
            results[4 * i + 3] = c.tuning[i].ms;
        }
        if (nResults) *nResults = static_cast<int>(c.tuning.size());
    });
}

extern "C" int olfgpu_solve_batch_context(int64_t context, const double* x0Base, const double* x0Full,
                                          const double* targetBase, const int* baseRowMode, int nRowModeEntries,
                                          const int* rowModeEntries, int nScenarios, int nElements,
                                          const unsigned char* disabled, int nTargetOverrides,
                                          const int* targetOverrideIndex, const double* targetOverrideValue,
                                          int maxIter, double tol, double reactiveLimitTol, int maxOuter,
                                          int maxPqPvSwitch, double* out) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        const SolveRequest r = requestOf(x0Base, x0Full, targetBase, baseRowMode, nRowModeEntries, rowModeEntries,
                                         nScenarios, nElements, disabled, nTargetOverrides, targetOverrideIndex,
                                         targetOverrideValue, maxIter, tol, reactiveLimitTol, maxOuter, maxPqPvSwitch);
        solveBatch(c, r, out);
    });
}

extern "C" int olfgpu_set_phase_timing(int64_t context, int enable) {
    return guarded([&] { contextOf(context).phaseTiming = enable != 0; });
}

extern "C" int olfgpu_last_phase_times(int64_t context, double* out8) {
    return guarded([&] {
        const BatchContext& c = contextOf(context);
        if (!out8) throw std::runtime_error("null output");
        for (int i = 0; i < 6; i++) out8[i] = c.phaseMs[i];
        out8[6] = static_cast<double>(c.phaseIterations);
        out8[7] = static_cast<double>(c.phaseLanes);
    });
}

extern "C" int olfgpu_set_mixed_precision_controls(int64_t context, double refineBelow, double growthLimit) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        if (!(refineBelow > 0)) throw std::runtime_error("refineBelow must be positive (infinity: every iteration)");
        if (!(growthLimit >= 1)) throw std::runtime_error("growthLimit must be >= 1 (infinity: never refactor)");
        c.refineBelow = refineBelow;
        c.growthLimit = growthLimit;
    });
}

extern "C" int olfgpu_last_fp64_refactors(int64_t context, unsigned char* flagged, int* count) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        std::vector<unsigned char> f(c.nS);
        OLF_CUDA(cudaSetDevice(c.device));
        OLF_CUDA(cudaMemcpy(f.data(), c.precision64.p, c.nS, cudaMemcpyDeviceToHost));
        int k = 0;
        for (int i = 0; i < c.nS; i++) k += f[i] ? 1 : 0;
        if (flagged) std::memcpy(flagged, f.data(), c.nS);
        if (count) *count = k;
    });
}

extern "C" int olfgpu_set_device_start(int64_t context, const double* x0FullDevice) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        if (x0FullDevice) {
            cudaPointerAttributes a{};
            OLF_CUDA(cudaPointerGetAttributes(&a, x0FullDevice));
            if (a.type != cudaMemoryTypeDevice || a.device != c.device) {
                throw std::runtime_error("x0FullDevice is not device memory of the context's GPU");
            }
        }
        c.deviceStart = x0FullDevice;
    });
}

extern "C" int olfgpu_set_fallback_start(int64_t context, int enable) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        if (enable && c.rl.nRl > 0) throw std::runtime_error("the fallback start is not available with reactive limits");
        c.fallbackStart = enable != 0;
    });
}

extern "C" int olfgpu_last_fallbacks(int64_t context, unsigned char* fellBack, int* count) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        std::vector<unsigned char> f(c.nS);
        OLF_CUDA(cudaSetDevice(c.device));
        OLF_CUDA(cudaMemcpy(f.data(), c.fellBack.p, c.nS, cudaMemcpyDeviceToHost));
        int k = 0;
        for (int i = 0; i < c.nS; i++) k += f[i] ? 1 : 0;
        if (fellBack) std::memcpy(fellBack, f.data(), c.nS);
        if (count) *count = k;
    });
}

extern "C" int olfgpu_stage_batch_context(int64_t context, const double* x0Base, const double* x0Full,
                                          const double* targetBase, const int* baseRowMode, int nRowModeEntries,
                                          const int* rowModeEntries, int nScenarios, int nElements,
                                          const unsigned char* disabled, int nTargetOverrides,
                                          const int* targetOverrideIndex, const double* targetOverrideValue,
                                          int maxIter, double tol, double reactiveLimitTol, int maxOuter,
                                          int maxPqPvSwitch) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        const SolveRequest r = requestOf(x0Base, x0Full, targetBase, baseRowMode, nRowModeEntries, rowModeEntries,
                                         nScenarios, nElements, disabled, nTargetOverrides, targetOverrideIndex,
                                         targetOverrideValue, maxIter, tol, reactiveLimitTol, maxOuter, maxPqPvSwitch);
        stageRequest(c, r);
    });
}

extern "C" int olfgpu_create_multi_context(int nContexts, const int64_t* contexts, int64_t* multiOut) {
    return guarded([&] {
        if (!multiOut) throw std::runtime_error("null output handle");
        *multiOut = 0;
        if (nContexts < 1 || !contexts) throw std::runtime_error("no batch contexts");
        std::vector<BatchContext*> members;
        for (int i = 0; i < nContexts; i++) members.push_back(&contextOf(contexts[i]));
        *multiOut = reinterpret_cast<int64_t>(createMultiContext(members));
    });
}

extern "C" int olfgpu_destroy_multi_context(int64_t multi) {
    return guarded([&] { delete reinterpret_cast<MultiContext*>(multi); });
}

extern "C" int olfgpu_set_multi_schedule(int64_t multi, int lanesPerTile, int threads, int order) {
    return guarded([&] {
        MultiContext& m = multiOf(multi);
        if (lanesPerTile == -1) {
            m.autotunePending = true;
            return;
        }
        if (lanesPerTile != 1 && lanesPerTile != 2 && lanesPerTile != 4 && lanesPerTile != 8) {
            throw std::runtime_error("lanesPerTile must be 1, 2, 4 or 8 (or -1: autotune)");
        }
        if (threads != 256 && threads != 512) throw std::runtime_error("threads must be 256 or 512");
        if (order != 0 && order != 1) throw std::runtime_error("order must be 0 (as given) or 1 (most buses first)");
        m.lanesPerTile = lanesPerTile;
        m.threads = threads;
        m.order = order;
        m.autotunePending = false;
    });
}

extern "C" int olfgpu_get_multi_schedule(int64_t multi, int* lanesPerTile, int* threads, int* order, int maxResults,
                                         double* results, int* nResults) {
    return guarded([&] {
        MultiContext& m = multiOf(multi);
        if (lanesPerTile) *lanesPerTile = m.lanesPerTile;
        if (threads) *threads = m.threads;
        if (order) *order = m.order;
        const int k = std::min<int>(maxResults, static_cast<int>(m.tuning.size()));
        for (int i = 0; results && i < k; i++) {
            results[4 * i] = m.tuning[i].lanesPerTile;
            results[4 * i + 1] = m.tuning[i].threads;
            results[4 * i + 2] = m.tuning[i].order;
            results[4 * i + 3] = m.tuning[i].ms;
        }
        if (nResults) *nResults = static_cast<int>(m.tuning.size());
    });
}

extern "C" int olfgpu_solve_multi_context(int64_t multi, double* const* outs, float* deviceMs) {
    return guarded([&] {
        MultiContext& m = multiOf(multi);
        solveMulti(m, outs);
        if (deviceMs) *deviceMs = m.lastMs;
    });
}

extern "C" int olfgpu_last_solve_stats(int64_t context, float* deviceMs, int* batchedIterations, int* totalIterations) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        if (deviceMs) *deviceMs = c.lastMs;
        if (batchedIterations) *batchedIterations = c.lastIterations;
        if (totalIterations) {
            OLF_CUDA(cudaMemcpy(totalIterations, c.totalIter.p, sizeof(int) * c.nS, cudaMemcpyDeviceToHost));
        }
    });
}

extern "C" int olfgpu_debug_fill(int64_t context, const double* xFull, const double* targetBase, const int* baseRowMode,
                                 const unsigned char* disabled, double* jacobianOut, double* mismatchOut) {
    return guarded([&] {
        debugFill(contextOf(context), xFull, targetBase, baseRowMode, disabled, jacobianOut, mismatchOut);
    });
}

extern "C" int olfgpu_debug_linear_solve(int64_t context, const double* csrVals, const double* rhs, int precision,
                                         double* out) {
    return guarded([&] { debugLinearSolve(contextOf(context), csrVals, rhs, precision, out); });
}

namespace olfb200 {
void linearSolveNoAlloc(const std::shared_ptr<NetStructure>& net, int nScenarios, const double* csrVals,
                        const double* rhs, double* out, int precision, cudaStream_t st);
}

extern "C" int olfgpu_linear_solve_noalloc(int64_t structure, int nScenarios, const double* csrValsDevice,
                                           const double* rhsDevice, double* outDevice, int precision, void* stream) {
    return guarded([&] {
        linearSolveNoAlloc(structureOf(structure), nScenarios, csrValsDevice, rhsDevice, outDevice, precision,
                           static_cast<cudaStream_t>(stream));
    });
}
