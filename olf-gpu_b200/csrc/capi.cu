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

extern "C" int olfgpu_create_structure_full(
    int n, const double* cbParams, int cbParamsLength, const int* cbIndices, int cbIndicesLength,
    const double* obParams, int obParamsLength, const int* obIndices, int obIndicesLength, const double* shParams,
    int shParamsLength, const int* shIndices, int shIndicesLength, const double* hvdcParams, int hvdcParamsLength,
    const int* hvdcIndices, int hvdcIndicesLength, const int* distrQElement, int distrQElementLength,
    const int* distrQSide, int distrQSideLength, const double* distrQWeight, int distrQWeightLength,
    const int* distrQRow, int distrQRowLength, const int* distrQKind, int distrQKindLength, const double* zibParams,
    int zibParamsLength, const int* zibIndices, int zibIndicesLength, const int* distrRhoRow, int distrRhoRowLength,
    const int* distrRhoColumn, int distrRhoColumnLength, const double* distrRhoCoefficient,
    int distrRhoCoefficientLength, const int* distrShuntBRow, int distrShuntBRowLength, const int* distrShuntBColumn,
    int distrShuntBColumnLength, const double* distrShuntBCoefficient, int distrShuntBCoefficientLength,
    const int* cbPhaseControlSide, int cbPhaseControlSideLength, const double* loadModelParams,
    int loadModelParamsLength, const int* loadModelIndices, int loadModelIndicesLength,
    const int* reactiveRelocationGroupStart, int reactiveRelocationGroupStartLength,
    const int* reactiveRelocationCandidateRows, int reactiveRelocationCandidateRowsLength,
    const int* obAlternateReactiveDestination, int obAlternateReactiveDestinationLength,
    const int* zibAlternateReactiveDestination, int zibAlternateReactiveDestinationLength,
    const int* reactiveRelocationDependentBaseGroup, int reactiveRelocationDependentBaseGroupLength,
    const int* reactiveRelocationBaseTargetRow, int reactiveRelocationBaseTargetRowLength,
    const int* reactiveRelocationDependentGroupOfRow, int reactiveRelocationDependentGroupOfRowLength,
    const int* identityRows, int identityRowsLength, int ordering, int64_t* structureOut) {
    return guarded([&] {
        if (!structureOut) throw std::runtime_error("null output handle");
        *structureOut = 0;
        // element counts from the index strides (structure_jni.cu:55-63)
        const int nCb = cbIndicesLength / 12, nOb = obIndicesLength / 6, nSh = shIndicesLength / 5;
        if (cbIndicesLength % 12 || cbParamsLength != nCb * 8) throw std::runtime_error("closed-branch arrays: bad lengths");
        if (obIndicesLength % 6 || obParamsLength != nOb * 7) throw std::runtime_error("open-branch arrays: bad lengths");
        if (shIndicesLength % 5 || shParamsLength != nSh * 2) throw std::runtime_error("shunt arrays: bad lengths");
        (void)hvdcParams; (void)hvdcIndices; (void)distrQElement; (void)distrQSide; (void)distrQWeight; (void)distrQRow;
        (void)distrQKind; (void)zibParams; (void)zibIndices; (void)distrRhoRow; (void)distrRhoColumn;
        (void)distrRhoCoefficient; (void)distrShuntBRow; (void)distrShuntBColumn; (void)distrShuntBCoefficient;
        (void)loadModelParams; (void)loadModelIndices; (void)reactiveRelocationCandidateRows;
        (void)zibAlternateReactiveDestination;
        const std::pair<const char*, int> empty[] = {
            {"hvdcAcEmulationParameters", hvdcParamsLength}, {"hvdcAcEmulationIndices", hvdcIndicesLength},
            {"distrQElement", distrQElementLength}, {"distrQSide", distrQSideLength},
            {"distrQWeight", distrQWeightLength}, {"distrQRow", distrQRowLength}, {"distrQKind", distrQKindLength},
            {"zeroImpedanceBranchParameters", zibParamsLength}, {"zeroImpedanceBranchIndices", zibIndicesLength},
            {"distrRhoRow", distrRhoRowLength}, {"distrRhoColumn", distrRhoColumnLength},
            {"distrRhoCoefficient", distrRhoCoefficientLength}, {"distrShuntBRow", distrShuntBRowLength},
            {"distrShuntBColumn", distrShuntBColumnLength}, {"distrShuntBCoefficient", distrShuntBCoefficientLength},
            {"loadModelParameters", loadModelParamsLength}, {"loadModelIndices", loadModelIndicesLength},
            {"reactiveRelocationCandidateRows", reactiveRelocationCandidateRowsLength},
            {"zeroImpedanceBranchAlternateReactiveDestination", zibAlternateReactiveDestinationLength},
        };
        for (const auto& e : empty) {
            if (e.second != 0) {
                throw std::runtime_error(std::string("createStructure: ") + e.first +
                                         " is not supported by this engine (pass null or an empty array)");
            }
        }
        // arrays that may carry "none" entries: every entry must say none
        auto allNone = [](const char* what, const int* a, int len) {
            for (int k = 0; k < len; k++) {
                if (a[k] != -1) {
                    throw std::runtime_error(std::string("createStructure: ") + what + " holds an entry (" +
                                             std::to_string(a[k]) + " at " + std::to_string(k) +
                                             "): not supported by this engine");
                }
            }
        };
        allNone("closedBranchPhaseControlSide", cbPhaseControlSide, cbPhaseControlSideLength);
        allNone("openBranchAlternateReactiveDestination", obAlternateReactiveDestination,
                obAlternateReactiveDestinationLength);
        allNone("reactiveRelocationDependentBaseGroup", reactiveRelocationDependentBaseGroup,
                reactiveRelocationDependentBaseGroupLength);
        allNone("reactiveRelocationBaseTargetRow", reactiveRelocationBaseTargetRow, reactiveRelocationBaseTargetRowLength);
        allNone("reactiveRelocationDependentGroupOfRow", reactiveRelocationDependentGroupOfRow,
                reactiveRelocationDependentGroupOfRowLength);
        // reactiveRelocationGroupStart = [0] (or empty) when there is no relocation group
        if (reactiveRelocationGroupStartLength > 1 ||
            (reactiveRelocationGroupStartLength == 1 && reactiveRelocationGroupStart[0] != 0)) {
            throw std::runtime_error("createStructure: reactive relocation groups are not supported by this engine");
        }
        auto s = std::make_shared<NetStructure>();
        s->host = buildStructure(n, nCb, cbParams, cbIndices, nOb, obParams, obIndices, nSh, shParams, shIndices,
                                 identityRowsLength, identityRows, ordering);
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

extern "C" int olfgpu_structure_check_plan(int64_t structure, int plantedFault, int64_t* violations,
                                           char* firstViolation, int capacity) {
    return guarded([&] {
        if (plantedFault < 0 || plantedFault > 3) throw std::runtime_error("plantedFault must be 0..3");
        if (!violations) throw std::runtime_error("null output");
        std::string first;
        *violations = checkBlockPlan(structureOf(structure)->host.plan, plantedFault, first);
        if (firstViolation && capacity > 0) {
            const size_t k = std::min(first.size(), static_cast<size_t>(capacity - 1));
            std::memcpy(firstViolation, first.data(), k);
            firstViolation[k] = 0;
        }
    });
}

extern "C" int olfgpu_structure_subtrees(int64_t structure, int64_t* stats6) {
    return guarded([&] {
        const BlockPlan& p = structureOf(structure)->host.plan;
        const NarrowBounds nbd = binBounds(p);
        const SubtreeBinsHost h = planSubtreeBins(p, nbd);
        const std::string err = checkSubtreeBins(p, nbd, h);
        if (!err.empty()) throw std::runtime_error("subtree bins: " + err);
        if (stats6) {
            int maxLevels = 0;
            for (int b = 0; b < h.nBins; b++) maxLevels = std::max(maxLevels, h.levPtr[b + 1] - h.levPtr[b]);
            int topWide = 0;
            for (int l = 0; l < nbd.factorFrom; l++) topWide += h.topLevelPtr[l + 1] - h.topLevelPtr[l];
            int binPos = 0;
            for (int v : h.bwdBinOf) binPos += v >= 0;
            stats6[0] = h.nBins * 100 + static_cast<int>(h.phasePtr.size()) - 1;
            stats6[1] = static_cast<int64_t>(h.task.size());
            stats6[2] = maxLevels;
            stats6[3] = topWide;
            stats6[4] = binPos;
            stats6[5] = nbd.factorFrom;
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

extern "C" int olfgpu_create_batch_context_full(
    int64_t structure, int nScenarios, int mode, const int* rlVoltageRow, int rlVoltageRowLength,
    const double* rlMinQ, int rlMinQLength, const double* rlMaxQ, int rlMaxQLength, const double* rlLoadQ,
    int rlLoadQLength, const double* rlTargetV, int rlTargetVLength, const signed char* rlFlags, int rlFlagsLength,
    const double* rowSlope, int rowSlopeLength, const int* dsBusPhiRow, int dsBusPhiRowLength,
    const double* dsBusFactor, int dsBusFactorLength, int slackBusPhiRow, double slackBusTargetP,
    const double* dsBusBaseTargetP, int dsBusBaseTargetPLength, const double* dsBusMaxDelta, int dsBusMaxDeltaLength,
    const double* dsBusMinDelta, int dsBusMinDeltaLength, int dsFactorMode, const double* dsBusMarginUp,
    int dsBusMarginUpLength, const double* dsBusMarginDown, int dsBusMarginDownLength, double slackBusMarginUp,
    double slackBusMarginDown, int64_t* contextOut) {
    return guarded([&] {
        if (!contextOut) throw std::runtime_error("null output handle");
        *contextOut = 0;
        const int nRl = rlVoltageRowLength;
        if (rlMinQLength != nRl || rlMaxQLength != nRl || rlLoadQLength != nRl || rlTargetVLength != nRl ||
            (rlFlagsLength != 0 && rlFlagsLength != nRl)) {
            throw std::runtime_error("createBatchContext: reactive-limit arrays differ in length");
        }
        for (int i = 0; i < rlFlagsLength; i++) {
            if (rlFlags[i] != 0) {
                throw std::runtime_error("createBatchContext: reactive-limit entry " + std::to_string(i) +
                                         " is a voltage-monitoring SVC (flag 1): not supported by this engine");
            }
        }
        for (int r = 0; r < rowSlopeLength; r++) {
            if (rowSlope[r] != 0.0) {
                throw std::runtime_error("createBatchContext: voltage slope on row " + std::to_string(r) +
                                         " is not supported by this engine");
            }
        }
        // distributed slack: bus-level participants with static factors (GpuDistributedSlackFactorMode STATIC 0);
        // the REMAINING_MARGIN mode and its margins are not modelled
        (void)dsBusMarginUp; (void)dsBusMarginDown; (void)slackBusMarginUp; (void)slackBusMarginDown;
        const int nDs = dsBusPhiRowLength;
        if (dsBusFactorLength != nDs || dsBusBaseTargetPLength != nDs || dsBusMaxDeltaLength != nDs ||
            dsBusMinDeltaLength != nDs) {
            throw std::runtime_error("createBatchContext: distributed-slack arrays differ in length");
        }
        if (nDs > 0 && dsFactorMode != 0) {
            throw std::runtime_error("createBatchContext: distributed-slack factor mode " + std::to_string(dsFactorMode) +
                                     " (REMAINING_MARGIN) is not supported by this engine");
        }
        if (dsBusMarginUpLength != 0 || dsBusMarginDownLength != 0) {
            if (dsFactorMode != 0) throw std::runtime_error("createBatchContext: margins are not supported");
        }
        std::unique_ptr<BatchContext> c(createContext(structureOf(structure), nScenarios, mode, nRl, rlVoltageRow, rlMinQ,
                                                      rlMaxQ, rlLoadQ, rlTargetV, nullptr, nullptr, nullptr, nullptr));
        if (nDs > 0) {
            setDistributedSlack(*c, nDs, dsBusPhiRow, dsBusFactor, dsBusBaseTargetP, dsBusMaxDelta, dsBusMinDelta,
                                slackBusPhiRow, slackBusTargetP);
        }
        *contextOut = reinterpret_cast<int64_t>(c.release());
    });
}

extern "C" int olfgpu_last_slack_distribution_failures(int64_t context, unsigned char* failed, int* count) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        std::vector<unsigned char> f(c.nS, 0);
        if (c.ds.nDs > 0) {
            OLF_CUDA(cudaSetDevice(c.device));
            OLF_CUDA(cudaMemcpy(f.data(), c.dsFailed.p, c.nS, cudaMemcpyDeviceToHost));
        }
        int k = 0;
        for (int i = 0; i < c.nS; i++) k += f[i] ? 1 : 0;
        if (failed) std::memcpy(failed, f.data(), c.nS);
        if (count) *count = k;
    });
}

extern "C" int olfgpu_set_reactive_limit_strongest_pv_keys(int64_t context, const double* nomV, const int* pRow,
                                                           const double* staticP, const int* idRank, int count) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        if (c.rl.nRl == 0) return;
        if (count != c.rl.nRl || !nomV || !pRow || !staticP || !idRank) {
            throw std::runtime_error("setBatchReactiveLimitStrongestPvKeys: array length != nReactiveLimitEntries");
        }
        setStrongestPvKeys(c, nomV, pRow, staticP, idRank);
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
            schedule != SCHEDULE_LEVELS_SHARED && schedule != SCHEDULE_LEVELS_SHARED_ALL &&
            schedule != SCHEDULE_SUBTREES) {
            throw std::runtime_error("unknown schedule");
        }
        c.regionFactor = schedule == SCHEDULE_LEVELS_SHARED || schedule == SCHEDULE_LEVELS_SHARED_ALL ||
                         schedule == SCHEDULE_SUBTREES;
        c.regionSolve = schedule == SCHEDULE_LEVELS_SHARED_ALL || schedule == SCHEDULE_SUBTREES;
        c.subtrees = schedule == SCHEDULE_SUBTREES;
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
                        : c.subtrees                 ? SCHEDULE_SUBTREES
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

extern "C" int olfgpu_solve_batch_context_full(
    int64_t context, const double* x0Base, int x0BaseLength, const double* targetBase, int targetBaseLength,
    const int* rowModeEntries, int rowModeEntriesLength, const int* baseRowMode, int baseRowModeLength,
    const unsigned char* disabledMask, int nScenarios, int nElements, const int* targetOverrideIndex,
    int targetOverrideIndexLength, const double* targetOverrideValue, int targetOverrideValueLength,
    const int* distributedSlackOverrideBus, int distributedSlackOverrideBusLength,
    const double* distributedSlackOverrideFactorDelta, int distributedSlackOverrideFactorDeltaLength,
    const double* distributedSlackOverrideBaseTargetPDelta, int distributedSlackOverrideBaseTargetPDeltaLength,
    const double* distributedSlackOverrideMaxDelta, int distributedSlackOverrideMaxDeltaLength,
    const double* distributedSlackOverrideMinDelta, int distributedSlackOverrideMinDeltaLength,
    const double* distributedSlackBusAnchorShift, int distributedSlackBusAnchorShiftLength,
    const double* slackBusAnchorShift, int slackBusAnchorShiftLength,
    const int* reactiveLimitTargetVOverrideScenarioEntry, int reactiveLimitTargetVOverrideScenarioEntryLength,
    const double* reactiveLimitTargetVOverrideValue, int reactiveLimitTargetVOverrideValueLength,
    const int* reactiveLimitDeltaOverrideScenarioEntry, int reactiveLimitDeltaOverrideScenarioEntryLength,
    const double* reactiveLimitDeltaOverrideValues, int reactiveLimitDeltaOverrideValuesLength,
    const int* reactiveCapabilityCurveOverrideScenarioCurve, int reactiveCapabilityCurveOverrideScenarioCurveLength,
    const double* reactiveCapabilityCurveOverrideStepScale, int reactiveCapabilityCurveOverrideStepScaleLength,
    int maxIter, double tol, double reactiveLimitTol, double slackDistTol, double convEpsPerEq,
    int stateVectorScalingMode, double maxDv, double maxDphi, const int* varType, int varTypeLength,
    const double* x0PerScenario, int x0PerScenarioLength, const int* shuntOvSlotElem, int shuntOvSlotElemLength,
    const double* shuntOvGb, int shuntOvGbLength, const int* reactiveLimitsSeedState, int reactiveLimitsSeedStateLength,
    const int* closedBranchParameterOverrideScenarioElement, int closedBranchParameterOverrideScenarioElementLength,
    const double* closedBranchParameterOverrideValues, int closedBranchParameterOverrideValuesLength,
    int maxOuterIterations, int maxPqPvSwitch, int rejectSlackDistributionFailure, int skipReactiveLimitsPhase,
    int nBaseClosedZeroImpedanceBranches, const int* zeroImpedanceBranchCloseScenarioElement,
    int zeroImpedanceBranchCloseScenarioElementLength, const int* zeroImpedanceBranchOpenScenarioElement,
    int zeroImpedanceBranchOpenScenarioElementLength, int pauseAtEnded, double* out) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        const int n = c.net->host.n;
        // the families and overrides this engine does not model must be empty (the Java side passes null or a
        // zero-length array when it has none); the pointers themselves are never read
        (void)distributedSlackOverrideBus; (void)distributedSlackOverrideFactorDelta;
        (void)distributedSlackOverrideBaseTargetPDelta; (void)distributedSlackOverrideMaxDelta;
        (void)distributedSlackOverrideMinDelta; (void)distributedSlackBusAnchorShift; (void)slackBusAnchorShift;
        (void)reactiveLimitTargetVOverrideScenarioEntry; (void)reactiveLimitTargetVOverrideValue;
        (void)reactiveLimitDeltaOverrideScenarioEntry; (void)reactiveLimitDeltaOverrideValues;
        (void)reactiveCapabilityCurveOverrideScenarioCurve; (void)reactiveCapabilityCurveOverrideStepScale;
        (void)shuntOvSlotElem; (void)shuntOvGb; (void)reactiveLimitsSeedState;
        (void)closedBranchParameterOverrideScenarioElement; (void)closedBranchParameterOverrideValues;
        (void)zeroImpedanceBranchCloseScenarioElement; (void)zeroImpedanceBranchOpenScenarioElement;

        const std::pair<const char*, int> unsupported[] = {
            {"distributedSlackOverrideBus", distributedSlackOverrideBusLength},
            {"distributedSlackOverrideFactorDelta", distributedSlackOverrideFactorDeltaLength},
            {"distributedSlackOverrideBaseTargetPDelta", distributedSlackOverrideBaseTargetPDeltaLength},
            {"distributedSlackOverrideMaxDelta", distributedSlackOverrideMaxDeltaLength},
            {"distributedSlackOverrideMinDelta", distributedSlackOverrideMinDeltaLength},
            {"distributedSlackBusAnchorShift", distributedSlackBusAnchorShiftLength},
            {"slackBusAnchorShift", slackBusAnchorShiftLength},
            {"reactiveLimitTargetVOverrideScenarioEntry", reactiveLimitTargetVOverrideScenarioEntryLength},
            {"reactiveLimitTargetVOverrideValue", reactiveLimitTargetVOverrideValueLength},
            {"reactiveLimitDeltaOverrideScenarioEntry", reactiveLimitDeltaOverrideScenarioEntryLength},
            {"reactiveLimitDeltaOverrideValues", reactiveLimitDeltaOverrideValuesLength},
            {"reactiveCapabilityCurveOverrideScenarioCurve", reactiveCapabilityCurveOverrideScenarioCurveLength},
            {"reactiveCapabilityCurveOverrideStepScale", reactiveCapabilityCurveOverrideStepScaleLength},
            {"shuntOvSlotElem", shuntOvSlotElemLength},
            {"shuntOvGb", shuntOvGbLength},
            {"reactiveLimitsSeedState", reactiveLimitsSeedStateLength},
            {"closedBranchParameterOverrideScenarioElement", closedBranchParameterOverrideScenarioElementLength},
            {"closedBranchParameterOverrideValues", closedBranchParameterOverrideValuesLength},
            {"zeroImpedanceBranchCloseScenarioElement", zeroImpedanceBranchCloseScenarioElementLength},
            {"zeroImpedanceBranchOpenScenarioElement", zeroImpedanceBranchOpenScenarioElementLength},
        };
        for (const auto& u : unsupported) {
            if (u.second < 0) throw std::runtime_error(std::string("negative length of ") + u.first);
            if (u.second > 0) {
                throw std::runtime_error(std::string("solveBatchContext: ") + u.first +
                                         " is not supported by this engine (pass null or an empty array)");
            }
        }
        if (nBaseClosedZeroImpedanceBranches != 0) {
            throw std::runtime_error("solveBatchContext: zero-impedance branches are not supported by this engine");
        }
        if (pauseAtEnded != 0) {
            throw std::runtime_error("solveBatchContext: pausing at ended scenarios (pauseAtEnded) is not supported");
        }
        auto need = [&](const char* what, const void* p, int len, int want) {
            if (!p) return;
            if (len != want) {
                throw std::runtime_error(std::string("solveBatchContext: ") + what + " has length " +
                                         std::to_string(len) + ", expected " + std::to_string(want));
            }
        };
        need("x0Base", x0Base, x0BaseLength, n);
        need("targetBase", targetBase, targetBaseLength, n);
        need("baseRowMode", baseRowMode, baseRowModeLength, n);
        need("varType", varType, varTypeLength, n);
        need("x0PerScenario", x0PerScenario, x0PerScenarioLength, nScenarios * n);
        if (rowModeEntriesLength % 3 != 0) throw std::runtime_error("rowModeEntries must hold (scenario, row, mode) triples");
        if (targetOverrideIndexLength != targetOverrideValueLength) {
            throw std::runtime_error("targetOverrideIndex and targetOverrideValue differ in length");
        }
        // the scenarios of this solve go into the bank slots chosen by olfgpu_begin_batch_install (local scenario j
        // into slot installSlots[j]; none chosen: the whole bank, j into j); the other slots stay idle
        const std::vector<int> slots = c.installSlots;
        const int nLocal = slots.empty() ? c.nS : static_cast<int>(slots.size());
        if (nScenarios != nLocal) {
            throw std::runtime_error("scenario count " + std::to_string(nScenarios) +
                                     " mismatch with the installed slots (" + std::to_string(nLocal) + ")");
        }
        if (!slots.empty() && c.deviceStart) {
            throw std::runtime_error("a device-resident start cannot be combined with an installation into chosen slots");
        }
        // expanded to the whole bank when slots are chosen
        std::vector<unsigned char> disBank, live;
        std::vector<double> x0Bank, ovVal;
        std::vector<int> rmeBank, ovIdx;
        const unsigned char* dis = disabledMask;
        const double* x0f = x0PerScenario;
        const int* rme = rowModeEntries;
        const int* toi = targetOverrideIndex;
        const double* tov = targetOverrideValue;
        int nS = nScenarios;
        if (!slots.empty()) {
            nS = c.nS;
            disBank.assign(static_cast<size_t>(nS) * nElements, 0);
            live.assign(nS, 0);
            for (int j = 0; j < nLocal; j++) {
                live[slots[j]] = 1;
                if (disabledMask) {
                    std::memcpy(&disBank[static_cast<size_t>(slots[j]) * nElements],
                                disabledMask + static_cast<size_t>(j) * nElements, nElements);
                }
            }
            dis = disabledMask ? disBank.data() : nullptr;
            if (x0PerScenario) {
                x0Bank.assign(static_cast<size_t>(nS) * n, 0.0);
                for (int s2 = 0; s2 < nS; s2++)
                    if (x0Base) std::memcpy(&x0Bank[static_cast<size_t>(s2) * n], x0Base, sizeof(double) * n);
                for (int j = 0; j < nLocal; j++) {
                    std::memcpy(&x0Bank[static_cast<size_t>(slots[j]) * n], x0PerScenario + static_cast<size_t>(j) * n,
                                sizeof(double) * n);
                }
                x0f = x0Bank.data();
            }
            rmeBank.assign(rowModeEntries ? rowModeEntries : nullptr,
                           rowModeEntries ? rowModeEntries + rowModeEntriesLength : nullptr);
            for (size_t k = 0; k < rmeBank.size(); k += 3) {
                if (rmeBank[k] < 0 || rmeBank[k] >= nLocal) throw std::runtime_error("rowMode entry outside the installed slots");
                rmeBank[k] = slots[rmeBank[k]];
            }
            rme = rmeBank.empty() ? nullptr : rmeBank.data();
            ovIdx.resize(targetOverrideIndexLength);
            for (int k = 0; k < targetOverrideIndexLength; k++) {
                const int v = targetOverrideIndex[k];
                if (v < 0 || v >= nLocal * n) throw std::runtime_error("target override index out of range");
                ovIdx[k] = slots[v / n] * n + v % n;
            }
            toi = ovIdx.empty() ? nullptr : ovIdx.data();
        }
        SolveRequest r = requestOf(x0Base, x0f, targetBase, baseRowMode, rowModeEntriesLength / 3, rme, nS,
                                   nElements, dis, targetOverrideIndexLength, toi, tov, maxIter, tol,
                                   reactiveLimitTol, maxOuterIterations, maxPqPvSwitch);
        r.convEpsPerEq = convEpsPerEq;
        r.stateVectorScalingMode = stateVectorScalingMode;
        r.maxDv = maxDv;
        r.maxDphi = maxDphi;
        r.varType = varType;
        r.skipReactiveLimits = skipReactiveLimitsPhase != 0;
        r.slackDistTol = slackDistTol;
        r.rejectDsFailure = rejectSlackDistributionFailure != 0;
        r.laneLive = live.empty() ? nullptr : live.data();
        c.handedBack.resize(nLocal);
        for (int j = 0; j < nLocal; j++) c.handedBack[j] = slots.empty() ? j : slots[j];
        if (slots.empty() && c.statesToHost) {
            solveBatch(c, r, out);
            c.solveCount++;             // a refused request is not a solve
            return;
        }
        // result rows of the installed scenarios, in installation order: [x(n), iterations, ||F||inf, status], or the
        // three last alone when the states stay on the device (olfgpu_set_states_to_host)
        std::vector<double> bank(static_cast<size_t>(nS) * (n + 3));
        solveBatch(c, r, bank.data());
        c.solveCount++;
        const int width = c.statesToHost ? n + 3 : 3;
        for (int j = 0; j < nLocal; j++) {
            const double* row = &bank[static_cast<size_t>(c.handedBack[j]) * (n + 3)];
            if (out) std::memcpy(out + static_cast<size_t>(j) * width, row + (n + 3 - width), sizeof(double) * width);
        }
    });
}

extern "C" int olfgpu_context_info(int64_t context, int* n, int* nElements, int* nScenarios, int* installed,
                                   int* batchedIterations, int64_t* solveCount) {
    return guarded([&] {
        const BatchContext& c = contextOf(context);
        if (n) *n = c.net->host.n;
        if (nElements) *nElements = c.net->host.nElements;
        if (nScenarios) *nScenarios = c.nS;
        if (installed) *installed = c.installSlots.empty() ? c.nS : static_cast<int>(c.installSlots.size());
        if (batchedIterations) *batchedIterations = c.lastIterations;
        if (solveCount) *solveCount = c.solveCount;
    });
}

extern "C" int olfgpu_begin_batch_install(int64_t context, const int* bankSlots, int count) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        if (count < 0 || (count > 0 && !bankSlots)) throw std::runtime_error("bad bank slot list");
        std::vector<char> taken(c.nS, 0);
        for (int k = 0; k < count; k++) {
            const int s2 = bankSlots[k];
            if (s2 < 0 || s2 >= c.nS || taken[s2]) {
                throw std::runtime_error("bank slot " + std::to_string(s2) + " outside the bank of " +
                                         std::to_string(c.nS) + " or installed twice");
            }
            taken[s2] = 1;
        }
        c.installSlots.assign(bankSlots, bankSlots + count);
    });
}

extern "C" int olfgpu_read_handed_back_slots(int64_t context, int* slots, int maxCount, int* count) {
    return guarded([&] {
        const BatchContext& c = contextOf(context);
        const int k = static_cast<int>(c.handedBack.size());
        for (int j = 0; slots && j < std::min(k, maxCount); j++) slots[j] = c.handedBack[j];
        if (count) *count = k;
    });
}

extern "C" int olfgpu_set_states_to_host(int64_t context, int statesToHost) {
    return guarded([&] { contextOf(context).statesToHost = statesToHost != 0; });
}

extern "C" int olfgpu_states_to_host(int64_t context, int* statesToHost) {
    return guarded([&] {
        if (!statesToHost) throw std::runtime_error("null output");
        *statesToHost = contextOf(context).statesToHost ? 1 : 0;
    });
}

namespace {

// Rows [nSlots][width] of chosen bank slots out of a lane-interleaved device table ([width][S] of T), after the
// context's stream has drained.
template <typename T, typename U>
void readSlotRows(BatchContext& c, const void* device, int width, int nSlots, const int* slots, U* out) {
    const int n = width;
    if (nSlots < 0 || (nSlots > 0 && (!slots || !out))) throw std::runtime_error("bad slot list or output");
    if (n == 0 || nSlots == 0) return;
    for (int j = 0; j < nSlots; j++) {
        if (slots[j] < 0 || slots[j] >= c.nS) throw std::runtime_error("slot outside the bank");
    }
    OLF_CUDA(cudaSetDevice(c.device));
    OLF_CUDA(cudaStreamSynchronize(c.stream));
    std::vector<T> col(static_cast<size_t>(n) * c.S);
    OLF_CUDA(cudaMemcpy(col.data(), device, col.size() * sizeof(T), cudaMemcpyDeviceToHost));
    for (int j = 0; j < nSlots; j++) {
        for (int r = 0; r < n; r++) {
            out[static_cast<size_t>(j) * n + r] = static_cast<U>(col[static_cast<size_t>(r) * c.S + slots[j]]);
        }
    }
}

}  // namespace

extern "C" int olfgpu_read_batch_states(int64_t context, int nSlots, const int* slots, double* out) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        readSlotRows<double>(c, c.x.p, c.net->host.n, nSlots, slots, out);
    });
}

extern "C" int olfgpu_read_batch_targets(int64_t context, int nSlots, const int* slots, double* out) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        readSlotRows<double>(c, c.target.p, c.net->host.n, nSlots, slots, out);
    });
}

extern "C" int olfgpu_read_batch_row_modes(int64_t context, int nSlots, const int* slots, int* out) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        readSlotRows<int8_t>(c, c.mode.p, c.net->host.n, nSlots, slots, out);
    });
}

extern "C" int olfgpu_read_reactive_limits_state(int64_t context, int nSlots, const int* slots, int* out,
                                                 int* nEntries) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        const int nRl = c.rl.nRl;
        if (nEntries) *nEntries = nRl;
        if (nRl == 0) return;
        std::vector<int> limitType(static_cast<size_t>(std::max(nSlots, 0)) * nRl);
        std::vector<int> switches(limitType.size());
        readSlotRows<int8_t>(c, c.rlLimitType.p, nRl, nSlots, slots, limitType.data());
        readSlotRows<int8_t>(c, c.rlSwitchCount.p, nRl, nSlots, slots, switches.data());
        // GpuReactiveLimitsState: the limit type (0 none, 1 MIN_Q, 2 MAX_Q) in the low three bits, the PV -> PQ
        // switch count above them (gpu_reactive_limits_state.cuh:10-26)
        for (size_t k = 0; k < limitType.size(); k++) out[k] = (limitType[k] & 7) | (switches[k] << 3);
    });
}

extern "C" int olfgpu_set_outer_loops(int64_t context, int distributedSlack, int reactiveLimits) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        c.dsLoop = distributedSlack != 0;
        c.reactiveLimitsLoop = reactiveLimits != 0;
    });
}

extern "C" int olfgpu_set_realistic_check(int64_t context, const unsigned char* rowChecked, double minV, double maxV,
                                          int enabled) {
    return guarded([&] {
        BatchContext& c = contextOf(context);
        c.hasVCheck = false;
        if (!enabled || !rowChecked) return;
        if (!(minV <= maxV)) throw std::runtime_error("realistic voltage band: minV must not exceed maxV");
        const int n = c.net->host.n;
        std::vector<int8_t> rc(n);
        for (int r = 0; r < n; r++) rc[r] = rowChecked[r] ? 1 : 0;
        OLF_CUDA(cudaSetDevice(c.device));
        OLF_CUDA(cudaMemcpyAsync(c.vCheck.p, rc.data(), n, cudaMemcpyHostToDevice, c.stream));
        OLF_CUDA(cudaStreamSynchronize(c.stream));
        c.realisticMinV = minV;
        c.realisticMaxV = maxV;
        c.hasVCheck = true;
    });
}

extern "C" int olfgpu_set_refinement_bound(int64_t context, double correctionBound) {
    return guarded([&] {
        if (!(correctionBound >= 0)) throw std::runtime_error("correctionBound must be >= 0");
        contextOf(context).corrBound = correctionBound;
    });
}

extern "C" int olfgpu_set_start_polish(int64_t context, double polishRatio) {
    return guarded([&] {
        if (!(polishRatio >= 0 && polishRatio <= 1)) throw std::runtime_error("polishRatio must lie in [0, 1]");
        contextOf(context).polishRatio = polishRatio;
    });
}

extern "C" int olfgpu_set_device_loop(int64_t context, int enable) {
    return guarded([&] { contextOf(context).deviceLoop = enable != 0; });
}

extern "C" int olfgpu_set_fp64_restart(int64_t context, int enable) {
    return guarded([&] { contextOf(context).fp64Restart = enable != 0; });
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

extern "C" int olfgpu_set_mixed_precision_policy(int64_t context, int policy) {
    return guarded([&] {
        if (policy != MIXED_REFINE && policy != MIXED_FP64_NEAR) {
            throw std::runtime_error("mixed-precision policy " + std::to_string(policy) + " unknown (0 or 1)");
        }
        contextOf(context).mixedPolicy = policy;
    });
}

extern "C" int olfgpu_last_fp64_iterations(int64_t context, int* iterations) {
    return guarded([&] {
        if (!iterations) throw std::runtime_error("null output");
        *iterations = contextOf(context).fp64Iterations;
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
        if (lanesPerTile == 0) {   // the members' device-resident level-schedule loops, one graph
            m.lanesPerTile = 0;
            m.autotunePending = false;
            return;
        }
        if (lanesPerTile != 1 && lanesPerTile != 2 && lanesPerTile != 4 && lanesPerTile != 8) {
            throw std::runtime_error("lanesPerTile must be 0, 1, 2, 4 or 8 (or -1: autotune)");
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

extern "C" int olfgpu_screen_violations(int64_t context, int nElem, const int* elemId, const int* groupPtr,
                                        const int* groupSide, const int* groupQty, const int* limPtr,
                                        const double* limThreshold, int nBus, const int* busVRow,
                                        const double* busHigh, const double* busLow, int realistic, double minV,
                                        double maxV, double band, int capacity, int* records, int* counts) {
    return guarded([&] {
        if ((nElem > 0 && (!elemId || !groupPtr || !limPtr)) || (nBus > 0 && (!busVRow || !busHigh || !busLow))) {
            throw std::runtime_error("null table with a non-zero count");
        }
        if (!(band >= 0.0)) throw std::runtime_error("band must be >= 0");
        ViolationTables t;
        t.nElem = nElem;
        t.elemId = elemId;
        t.groupPtr = groupPtr;
        t.groupSide = groupSide;
        t.groupQty = groupQty;
        t.limPtr = limPtr;
        t.limThreshold = limThreshold;
        t.nBus = nBus;
        t.busVRow = busVRow;
        t.busHigh = busHigh;
        t.busLow = busLow;
        t.realistic = realistic;
        t.minV = minV;
        t.maxV = maxV;
        t.band = band;
        screenViolations(contextOf(context), t, capacity, records, counts);
    });
}

extern "C" int olfgpu_linear_solve_transposed(int64_t context, const double* csrVals, const double* rhs,
                                              const double* rhsTransposed, int precision, double* solution,
                                              double* solutionTransposed) {
    return guarded([&] {
        if (precision != 0 && precision != 1) throw std::runtime_error("precision must be 0 (FP64) or 1 (FP32)");
        if (!csrVals) throw std::runtime_error("null Jacobian values");
        linearSolveBoth(contextOf(context), csrVals, rhs, rhsTransposed, precision, solution, solutionTransposed);
    });
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
