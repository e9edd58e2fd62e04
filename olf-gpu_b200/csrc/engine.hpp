// Batched Newton-Raphson engine: device copy of a structure, batch contexts and the solve driver.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "coop.cuh"
#include "persistent.cuh"
#include "structure.hpp"

namespace olfb200 {

#define OLF_CUDA(call)                                                                                              \
    do {                                                                                                            \
        cudaError_t err_ = (call);                                                                                  \
        if (err_ != cudaSuccess) {                                                                                  \
            throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(err_) + " at " __FILE__ ":" + \
                                     std::to_string(__LINE__));                                                     \
        }                                                                                                           \
    } while (0)

// A device allocation owned by its holder (freed on destruction; zero-filled on allocation).
struct DeviceBuffer {
    void* p = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() {
        if (p) cudaFree(p);
    }
    void alloc(size_t n) {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = n;
        if (n) {
            OLF_CUDA(cudaMalloc(&p, n));
            OLF_CUDA(cudaMemset(p, 0, n));
        }
    }
    template <typename T>
    void upload(const std::vector<T>& v) {
        alloc(v.size() * sizeof(T));
        if (!v.empty()) OLF_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

// The structure's read-only device data (shared by every context built on it, on one device).
struct DeviceNet {
    int device = 0;
    DevNet view{};
    std::vector<int> levelPtr, fwdPtr, bwdPtr;   // host copies of the level boundaries (launch geometry)
    std::vector<int> levelSplit, fwdSplit, bwdSplit;  // threads sharing one task / row, per level
    LevelSchedule fwd() const {
        return LevelSchedule{static_cast<int>(fwdPtr.size()) - 1, fwdPtr.data(), fwdPos.as<int>(), fwdSplit.data()};
    }
    LevelSchedule bwd() const {
        return LevelSchedule{static_cast<int>(bwdPtr.size()) - 1, bwdPtr.data(), bwdPos.as<int>(), bwdSplit.data()};
    }
    std::vector<int> csrToA;                      // CSR slot -> A block * 4 + entry (debug readback of J)
    DeviceBuffer csrToAD;                         // the same map on the device
    DeviceBuffer nodeCol, sidePtr, side, cbPar, cbTrig, aPtr, aCol, aDiag, shPtr, shList, shPar, obPtr, obList, obPar;
    DeviceBuffer frontBlocks;
    DeviceBuffer task, ops, levelTask, perm, iperm, lrowPtr, lrowEnd, lrow, uPtr, uCol, fwdPos, bwdPos, lrowU, uRowL;
    DeviceBuffer levelPtrD, levelLongestD, fwdPtrD, fwdLongestD, bwdPtrD, bwdLongestD, levelSplitD, fwdSplitD, bwdSplitD;
    CoopPlan coop{};
    PersistentPlan persistent{};
    int factorFrom = 0, factorTo = 0, fwdFrom = 0, bwdUntil = 0;   // narrow-level boundaries of the level schedule
    // shared-memory region of the narrow factorization levels [regionFrom, factorTo) (regionSlots 0: none)
    int regionFrom = 0, regionBase = 0, regionSlots = 0;
    DeviceBuffer regionTask;
    // shared-memory solve regions: the forward tail [fwdFrom, nFwd) and the backward head [0, bwdUntil) (slots 0: none)
    int fwdRegionBase = 0, fwdRegionSlots = 0, bwdRegionSlots = 0;
    DeviceBuffer lrowSlot, uSlot, fwdRegionStart;
    // subtree bins of the wide levels (sub.nBins 0: none) and the top lists of the wide levels
    SubtreePlan sub{};
    DeviceBuffer binLevPtr, binLevOff, binTask, binFwdPtr, binFwdOff, binFwdPos, binBwdPtr, binBwdOff, binBwdPos,
        topLevelTaskD, topFwdPosD, topBwdPosD;
    std::vector<int> topLevelPtr, topLevelSplit, topFwdPtr, topFwdSplit, topBwdPtr, topBwdSplit, binPhasePtr,
        binFwdPhasePtr, binBwdPhasePtr;
    int binTasks = 0;               // LU blocks the bins factorize (of nLu)
};

// A structure and its device copies, one per device ordinal (uploaded on first use there).  Contexts hold their own
// device copy, so creating a context on another GPU never touches the copies that contexts on other GPUs use.
struct NetStructure {
    Structure host;
    std::mutex mu;
    std::map<int, std::shared_ptr<DeviceNet>> devs;
    // The copy on `device` (which the caller has made current), uploaded on first use.
    std::shared_ptr<DeviceNet> onDevice(int device);
    // The copy on `device`, or null when none was uploaded there.
    std::shared_ptr<DeviceNet> find(int device);
};

std::shared_ptr<DeviceNet> uploadNet(const Structure& s);

// The level schedule's narrow boundaries: factorization levels [factorFrom, factorTo) hold at most 48 tasks (the range
// or shared-memory region), forward levels from fwdFrom and backward levels before bwdUntil likewise.
struct NarrowBounds {
    int factorFrom, factorTo, fwdFrom, bwdUntil;
};
NarrowBounds narrowBounds(const BlockPlan& p);
// The first level of the shared-memory factorization region (nbd.factorTo: none), and the bounds the subtree bins
// use: the narrow bounds with the wide levels ending where the region starts.
int regionStart(const BlockPlan& p, const NarrowBounds& nbd);
NarrowBounds binBounds(const BlockPlan& p);

// The subtree bins of a plan's wide levels and the top lists of every level (host arrays; see SubtreePlan).
struct SubtreeBinsHost {
    int nBins = 0;
    std::vector<int> phasePtr;       // bins of phase f: [phasePtr[f], phasePtr[f + 1])
    std::vector<int> levPtr, levOff, task, fwdPtr, fwdOff, fwdPos, bwdPtr, bwdOff, bwdPos;
    std::vector<int> topLevelPtr, topTask, topFwdPtr, topFwd, topBwdPtr, topBwd;
    std::vector<int> fwdPhasePtr, bwdPhasePtr;   // the forward and backward sweeps' bins per phase
    std::vector<int> taskBin, fwdBinOf, bwdBinOf;  // factorization bin of each LU block, sweep bins of each position
    std::vector<int> posOf;          // position of each LU block
};
SubtreeBinsHost planSubtreeBins(const BlockPlan& p, const NarrowBounds& nbd);
// "" when the bins keep every dependency of the factorization and both sweeps, else the first violation.
std::string checkSubtreeBins(const BlockPlan& p, const NarrowBounds& nbd, const SubtreeBinsHost& h);

// Schedules of the Newton iterations: one launch per dependency level (captured in a CUDA graph per iteration), or
// the persistent kernel with one CTA per lane tile running the whole loop.
// SCHEDULE_LEVELS_SHARED and SCHEDULE_LEVELS_SHARED_ALL are API values only: the level schedule with the narrow
// factorization levels (BatchContext::regionFactor), and also the solves' narrow levels (regionSolve), in shared memory.
enum {
    SCHEDULE_LEVELS = 0,
    SCHEDULE_PERSISTENT = 1,
    SCHEDULE_COOP = 2,
    SCHEDULE_LEVELS_SHARED = 3,
    SCHEDULE_LEVELS_SHARED_ALL = 4,
    SCHEDULE_SUBTREES = 5          // schedule 4 with the wide levels' subtrees in one launch per phase (subtree bins)
};

// Mixed-precision policies (BatchContext::mixedPolicy)
enum { MIXED_REFINE = 0, MIXED_FP64_NEAR = 1 };

// Mixed precision: a refinement step's correction solve runs only while some lane's FP64 residual max |r| is above
// this fraction of the mismatch tolerance (below it the FP32 solve is already accurate enough for the test).
constexpr double REFINE_RESIDUAL = 0.1;

struct TuningResult {
    int schedule, lanesPerTile, threads;
    float ms;
};

// Linear-solve modes accepted at the boundary (codes/gpu_linear_solve_mode.cuh:10-12): all run the engine's own
// batched block LU.
enum { MODE_UBATCH = 3, MODE_ROBUST = 6, MODE_BATCHED_LU = 7 };

struct SolveRequest {
    const double* x0Base = nullptr;      // [n]
    const double* x0Full = nullptr;      // [nS][n] or null
    const double* targetBase = nullptr;  // [n]
    const int* baseRowMode = nullptr;    // [n]
    const int* rowModeEntries = nullptr; // (scenario, row, mode) triples
    int nRowModeEntries = 0;
    const unsigned char* disabled = nullptr;  // [nS][nElements]
    int nScenarios = 0;
    int nElements = 0;
    const int* targetOverrideIndex = nullptr;  // flat scenario * n + row
    const double* targetOverrideValue = nullptr;
    int nTargetOverrides = 0;
    int maxIter = 15;
    double tol = 1e-8;
    double reactiveLimitTol = 1e-4;
    int maxOuter = 20;
    int maxPqPvSwitch = 3;
    double convEpsPerEq = 0.0;       // > 0: OLF's ||F||2 < sqrt(convEpsPerEq^2 n) stopping criterion
    int stateVectorScalingMode = 0;  // 0 NONE, 2 MAX_VOLTAGE_CHANGE
    double maxDv = 0.1, maxDphi = 0.17453292519943295;
    const int* varType = nullptr;    // [n] 0 BUS_V, 1 BUS_PHI (MAX_VOLTAGE_CHANGE)
    bool skipReactiveLimits = false; // this solve runs without the reactive-limit outer loop
    double slackDistTol = 1e-2;      // distributed slack: the mismatch above which it is distributed (pu)
    bool rejectDsFailure = false;    // distributed slack: a failed distribution ends the scenario REJECTED
    const unsigned char* laneLive = nullptr;  // [nS] or null: the bank lanes that hold a scenario of this solve
};

struct BatchContext {
    std::shared_ptr<NetStructure> net;
    std::shared_ptr<DeviceNet> dn;     // the structure's copy on this context's device
    int device = 0;
    int nS = 0, S = 0;
    cudaStream_t stream = nullptr;
    Settings cfg{};
    int precision = 0;              // 0 FP64, 1 mixed (FP32 LU + FP64 refinement)
    int refinementSteps = 1;
    // lane-interleaved state
    DeviceBuffer x, target, mode, F, J, lu64, lu32, w64, w32, dx, res, qbuf, disabled, norm, iter, status, outer,
        totalIter, trouble, normOut, active, pending, precision64, nActive, fallbackLeft, fellBack, resNorm, fp64Left,
        refine, ssqPart, solveRatio, stepMax, varType, vCheck;
    bool fp64Restart = true;        // mixed: a lane whose solve fails restarts once in FP64 (persistent: fully refined)
    bool fp64RestartOn = false;     // in force for the installed batch
    bool hasVarType = false;        // the request carried the variable types of the MAX_VOLTAGE_CHANGE clamp
    bool hasVCheck = false;         // the realistic-voltage rows are set
    DeviceBuffer laneLive;          // [S] installed lanes of the solve (hasLaneLive)
    std::vector<int8_t> liveHost;
    bool hasLaneLive = false;
    // the boundary's slot bookkeeping (BatchSolveNative.beginBatchInstall / readBatchHandedBackSlots /
    // setBatchStatesToHost): the bank slots the next solve installs (empty: the whole bank), the slots the last solve
    // handed back, whether result rows carry the states, and the reactive-limit outer loop switch
    std::vector<int> installSlots, handedBack;
    bool statesToHost = true;
    int64_t solveCount = 0;         // solves run through the full entry (BatchReadbackNative.readBatchSolveCount)
    bool reactiveLimitsLoop = true;
    bool fallbackStart = false;     // lanes that fail from x0Full restart once from x0Base (both given)
    double polishRatio = 1e-2;      // fallback mode: polish a lane converged from its own start above polishRatio * tol
    bool rlKeys = false;            // the reactive-limit entries' forced-PV election keys are set
    const double* deviceStart = nullptr;  // caller's device array [nS][n] used as x0Full by the solves
    const double* fullSrc = nullptr;      // where the installed x0Full rows come from
    DeviceBuffer stage;             // upload staging (base vectors)
    DeviceBuffer ovIdx, ovVal, rowModeE;  // per-scenario overrides of the installed batch
    int nTargetOverrides = 0, nRowModeEntries = 0;
    bool hasX0Base = false, hasX0Full = false;
    // schedule of the Newton iterations (set explicitly or picked by the autotuner on the next solve)
    int schedule = SCHEDULE_LEVELS;
    int lanesPerTile = 2;
    int threads = 512;
    bool autotunePending = false;
    int narrowLanes = 2;            // level schedule: lanes per tile of the narrow-level range launches (0: none)
    bool regionFactor = false;      // level schedule: the narrow factorization levels in shared memory
    bool regionSolve = false;       // level schedule: the solves' narrow levels in shared memory too
    bool subtrees = false;          // level schedule: the wide levels' independent subtrees as bins (schedule 5)
    Hybrid hybrid() const {
        const DeviceNet& d = *dn;
        Hybrid h{d.factorFrom, d.factorTo, d.fwdFrom, d.bwdUntil, narrowLanes, d.persistent};
        h.plan.maxRounds = 1;
        if (regionFactor && d.regionSlots > 0) {
            h.regionFrom = d.regionFrom;
            h.regionBase = d.regionBase;
            h.regionSlots = d.regionSlots;
            h.regionTask = d.regionTask.as<int4>();
        }
        if (subtrees && d.sub.nBins > 0) h.sub = &d.sub;
        if (regionSolve) {
            h.solveRegion = true;
            h.fwdRegionBase = d.fwdRegionBase;
            h.fwdRegionSlots = d.fwdRegionSlots;
            h.bwdRegionSlots = d.bwdRegionSlots;
            h.lrowSlot = d.lrowSlot.as<int>();
            h.uSlot = d.uSlot.as<int>();
            h.fwdRegionStart = d.fwdRegionStart.as<int>();
        }
        return h;
    }
    bool useHybrid() const { return narrowLanes > 0 || regionFactor || regionSolve || subtrees; }
    std::vector<TuningResult> tuning;
    DeviceBuffer out;               // [nS][n + 3] scenario-major results
    // reactive limits
    DevDs ds{};                     // distributed-slack participants (ds.nDs 0: none)
    DeviceBuffer dsRow, dsFactor, dsBase, dsMax, dsMin, dsPrev, dsFailed, dsRestartBuf;
    bool dsLoop = true;             // the distributed-slack outer loop switch (DriverNative.setBatchOuterLoops)
    DevRl rl{};
    DeviceBuffer rlVoltageRow, rlMinQ, rlMaxQ, rlLoadQ, rlTargetV, rlNomV, rlPRow, rlStaticP, rlIdRank, rlLimitType,
        rlSwitchCount, rlPassSwitched, rlSavedMode, rlSavedTarget, rlRemainingPv, rlSwitched;
    // host staging (pinned) and the per-scenario start states
    uint32_t* hostBitsPinned = nullptr;
    DeviceBuffer full;
    int* hostActive = nullptr;      // pinned [8]: lanes iterating, factorizing, to refine, flagged for FP64, scored
    cudaEvent_t countReady = nullptr;  // mixed: the FP64-flag count has reached the host
    // one Newton iteration as a CUDA graph (captured on first use per settings)
    cudaGraphExec_t graph = nullptr;       // fill, test, reactive limits, lane counts
    cudaGraphExec_t graphSolve = nullptr;  // FP64: factorization, solves, step; mixed: FP32 solves
    // mixed precision only: FP32 factorization + count of FP64-flagged lanes; refinement steps; the FP64 refactor and
    // solve of the flagged lanes; the step
    cudaGraphExec_t graphFactor = nullptr, graphResidual = nullptr, graphCorrect = nullptr, graph64 = nullptr,
                    graphStep = nullptr;
    cudaGraphExec_t graph64All = nullptr;  // MIXED_FP64_NEAR: FP64 factorization and solves of every factorizing lane
    // the same iteration with the linear-solve scoring before the step (FP64: factorization, solves, scoring, step;
    // mixed: scoring, step)
    cudaGraphExec_t graphSolveScored = nullptr, graphStepScored = nullptr;
    int graphKey = -1;
    DevBatch graphBatch{};          // the batch view and settings the iteration graphs were captured with
    Settings graphCfg{};
    // the whole Newton loop as one graph launch (conditional nodes; level schedules), and what it was built with
    bool deviceLoop = false;
    cudaGraphExec_t loopGraph = nullptr;
    long long loopGraphKey = -1;
    DevBatch loopBatch{};
    Settings loopCfg{};
    DeviceBuffer loopState;         // int [8]: iterations, refinement steps, iteration kind, FP64 iterations
    cudaStream_t loopStreams[3] = {nullptr, nullptr, nullptr};   // capture streams of the loop graph's bodies
    // mixed: a lane refines only in an iteration where its max |F| is below refineBelow; 1e-2 covers every step from
    // which Newton can land below the tolerance, so a converged state's last step is FP64-accurate
    double refineBelow = 1e-2;
    // mixed precision: MIXED_REFINE refines the FP32 solves of the lanes below refineBelow; MIXED_FP64_NEAR factors
    // and solves an iteration with such a lane in FP64 (all its lanes), and iterations without one in FP32, unrefined
    int mixedPolicy = 0;
    double corrBound = 1e-11;       // mixed: a lane keeps refining while its last correction's max |d| is above it
    double realisticMinV = 0.0, realisticMaxV = 0.0;   // realistic-voltage band (hasVCheck)
    double growthLimit = 1e4;       // mixed: FP32 pivot growth above which a lane refactors in FP64
    // statistics of the last solve
    int lastIterations = 0;         // batched iterations run
    float lastMs = 0.f;
    bool staged = false;            // inputs of a request uploaded (a multi-grid launch runs staged contexts)
    // phase timing (level schedule): each iteration launched phase by phase between CUDA events
    bool phaseTiming = false;
    double phaseMs[6] = {0, 0, 0, 0, 0, 0};   // fill, test, factorization, solves, refinement, step (summed)
    long long phaseLanes = 0;       // lanes that factorized, summed over the iterations
    int phaseIterations = 0;
    int fp64Iterations = 0;         // iterations of the last solve that MIXED_FP64_NEAR ran in FP64
    ~BatchContext();
    DevBatch batch() const;
};

BatchContext* createContext(std::shared_ptr<NetStructure> net, int nScenarios, int mode, int nRl, const int* voltageRow,
                            const double* minQ, const double* maxQ, const double* loadQ, const double* targetV,
                            const double* nomV, const int* pRow, const double* staticP, const int* idRank);

// Installs the distributed-slack participants of a context: P rows, factors (normalised here to sum 1), base targets,
// bounds of their move from the base; the slack bus's angle row and net P target.
void setDistributedSlack(BatchContext& ctx, int nDs, const int* row, const double* factor, const double* baseTarget,
                         const double* maxDelta, const double* minDelta, int slackRow, double slackTargetP);

// Runs the batch; out = [nS][n + 3] per scenario [x(n), iterations, ||F||inf, status].
void solveBatch(BatchContext& ctx, const SolveRequest& req, double* out);

// Validates a request and uploads its inputs to the context (the first half of solveBatch).
void stageRequest(BatchContext& ctx, const SolveRequest& req);

// The forced-PV election keys of the context's reactive-limit entries (reactive_limits.cu:417-448): nominal V, P row
// (-1: static P), static P, id rank, one per entry.
void setStrongestPvKeys(BatchContext& ctx, const double* nomV, const int* pRow, const double* staticP,
                        const int* idRank);

struct MultiTuning {
    int lanesPerTile, threads, order;   // lanesPerTile 0: every member's device-resident level-schedule loop
    float ms;
};

// Batch contexts of different grids run by one persistent launch (one CTA per lane tile of any member, captured in
// a CUDA graph with the members' result gathers).  The members stay owned by their creator.
struct MultiContext {
    std::vector<BatchContext*> members;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<cudaEvent_t> ready;      // per member: its lanes are installed
    std::vector<cudaEvent_t> done;       // per member: its results are gathered (an event node of the loop graph)
    int lanesPerTile = 2, threads = 256, order = 0;   // order 0: as given, 1: most buses first
    // lanesPerTile 0: one graph whose branches are the members' own device-resident Newton loops (their level
    // schedules, concurrent on the device), instead of the persistent tiles
    cudaGraphExec_t loopGraph = nullptr;
    std::vector<long long> loopKeys;
    std::vector<DevBatch> loopBatches;
    std::vector<Settings> loopCfgs;
    cudaStream_t capStreams[3] = {nullptr, nullptr, nullptr};
    bool autotunePending = false;
    std::vector<MultiTuning> tuning;
    DeviceBuffer itemsDev;
    MultiItem* hostItems = nullptr;      // pinned
    cudaGraphExec_t graph = nullptr;
    int graphKey = -1;
    float lastMs = 0.f;
    ~MultiContext();
};

MultiContext* createMultiContext(const std::vector<BatchContext*>& members);
// One launch over every member's staged batch; outs[i] (host, may be null) = member i's [nS][n + 3] results.
void solveMulti(MultiContext& m, double* const* outs);

// Debug/test surface: the Jacobian (CSR values of the reference-compatible pattern) and mismatch of every
// scenario at the given states, through the engine's fill; and a batched linear solve through the engine's LU.
void debugFill(BatchContext& ctx, const double* xFull, const double* targetBase, const int* baseRowMode,
               const unsigned char* disabled, double* jOut, double* fOut);
void debugLinearSolve(BatchContext& ctx, const double* csrVals, const double* rhs, int precision, double* out);
// Limit tables of the violation screening (host arrays; see violations.cu).
struct ViolationTables {
    int nElem = 0;
    const int* elemId = nullptr;       // [nElem] element (closed branch e, or open branch nCb + e)
    const int* groupPtr = nullptr;     // [nElem + 1] its limit groups
    const int* groupSide = nullptr;    // [groups] 1 or 2
    const int* groupQty = nullptr;     // [groups] 0 current I, 1 active power |P|, 2 apparent power S
    const int* limPtr = nullptr;       // [groups + 1] its thresholds
    const double* limThreshold = nullptr;
    int nBus = 0;
    const int* busVRow = nullptr;      // [nBus] the bus's V row (-1: none)
    const double* busHigh = nullptr;   // [nBus] high / low voltage limits (NaN: none)
    const double* busLow = nullptr;
    int realistic = 0;                 // 1: also the buses outside [minV, maxV]
    double minV = 0.0, maxV = 0.0;
    double band = 1e-7;                // relative relaxation of every threshold
};
// Screens the context's last solve: per scenario, up to `capacity` record ids (sorted) into records [nS][capacity] and
// the count of candidates into counts [nS] (a count above capacity: the list is truncated).
void screenViolations(BatchContext& ctx, const ViolationTables& t, int capacity, int* records, int* counts);

// One factorization of J (CSR values [nS][nnz]), then both J x = rhs and J^T y = rhsT on its factors (either rhs may be
// null, its output then untouched); all arrays scenario-major host arrays.
void linearSolveBoth(BatchContext& ctx, const double* csrVals, const double* rhs, const double* rhsT, int precision,
                     double* x, double* y);

}  // namespace olfb200
