// Batched Newton-Raphson engine: device copy of a structure, batch contexts and the solve driver.
#pragma once

#include <cuda_runtime.h>

#include <memory>
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
    DeviceBuffer task, ops, levelTask, perm, iperm, lrowPtr, lrowEnd, lrow, uPtr, uCol, fwdPos, bwdPos;
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
};

struct NetStructure {
    Structure host;
    std::shared_ptr<DeviceNet> dev;
};

std::shared_ptr<DeviceNet> uploadNet(const Structure& s);

// Schedules of the Newton iterations: one launch per dependency level (captured in a CUDA graph per iteration), or
// the persistent kernel with one CTA per lane tile running the whole loop.
// SCHEDULE_LEVELS_SHARED and SCHEDULE_LEVELS_SHARED_ALL are API values only: the level schedule with the narrow
// factorization levels (BatchContext::regionFactor), and also the solves' narrow levels (regionSolve), in shared memory.
enum {
    SCHEDULE_LEVELS = 0,
    SCHEDULE_PERSISTENT = 1,
    SCHEDULE_COOP = 2,
    SCHEDULE_LEVELS_SHARED = 3,
    SCHEDULE_LEVELS_SHARED_ALL = 4
};

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
};

struct BatchContext {
    std::shared_ptr<NetStructure> net;
    int device = 0;
    int nS = 0, S = 0;
    cudaStream_t stream = nullptr;
    Settings cfg{};
    int precision = 0;              // 0 FP64, 1 mixed (FP32 LU + FP64 refinement)
    int refinementSteps = 1;
    // lane-interleaved state
    DeviceBuffer x, target, mode, F, J, lu64, lu32, w64, w32, dx, res, qbuf, disabled, norm, iter, status, outer,
        totalIter, trouble, normOut, active, pending, precision64, nActive, fallbackLeft, fellBack, resNorm;
    bool fallbackStart = false;     // lanes that fail from x0Full restart once from x0Base (both given)
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
    Hybrid hybrid() const {
        const DeviceNet& d = *net->dev;
        Hybrid h{d.factorFrom, d.factorTo, d.fwdFrom, d.bwdUntil, narrowLanes, d.persistent};
        h.plan.maxRounds = 1;
        if (regionFactor && d.regionSlots > 0) {
            h.regionFrom = d.regionFrom;
            h.regionBase = d.regionBase;
            h.regionSlots = d.regionSlots;
            h.regionTask = d.regionTask.as<int4>();
        }
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
    bool useHybrid() const { return narrowLanes > 0 || regionFactor || regionSolve; }
    std::vector<TuningResult> tuning;
    DeviceBuffer out;               // [nS][n + 3] scenario-major results
    // reactive limits
    DevRl rl{};
    DeviceBuffer rlVoltageRow, rlMinQ, rlMaxQ, rlLoadQ, rlTargetV, rlNomV, rlPRow, rlStaticP, rlIdRank, rlLimitType,
        rlSwitchCount, rlPassSwitched, rlSavedMode, rlSavedTarget, rlRemainingPv, rlSwitched;
    // host staging (pinned) and the per-scenario start states
    uint32_t* hostBitsPinned = nullptr;
    DeviceBuffer full;
    int* hostActive = nullptr;      // pinned [4]: lanes iterating, factorizing, to refine, flagged for FP64
    cudaEvent_t countReady = nullptr;  // mixed: the FP64-flag count has reached the host
    // one Newton iteration as a CUDA graph (captured on first use per settings)
    cudaGraphExec_t graph = nullptr;       // fill, test, reactive limits, lane counts
    cudaGraphExec_t graphSolve = nullptr;  // FP64: factorization, solves, step; mixed: FP32 solves
    // mixed precision only: FP32 factorization + count of FP64-flagged lanes; refinement steps; the FP64 refactor and
    // solve of the flagged lanes; the step
    cudaGraphExec_t graphFactor = nullptr, graphResidual = nullptr, graphCorrect = nullptr, graph64 = nullptr,
                    graphStep = nullptr;
    int graphKey = -1;
    double refineBelow = 1e-5;      // mixed: refinement steps only in iterations where a lane's max |F| is below it
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
    ~BatchContext();
    DevBatch batch() const;
};

BatchContext* createContext(std::shared_ptr<NetStructure> net, int nScenarios, int mode, int nRl, const int* voltageRow,
                            const double* minQ, const double* maxQ, const double* loadQ, const double* targetV,
                            const double* nomV, const int* pRow, const double* staticP, const int* idRank);

// Runs the batch; out = [nS][n + 3] per scenario [x(n), iterations, ||F||inf, status].
void solveBatch(BatchContext& ctx, const SolveRequest& req, double* out);

// Validates a request and uploads its inputs to the context (the first half of solveBatch).
void stageRequest(BatchContext& ctx, const SolveRequest& req);

struct MultiTuning {
    int lanesPerTile, threads, order;
    float ms;
};

// Batch contexts of different grids run by one persistent launch (one CTA per lane tile of any member, captured in
// a CUDA graph with the members' result gathers).  The members stay owned by their creator.
struct MultiContext {
    std::vector<BatchContext*> members;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<cudaEvent_t> ready;      // per member: its lanes are installed
    int lanesPerTile = 2, threads = 256, order = 0;   // order 0: as given, 1: most buses first
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

}  // namespace olfb200
