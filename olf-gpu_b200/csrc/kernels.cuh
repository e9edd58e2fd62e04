// Device kernels of the batched Newton-Raphson engine (sm_100a).
//
// Every per-scenario array is lane-interleaved: element e of lane s sits at [e * S + s], S = the lane count rounded
// up to a multiple of 32, so consecutive threads (lanes) of a warp touch consecutive addresses.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace olfb200 {

// Per-lane status codes (codes/gpu_ac_solver_status.cuh:10-15) and the engine's running state.
enum : int {
    ST_CONVERGED = 0,
    ST_MAX_ITERATION_REACHED = 1,
    ST_UNREALISTIC_STATE = 2,
    ST_DIVERGED = -1,
    ST_REJECTED = -2,
    ST_LINEAR_SOLVE_FAILED = -3,
    ST_RUNNING = 100,
};

// Row modes (codes/gpu_row_mode.cuh:10-15).
enum : int { MODE_FIXED_VARIABLE = 0, MODE_EQUATION = 1, MODE_BUS_TARGET_Q = 4 };

// One incident closed-branch side of a node, sorted by neighbour: branch element, which side the node is on (0: the
// node is bus 1, 1: bus 2), the neighbour node and the A block of (node, neighbour).
struct Side {
    int element;
    int side;
    int neighbour;
    int aBlock;
};

// One factorization task (an LU block): where its A block is (-1: fill-in), its update pairs, and for an L block the
// U diagonal block whose inverse it is multiplied by (-1 for U blocks, -2 for a U diagonal block).
struct Task {
    int aBlock;
    int opBegin;
    int opEnd;
    int diag;
};

// Everything the kernels read about one network (device pointers), built once per structure.
struct DevNet {
    int n, nb, nA, nLu, nU, ncb, nob, nsh, nElements;
    int deferredL;            // 1: the L factor is kept unscaled during the factorization (see structure.hpp)
    int frontStart, frontF;   // dense front: positions frontStart .. nb-1 (frontF = 0: none)
    const int* frontBlocks;   // [frontF * frontF] LU block of front positions (i, j)
    const int* nodeCol;       // [2 nb]
    const int* sidePtr;       // [nb + 1]
    const Side* side;         // incident closed-branch sides
    const double* cbPar;      // [ncb * 8] y g1 g2 b1 b2 ksi r1 a1
    const double2* cbTrig;    // [ncb] (sin ksi, cos ksi)
    const int* aPtr;          // [nb + 1] A blocks by node row
    const int* aCol;          // [nA]
    const int* aDiag;         // [nb]
    const int* shPtr;         // [nb + 1]
    const int* shList;        // shunt elements
    const double* shPar;      // [nsh * 2] g b
    const int* obPtr;         // [nb + 1]
    const int2* obList;       // (open-branch element, connected side 0/1)
    const double* obPar;      // [nob * 7] y ksi g1 b1 g2 b2 r1
    // LU
    const Task* task;         // [nLu]
    const int4* ops;          // updates (L block, U block, the pivot's inverted diagonal block or -1, unused)
    const int* levelTask;     // tasks grouped by level
    const int* perm;          // position -> node
    const int* iperm;         // node -> position
    const int* lrowPtr;       // [nb + 1] L blocks of each row position
    const int* lrowEnd;       // [nb] end of a row's forward-solve entries (a front row stops before the front columns)
    const int2* lrow;         // (L block id, column position)
    const int* uPtr;          // [nb + 1] U blocks of each row position (diagonal first: holds the inverse)
    const int* uCol;          // column position of each U block
    const int* lrowU;         // per L entry L(i, k) of lrow: the U block U(k, i) (transposed solve)
    const int* uRowL;         // per U block U(i, j), j > i: the L block L(j, i) (transposed solve)
};

// Programmatic dependent launch (level kernels): pdlTrigger lets the next grid in the stream start its CTAs once
// every CTA of this grid has started; pdlWait blocks until the previous grid has completed and its writes are
// visible (immediately when the grid was not launched as a dependent).  Every thread of a level kernel reaches
// pdlWait, so a level completes only after the one before it.
__device__ __forceinline__ void pdlTrigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdlWait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// The 2x2 block expressions with every rounding written out (the compiler contracts nothing here): the level kernels
// and the cooperative sweeps, compiled separately, give the same bits.  dot2(a, x, b, y) = a x + b y as
// fma(a, x, round(b y)).
__device__ __forceinline__ double rnMul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rnMul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rnFma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float rnFma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double rnSub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rnSub(float a, float b) { return __fsub_rn(a, b); }
template <typename T>
__device__ __forceinline__ T dot2(T a, T x, T b, T y) { return rnFma(a, x, rnMul(b, y)); }

// Per-batch device state (lane-interleaved arrays).
struct DevBatch {
    int S;                    // lane stride (multiple of 32)
    int nS;                   // installed scenarios (lanes >= nS are padding, never active)
    double* x;                // [n][S]
    double* target;           // [n][S]
    int8_t* mode;             // [n][S]
    double* F;                // [n][S]
    double* J;                // [nA][4][S]
    double* lu64;             // [nLu][4][S]
    float* lu32;              // [nLu][4][S] (mixed precision only)
    double* w64;              // [nb][2][S] solve work (positions)
    float* w32;               // [nb][2][S]
    double* dx;               // [n][S]
    double* res;              // [n][S] refinement residual
    double* qbuf;             // [n][S] closed-branch flows on their rows (reactive limits)
    const uint32_t* disabled; // [nElements][S / 32] outage bits
    unsigned long long* norm; // [S] max |F| as ordered bits
    int* iter;                // [S] Newton iteration of the current solve
    int* status;              // [S]
    int* outer;               // [S] reactive-limit outer iterations
    int* totalIter;           // [S] Newton iterations over all solves
    int* trouble;             // [S] near-singular pivots met in the last factorization
    double* normOut;          // [S] the last tested ||F||inf
    int8_t* active;           // [S] 1 while the lane iterates
    int8_t* pending;          // [S] 1: converged this iteration, reactive limits to check
    int8_t* precision64;      // [S] 1: this lane's last factorization fell back to FP64 (mixed precision)
    int* nActive;             // [8] lanes iterating, factorizing, refining, flagged for FP64, scored (read by the host)
    // fallback start: a lane whose solve ends unconverged (diverged, iteration cap, failed linear solve) while its
    // fallbackLeft flag is set restarts once from fallbackX (the base start, [n]) and marks fellBack
    const double* fallbackX;
    int nFallback;            // length of fallbackX (n)
    int fallbackOn;           // set fallbackLeft for every live lane at install
    int8_t* fallbackLeft;     // [S]
    int8_t* fellBack;         // [S]
    // mixed precision: a FP32 pivot block whose growth (condition estimate max|D| max|inv D|, or max|D| / max|A_kk|)
    // exceeds growthLimit flags its lane in precision64; laneMask (may be null) restricts the LU kernels to flagged lanes
    double growthLimit;
    const int8_t* laneMask;
    unsigned long long* resNorm;  // [S] max |refinement residual| (or correction) as ordered bits
    // mixed precision: a lane whose solve fails (diverged, iteration cap, failed linear solve) while fp64Left is set
    // restarts once with every factorization and solve in FP64 (precision64 stays set), from its own start row of
    // restartFull ([nS][n] scenario-major) or, when that is null, from fallbackX; fp64Left null: no such restart
    int8_t* fp64Left;
    const double* restartFull;
    int8_t* refine;           // [S] mixed: lanes whose refinement correction is still above the bound
    double* ssqPart;          // [SSQ_STRANDS][S] partial sums of F^2 (the 2-norm test)
    double* solveRatio;       // [S] the linear-solve residual ratio scored before the iteration budget
    unsigned long long* stepMax;  // [2][S] max |dV| and max |dphi| of the step (MAX_VOLTAGE_CHANGE), ordered bits
    const int8_t* varType;    // [n] 0 BUS_V, 1 BUS_PHI, -1 neither (MAX_VOLTAGE_CHANGE); may be null
    const int8_t* vCheck;     // [n] 1: a voltage row checked against the realistic band at convergence; may be null
    const int8_t* laneLive;   // [S] 1: the lane holds a scenario of this solve (null: lanes < nS); others stay idle
    int8_t* dsRestart;        // [S] distributed slack moved the targets this iteration: the lane re-solves (no RL check)
};

// Distributed-slack participants (bus level; BatchSolveNative.createBatchContext's tables): P rows, participation
// factors, base targets and the bounds of their move from the base; the slack bus's angle row (its P equation is the
// identity) and net P target; per lane the participants' targets before the last distribution and a failure flag.
struct DevDs {
    int nDs;
    const int* row;
    const double* factor;
    const double* baseTarget;
    const double* maxDelta;
    const double* minDelta;
    int slackRow;
    double slackTargetP;
    double* prevTarget;       // [nDs][S]
    int8_t* failed;           // [S] the last distribution left more than P_RESIDUE_EPS unplaced
};
// ActivePowerDistribution's residue epsilon (1e-5 pu): below it a mismatch is not distributed, above it an unplaced
// remainder is a distribution failure.
constexpr double P_RESIDUE_EPS = 1e-5;

// Strands of the deterministic 2-norm reduction (row r of a lane goes to strand r % SSQ_STRANDS, summed in row order,
// then the strands in strand order).
constexpr int SSQ_STRANDS = 64;
// The linear-solve residual ratio ||J dx + F||inf / ||F||inf above which a solve did not solve the system
// (iterative_refinement.cuh:21-23).
constexpr double LIN_SOLVE_FAIL_RATIO = 1e-2;
// trouble codes of a lane's last factorization / solve: 1 near-singular 2x2 pivot, 2 the linear-solve guard failed
enum : int { TROUBLE_PIVOT = 1, TROUBLE_GUARD = 2 };
// State-vector scaling modes (codes/gpu_state_vector_scaling_mode.cuh) and variable types
// (codes/gpu_ac_variable_type.cuh) of the MAX_VOLTAGE_CHANGE step clamp.
enum : int { SVS_NONE = 0, SVS_LINE_SEARCH = 1, SVS_MAX_VOLTAGE_CHANGE = 2 };
enum : int { VAR_BUS_V = 0, VAR_BUS_PHI = 1 };

// Reactive-limit entries (ReactiveLimitsPacker.java:76) and their per-lane state.
struct DevRl {
    int nRl;
    const int* voltageRow;
    const double* minQ;
    const double* maxQ;
    const double* loadQ;
    const double* targetV;
    const double* nomV;
    const int* pRow;
    const double* staticP;
    const int* idRank;
    int8_t* limitType;        // [nRl][S] 0 none, 1 min, 2 max
    int8_t* switchCount;      // [nRl][S]
    int8_t* passSwitched;     // [nRl][S]
    int8_t* savedMode;        // [nRl][S]
    double* savedTarget;      // [nRl][S]
    int* remainingPv;         // [S]
    int* switched;            // [S]
};

struct Settings {
    int maxIter;
    double tol;
    int reactiveLimits;
    double rlTol;
    int maxOuter;
    int maxSwitch;
    int mixed;                // 1: FP32 factorization and solves with FP64 refinement
    int refinementSteps;
    double growthLimit;       // pivot growth above which a mixed lane refactors in FP64
    double refineBelow;       // refinement steps run in an iteration where a factorizing lane's max |F| is below it
    double corrBound;         // mixed: a lane keeps refining while its last correction's max |d| is above it
    // fallback mode: a lane converged from its own start (the learned start) takes one more Newton step when its max
    // |F| is above polishBelow (0: never), so its state lies near the solution rather than anywhere in the tolerance
    // ball, and agrees with the state the base-start trajectory reaches
    double polishBelow;
    // OLF's stopping criterion when > 0 (newton_iteration.cu:105,241-250): converged when ||F||2 < norm2Threshold =
    // sqrt(convEpsPerEq^2 n); else the device's ||F||inf < tol
    double norm2Threshold;
    int batchOfOne;           // a bad last solve at the budget ends LINEAR_SOLVE_FAILED (one scenario) or REJECTED
    int svsMode;              // SVS_NONE or SVS_MAX_VOLTAGE_CHANGE (state_vector_scaling.cu:53-97)
    double maxDv, maxDphi;
    int realistic;            // 1: a converged state with a checked voltage outside [minV, maxV] is UNREALISTIC_STATE
    double minV, maxV;
    int distributedSlack;     // 1: the distributed-slack outer loop runs on converged lanes (before reactive limits)
    double slackDistTol;      // slack mismatch above which it is distributed (slackBusPMaxMismatch, pu)
    int rejectDsFailure;      // 1: a lane whose distribution fails ends REJECTED (else the rest stays on the slack)
};

// Kernel launchers (stream-ordered; all lanes of the batch).
void launchFill(const DevNet& net, const DevBatch& b, bool withJacobian, bool withQbuf, cudaStream_t st);
void launchTest(const DevNet& net, const DevBatch& b, const Settings& cfg, int* remainingPv, cudaStream_t st);
void launchReactiveLimits(const DevNet& net, const DevBatch& b, const DevRl& rl, const Settings& cfg,
                          cudaStream_t st);
// The distributed-slack check of the lanes that converged this iteration (distributed_slack.cu:211-616, bus level),
// after launchTest and before launchReactiveLimits.
void launchDistributedSlack(const DevBatch& b, const DevDs& ds, const Settings& cfg, cudaStream_t st);
// The dependency levels the persistent kernel walks (device pointers) and, per level, the longest update list of its
// tasks/rows (sets how many threads share a task).
struct PersistentPlan {
    int nLevels, nFwd, nBwd;
    const int* levelPtr;
    const int* levelLongest;
    const int* fwdPtr;
    const int* fwdLongest;
    const int* fwdPos;
    const int* bwdPtr;
    const int* bwdLongest;
    const int* bwdPos;
    int maxRounds;           // batched-iteration cap: lanes still iterating after it are REJECTED
};

// Level ranges for every tile of `lanes` lanes in one launch (the narrow levels of the level schedule).
void launchFactorRange(const DevNet& net, const DevBatch& b, const PersistentPlan& plan, int l0, int l1, int lanes,
                       bool fp32, cudaStream_t st);
void launchSolveRange(const DevNet& net, const DevBatch& b, const PersistentPlan& plan, int dir, int l0, int l1,
                      int lanes, bool fp32, cudaStream_t st);

// The narrow levels of the level schedule run as one range launch per phase: factorization levels [factorFrom,
// factorTo), forward levels >= fwdFrom, backward levels < bwdUntil, in tiles of `lanes` lanes (0: no range launches).
// Factorization levels from factorTo on (the dense front's assembly level) are launched level by level after the
// range.  With regionSlots > 0 the factorization levels [regionFrom, factorTo) run in shared memory instead
// (launchRegionFactor): slot k holds the block of task levelTask[regionBase + k]; regionTask[k] = (task, end of its
// updates, first update with an operand in the region, pivot code: -2 pivot, -1 / -3 stored as summed, >= 0 the
// inverted pivot's block outside the region, <= -4 its slot -4 - code).
// Subtree bins of the wide levels: independent subtrees of the elimination tree (a position's tasks only read blocks of
// its own subtree), packed into bins; one CTA per (bin, 32 lanes) runs its bin level by level with a barrier between
// levels, so the wide bottom of the factorization and of the solves costs one launch each instead of one per level.
// Factorization: bin b's levels are [levPtr[b], levPtr[b + 1]), level v holding the LU blocks task[levOff[v] ..
// levOff[v + 1]); the forward and backward solves likewise over positions.  The wide levels' other tasks (the
// separators above the bins: "top" tasks) keep their level launches from the top lists (device arrays; the level
// bounds and split factors are host arrays).
struct SubtreePlan {
    int nBins = 0;
    // host: the factorization's bins of phase f are [phasePtr[f], phasePtr[f + 1]), the sweeps' likewise; a phase
    // reads its own bin's values and earlier phases' (the backward sweep: later phases')
    int nPhases = 0, nFwdPhases = 0, nBwdPhases = 0;
    const int *phasePtr = nullptr, *fwdPhasePtr = nullptr, *bwdPhasePtr = nullptr;
    const int *levPtr = nullptr, *levOff = nullptr, *task = nullptr;
    const int *fwdPtr = nullptr, *fwdOff = nullptr, *fwdPos = nullptr;
    const int *bwdPtr = nullptr, *bwdOff = nullptr, *bwdPos = nullptr;
    const int* topLevelTask = nullptr;   // device: top tasks grouped by level (bounds topLevelPtr, host)
    const int *topLevelPtr = nullptr, *topLevelSplit = nullptr;
    const int* topFwdPos = nullptr;      // device: top positions grouped by forward level
    const int *topFwdPtr = nullptr, *topFwdSplit = nullptr;
    const int* topBwdPos = nullptr;      // device: top positions grouped by backward level
    const int *topBwdPtr = nullptr, *topBwdSplit = nullptr;
};
// The bins' factorization (before the wide levels' top tasks), forward sweep (before the top forward levels) and
// backward sweep (after every top backward level); no-op without bins.
void launchSubtreeFactor(const DevNet& net, const DevBatch& b, const SubtreePlan& sp, bool fp32, cudaStream_t st);
void launchSubtreeSolve(const DevNet& net, const DevBatch& b, const SubtreePlan& sp, bool fp32, int dir,
                        cudaStream_t st);

struct Hybrid {
    int factorFrom, factorTo, fwdFrom, bwdUntil, lanes;
    PersistentPlan plan;
    const SubtreePlan* sub = nullptr;   // subtree bins of the wide levels (null: every wide level as launches)
    int regionFrom = 0, regionBase = 0, regionSlots = 0;
    const int4* regionTask = nullptr;
    // the solves' narrow levels in shared memory (launchSolveRegion): the forward tail [fwdFrom, nFwd) (slot k: position
    // fwdPos[fwdRegionBase + k]) and the backward head [0, bwdUntil) (slot k: position bwdPos[k]); lrowSlot / uSlot:
    // per L / U entry, the slot + 1 of its column in the region of its row, 0 outside; fwdRegionStart[k]: the first
    // entry of forward slot k's row with a column in the region (the entries before it go to the prefix launch)
    bool solveRegion = false;
    int fwdRegionBase = 0, fwdRegionSlots = 0, bwdRegionSlots = 0;
    const int* lrowSlot = nullptr;
    const int* uSlot = nullptr;
    const int* fwdRegionStart = nullptr;
};
// The shared-memory factorization of the narrow levels (two launches; no-op when h.regionSlots == 0; every region
// level holds at most REGION_THREADS tasks).  prepareRegion raises the kernel's dynamic shared-memory limit for nSlots
// slots and nLevels levels on the current device.
constexpr int REGION_THREADS = 256;
void launchRegionFactor(const DevNet& net, const DevBatch& b, const Hybrid& h, bool fp32, cudaStream_t st);
// One sweep's narrow solve levels in shared memory (dir 0 the forward tail, 1 the backward head), one CTA per lane.
void launchSolveRegion(const DevNet& net, const DevBatch& b, const Hybrid& h, bool fp32, int dir, cudaStream_t st);
cudaError_t prepareRegion(int nSlots, int nLevels);

// Level boundaries (host), the positions of each level (device) and the split factor of each level (host).
struct LevelSchedule {
    int levels;
    const int* ptr;
    const int* pos;
    const int* split;
};

void launchFactor(const DevNet& net, const DevBatch& b, const int* levelPtrHost, const int* levelSplitHost,
                  int nLevels, bool fp32, const Hybrid* hybrid, cudaStream_t st);
void launchSolve(const DevNet& net, const DevBatch& b, const LevelSchedule& fwd, const LevelSchedule& bwd, bool fp32,
                 bool fromResidual, const Hybrid* hybrid, cudaStream_t st);
void launchResidual(const DevNet& net, const DevBatch& b, cudaStream_t st);
// The transposed solve J^T y = c on the factors of the last factorization (transposed_solve.cuh:1-30): U^T forward on
// the forward levels, then L^T backward on the backward levels, the dense front's positions swept in order between;
// c is read from b.res (n rows, lane-interleaved) and y written to b.dx.
void launchSolveTransposed(const DevNet& net, const DevBatch& b, const LevelSchedule& fwd, const LevelSchedule& bwd,
                           bool fp32, cudaStream_t st);
void launchStep(const DevNet& net, const DevBatch& b, const Settings& cfg, cudaStream_t st);
void launchIterationStart(const DevBatch& b, cudaStream_t st);
// Lanes that factorize this iteration (nActive[1]); of those, the lanes whose max |F| is below refineBelow
// (nActive[2], marked in b.refine: they start this iteration's refinement in mixed precision) and the lanes whose solve
// is scored this iteration (nActive[4]).
void launchCountSolving(const DevBatch& b, double refineBelow, int maxIter, cudaStream_t st);
// Factorizing lanes flagged for an FP64 refactor (nActive[3]).
void launchCountFp64(const DevBatch& b, cudaStream_t st);
// Mixed precision, after launchResidual: each lane's max |r| and the count of factorizing lanes with max |F| below
// refineBelow whose residual is above `threshold` (nActive[2]): the correction solve of a refinement step runs only
// when some lane needs it.
void launchResidualCheck(const DevNet& net, const DevBatch& b, double threshold, double refineBelow, cudaStream_t st);
// After a correction solve of the refining lanes (b.laneMask = b.refine; the solve left each correction d in b.res):
// a lane stays refining while max |d| > bound; nActive[2] = lanes still refining.
void launchCorrectionCheck(const DevNet& net, const DevBatch& b, double bound, cudaStream_t st);
// The 2-norm test's sum of squares of F per lane (deterministic strands), before launchTest.
void launchNorm2(const DevNet& net, const DevBatch& b, cudaStream_t st);
// Linear-solve scoring (iterative_refinement.cuh:21-23, newton_iteration.cu:378-392,615-647): for the lanes at the
// second iteration of their first solve (the guard) or one iteration before the budget, r = -F - J dx and its ratio
// max |r| / max |F|; a guard lane above LIN_SOLVE_FAIL_RATIO is marked TROUBLE_GUARD (no step; the next test ends it
// LINEAR_SOLVE_FAILED), a budget lane keeps the ratio for the budget's test.
void launchScoreSolve(const DevNet& net, const DevBatch& b, const Settings& cfg, cudaStream_t st);
// The dense front of a dense-front plan (after every factorization level); no-op without a front.  prepareDenseFront
// raises the kernels' dynamic shared-memory limit for a front of F pivots on the current device.
void launchDenseFront(const DevNet& net, const DevBatch& b, bool fp32, cudaStream_t st);
// The front positions' forward and backward solves (between the forward and the backward level sweeps).
void launchDenseFrontSolve(const DevNet& net, const DevBatch& b, bool fp32, cudaStream_t st);
cudaError_t prepareDenseFront(int F);

}  // namespace olfb200
