/*
 * olfgpu_b200 -- C ABI of the B200 batched AC Newton-Raphson N-1 engine.
 *
 * The entry points mirror the native calls the reference's Java layer binds for this path (its JNI symbols
 * Java_com_powsybl_openloadflow_<pkg>_<cls>_<method>, native/cuda/jni/olf_jni.h:9); each declaration below names the
 * reference interface it replaces.  Plain pointers and sizes only.  Every function returns 0 on success and -1 on
 * failure, with the reason in olfgpu_last_error() (the JNI layer turns it into a RuntimeException, as
 * structure_jni.cu:128-137 and batch_solve_jni.cu:302-306 do).  Per-scenario problems are status codes, never errors.
 *
 * Threading: one CUDA stream per batch context; a handle is used by one caller at a time.  Handles are opaque
 * 64-bit values; 0 is never a valid handle and destroying 0 is a no-op.
 *
 * Statuses (codes/gpu_ac_solver_status.cuh:10-15): 0 CONVERGED, 1 MAX_ITERATION_REACHED, 2 UNREALISTIC_STATE,
 * -1 DIVERGED, -2 REJECTED, -3 LINEAR_SOLVE_FAILED.
 * Row modes (codes/gpu_row_mode.cuh:10-15): 0 FIXED_VARIABLE, 1 EQUATION, 4 BUS_TARGET_Q.
 */
#ifndef OLFGPU_B200_H
#define OLFGPU_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The reason of the calling thread's last failure ("" when none). */
const char* olfgpu_last_error(void);

/*
 * StructureNative.createStructure (native/cuda/jni/structure_jni.cu:7-137; StructureNative.java:49-59).
 * Packed families in the reference layout (GpuAcFamilyPacker.java:140-181):
 *   closed branch: params [nCb][8] {y, g1, g2, b1, b2, ksi, r1, a1}, indices [nCb][12]
 *                  {P1, Q1, P2, Q2, ph1, v1, ph2, v2, a1col, r1col, altQ1, altQ2}
 *   open branch:   params [nOb][7] {y, ksi, g1, b1, g2, b2, r1}, indices [nOb][6] {P1, Q1, P2, Q2, v1, v2}
 *   shunt:         params [nSh][2] {g, b}, indices [nSh][5] {P, Q, v, bcol, altQ}
 *   identity rows: [nIdentityRows]
 * The families this engine does not model (HVDC AC emulation, DISTR_Q/RHO/SHUNT_B, zero-impedance branches, load
 * models, reactive relocation, transformer/shunt voltage-control columns) must be empty: a non-empty one, or a
 * control column >= 0, is rejected with an error.  ordering: 0 minimum degree (default), 1 nested dissection,
 * 2 natural, 3 minimum degree relaxed toward a shallow elimination tree (fewer dependency levels at about the same
 * fill; 3 + 16 = 19 is the fastest measured plan); plus 8 for the deferred-L block-LU plan (the L factor stays unscaled during the factorization: about
 * half the dependency levels, one more 2x2 block read per update), or 16 for the dense-front plan (the trailing
 * pivots whose blocks are all present, up to 32, are factorized as one dense front in shared memory; not runnable by
 * the persistent schedules or the multi-grid launch).
 */
int olfgpu_create_structure(int n, int nCb, const double* cbParams, const int* cbIndices, int nOb,
                            const double* obParams, const int* obIndices, int nSh, const double* shParams,
                            const int* shIndices, int nIdentityRows, const int* identityRows, int ordering,
                            int64_t* structureOut);

/*
 * StructureNative.createStructure with the reference's full argument list, in its order (structure_jni.cu:7-137;
 * StructureNative.java:49-59): every Java array as a pointer and its length (null / 0 when absent).  Element counts
 * come from the index strides (closed 12, open 6, shunt 5).  The families this engine does not model must be empty
 * (HVDC AC emulation, DISTR_Q, zero-impedance branches, DISTR_RHO, DISTR_SHUNT_B, load models, reactive relocation
 * candidates), and the per-element "none" arrays must hold -1 only (closedBranchPhaseControlSide,
 * openBranchAlternateReactiveDestination, the relocation group maps; reactiveRelocationGroupStart empty or [0]);
 * otherwise the call fails naming the argument.  ordering as olfgpu_create_structure.
 */
int olfgpu_create_structure_full(
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
    const int* identityRows, int identityRowsLength, int ordering, int64_t* structureOut);

/* StructureNative.destroyStructure (structure_jni.cu:143-149): drops the caller's reference; contexts keep theirs. */
int olfgpu_destroy_structure(int64_t structure);

/*
 * Read back of the reference-compatible structure (for parity checks): rowMap [n], rowPtr [n+1], colIdx [nnz],
 * diagPos [n], and the role-folded destinations cbDest [nCb][28], obDest [nOb][8], shDest [nSh][5]
 * (>= 0 J slot, -2-row F row, -1 skip; structure_build.cuh:51-66).  info receives
 * {n, nnz, nBuses, nLuBlocks, factorLevels, forwardLevels, backwardLevels, nElements, nABlocks}; blockOps the 2x2
 * block updates of one factorization.  Any output pointer may be null.
 */
int olfgpu_structure_info(int64_t structure, int* info9, int64_t* blockOps);
int olfgpu_structure_export(int64_t structure, int* rowMap, int* rowPtr, int* colIdx, int* diagPos, int* cbDest,
                            int* obDest, int* shDest);

/*
 * The block-LU schedule of the structure (no counterpart in the reference): level boundaries of the factorization
 * (factorLevelPtr [factorLevels + 1], over LU blocks), of the forward and backward solves ([levels + 1], over
 * elimination positions), and the block updates of each factorization level (levelOps [factorLevels]).  Sizes from
 * olfgpu_structure_info; any pointer may be null.
 */
int olfgpu_structure_levels(int64_t structure, int* factorLevelPtr, int* forwardLevelPtr, int* backwardLevelPtr,
                            int64_t* levelOps);

/*
 * The subtree bins of the structure's wide levels (no counterpart in the reference; the schedule 5 of
 * olfgpu_set_schedule runs them): plans them on the host, checks that they keep every dependency of the factorization
 * and of both sweeps (fails naming the first violation otherwise), and writes {bins, LU blocks in bins, most levels of
 * a bin, LU blocks left on the wide levels, positions in bins, wide factorization levels} into stats6.
 */
int olfgpu_structure_subtrees(int64_t structure, int64_t* stats6);

/*
 * A host check of the structure's block-LU plan (no counterpart in the reference's API; the reference checks its own
 * LU schedules for races the same way, native/host/lu_transposed_check.cpp:175-216), from the plan's dependency data
 * alone: the symbolic factorization is closed and every block's update list complete and ascending; every LU block is
 * one factorization level task and every block a task reads lies on a strictly earlier level (so the tasks of one
 * level launch share no data), the dense front's split included; every solve position is on one forward (and, outside
 * the dense front, one backward) level and reads only entries of strictly earlier levels.  violations receives the
 * number found (0 for a sound plan), firstViolation (capacity bytes, may be null) the first one.  plantedFault 1..3
 * checks a copy with one planted error (a task moved one level up, an update dropped, two forward positions swapped
 * between the first and the last level) to test the check itself; 0 checks the plan as built.
 */
int olfgpu_structure_check_plan(int64_t structure, int plantedFault, int64_t* violations, char* firstViolation,
                                int capacity);

/* StructureNative.recommendBatchSize (structure_jni.cu:151-180): the bank that fits 70 % of free device memory. */
int olfgpu_recommend_batch_size(int64_t structure, int maxCap, int mode, int* batchOut);

/*
 * BatchSolveNative.createBatchContext (batch_solve_jni.cu:29-81; BatchSolveNative.java:41-48).
 * mode: linear-solve mode (3 UBATCH, 6 ROBUST, 7 BATCHED_LU; all run the engine's own batched LU).
 * Reactive-limit entries (ReactiveLimitsPacker.java:76), nRl may be 0: per voltage-controlling bus its V row, Q limits,
 * load Q, voltage target, and the forced-PV election keys (nominal V, P row or -1 with a static P, id rank;
 * reactive_limits.cu:417-448).
 */
int olfgpu_create_batch_context(int64_t structure, int nScenarios, int mode, int nRl, const int* rlVoltageRow,
                                const double* rlMinQ, const double* rlMaxQ, const double* rlLoadQ,
                                const double* rlTargetV, const double* rlNomV, const int* rlPRow,
                                const double* rlStaticP, const int* rlIdRank, int64_t* contextOut);

/*
 * BatchSolveNative.createBatchContext with the reference's full argument list (batch_solve_jni.cu:29-81;
 * BatchSolveNative.java:41-48), arrays as pointer + length.  The reactive-limit entries (voltage row, Q limits, load Q,
 * target V; all of one length) are installed without their forced-PV election keys, which
 * olfgpu_set_reactive_limit_strongest_pv_keys supplies before the first solve (a solve with entries but no keys
 * fails, as batch_solve_jni.cu:103-111 does).  reactiveLimitFlags must be 0 (voltage-monitoring SVCs are not
 * modelled) and rowSlope zero (no voltage slope).  Distributed slack (outerloop/distributed_slack.cu:211-616, bus
 * level): the participants' P rows, factors (STATIC mode 0; normalised to sum 1), base targets and the bounds of their
 * move (maxDelta >= 0 >= minDelta), the slack bus's angle row and net P target; after a scenario converges, a slack
 * mismatch (its closed-branch P minus the target) above solveBatchContext's slackDistTol is water-filled over the
 * participants from their base targets and the scenario re-solves, before its reactive-limit check; a distribution
 * that leaves more than 1e-5 pu unplaced ends the scenario REJECTED when rejectSlackDistributionFailure is set, else
 * the rest stays on the slack.  The REMAINING_MARGIN mode (1) and its margins are rejected.
 * olfgpu_last_slack_distribution_failures writes per scenario 1 where the last solve's distribution failed.
 */
int olfgpu_create_batch_context_full(
    int64_t structure, int nScenarios, int mode, const int* rlVoltageRow, int rlVoltageRowLength,
    const double* rlMinQ, int rlMinQLength, const double* rlMaxQ, int rlMaxQLength, const double* rlLoadQ,
    int rlLoadQLength, const double* rlTargetV, int rlTargetVLength, const signed char* rlFlags, int rlFlagsLength,
    const double* rowSlope, int rowSlopeLength, const int* dsBusPhiRow, int dsBusPhiRowLength,
    const double* dsBusFactor, int dsBusFactorLength, int slackBusPhiRow, double slackBusTargetP,
    const double* dsBusBaseTargetP, int dsBusBaseTargetPLength, const double* dsBusMaxDelta, int dsBusMaxDeltaLength,
    const double* dsBusMinDelta, int dsBusMinDeltaLength, int dsFactorMode, const double* dsBusMarginUp,
    int dsBusMarginUpLength, const double* dsBusMarginDown, int dsBusMarginDownLength, double slackBusMarginUp,
    double slackBusMarginDown, int64_t* contextOut);

int olfgpu_last_slack_distribution_failures(int64_t context, unsigned char* failed, int* count);

/* ReactiveLimitsNative.setBatchReactiveLimitStrongestPvKeys (reactive_limits_jni.cu:118-145): per reactive-limit
 * entry its nominal V, P row (-1: static P), static P and id rank; count must equal the entries. */
int olfgpu_set_reactive_limit_strongest_pv_keys(int64_t context, const double* nomV, const int* pRow,
                                                const double* staticP, const int* idRank, int count);

/*
 * Bank slots (BatchSolveNative.beginBatchInstall / readBatchHandedBackSlots / setBatchStatesToHost,
 * batch_solve_jni.cu:404-465): olfgpu_begin_batch_install chooses the bank slots the next full solve installs its
 * scenarios into (local scenario j into bankSlots[j], each slot at most once; count 0: the whole bank, j into j); the
 * other slots stay idle during that solve.  olfgpu_read_handed_back_slots writes the slots of the last full solve's
 * result rows, in row order (count receives their number).  With olfgpu_set_states_to_host(ctx, 0) the full solve's
 * result rows are [iterations, ||F||inf, status] alone (rows of 3) and the states stay on the device, where
 * olfgpu_read_batch_states copies the states of chosen slots ([nSlots][n]).  olfgpu_states_to_host reads the switch.
 */
int olfgpu_begin_batch_install(int64_t context, const int* bankSlots, int count);
int olfgpu_read_handed_back_slots(int64_t context, int* slots, int maxCount, int* count);
int olfgpu_set_states_to_host(int64_t context, int statesToHost);
int olfgpu_states_to_host(int64_t context, int* statesToHost);
int olfgpu_read_batch_states(int64_t context, int nSlots, const int* slots, double* out);

/* BatchReadbackNative.readBatchTargets / readBatchRowModes (batch_readback_jni.cu:13-45; read by
 * GpuNewtonRaphson.java:194,227 and GpuBatchChunkSolver.java:1183): the per-scenario targets and row modes of chosen
 * bank slots ([nSlots][n], slot order) as the last solve ended with them.  The outer loops rewrite both: a PV bus that
 * the reactive-limit loop switched to PQ has its voltage row's mode and target (its Q limit less its load) changed,
 * and the distributed slack moves its participants' P targets, so a converged state solves these equations, not the
 * installed ones.  Row modes use the codes the solve takes (baseRowMode). */
int olfgpu_read_batch_targets(int64_t context, int nSlots, const int* slots, double* out);
int olfgpu_read_batch_row_modes(int64_t context, int nSlots, const int* slots, int* out);

/* ReactiveLimitsNative.readBatchReactiveLimitsFinalState (reactive_limits_jni.cu:407-427; read by
 * GpuNewtonRaphson.java:579 and GpuBatchChunkSolver.java): per chosen bank slot and reactive-limit entry
 * ([nSlots][nEntries], slot order), the entry's state as the last solve ended: its limit type (0 still PV, 1 at MIN_Q,
 * 2 at MAX_Q) in the low three bits and its PV -> PQ switch count above them (gpu_reactive_limits_state.cuh).
 * nEntries (may be null) receives the context's reactive-limit entries; with none, nothing is written. */
int olfgpu_read_reactive_limits_state(int64_t context, int nSlots, const int* slots, int* out, int* nEntries);

/* DriverNative.setBatchOuterLoops (driver_jni.cu:11-18): the distributed-slack and reactive-limit outer loops on or off
 * for the following solves (each acts only where the context holds its tables). */
int olfgpu_set_outer_loops(int64_t context, int distributedSlack, int reactiveLimits);

/* A context's sizes and counters: n, elements, bank size, scenarios the next full solve installs, batched Newton
 * iterations of the last solve (BatchReadbackNative.readBatchNewtonLoopIterations, batch_readback_jni.cu:103-107), full
 * solves run (BatchReadbackNative.readBatchSolveCount, batch_readback_jni.cu:112-116).  Any pointer may be null. */
int olfgpu_context_info(int64_t context, int* n, int* nElements, int* nScenarios, int* installed,
                        int* batchedIterations, int64_t* solveCount);

/* BatchSolveNative.destroyBatchContext (batch_solve_jni.cu:396-401). */
int olfgpu_destroy_batch_context(int64_t context);

/*
 * NewtonSettingsNative.setLinearSolverSettings (native/cuda/jni/newton_settings_jni.cu; LinearSolverSettings,
 * linear_solver_settings.cuh:48-58).  precision: 0 FP64 factorization and solves; 1 FP32 factorization and solves
 * with FP32 accumulation, corrected by refinementSteps FP64 iterative-refinement steps (residual with the FP64
 * Jacobian).
 */
int olfgpu_set_linear_solver_settings(int64_t context, int precision, int refinementSteps);

/*
 * Mixed-precision controls (no counterpart in the reference; precision 1 only).  The refinement steps run only in
 * iterations where some factorizing scenario's max |F| is below refineBelow (default 1e-2, every step
 * that can land below the tolerance; infinity: every iteration):
 * far from convergence the next Newton iteration corrects the FP32 solve's error itself.  Each step of such a
 * scenario computes the FP64 residual r = -F - J dx and the correction solve, until the correction is below the bound
 * of olfgpu_set_refinement_bound.  A scenario whose FP32
 * factorization meets a pivot block with growth above growthLimit (condition estimate max|D| max|inv D|, or max|D|
 * over the largest entry of its Jacobian block; default 1e4) is flagged: in the level schedule its factorization and
 * solve are redone in FP64 in the same iteration (and every later one of the solve); the persistent schedules give
 * its tile the refinement steps instead.  olfgpu_last_fp64_refactors writes per scenario 1 where the last solve
 * flagged it (flagged [nScenarios], may be null) and their count.
 */
int olfgpu_set_mixed_precision_controls(int64_t context, double refineBelow, double growthLimit);
/* Mixed-precision policy (no counterpart in the reference, whose LU is FP64 only; level and cooperative schedules):
 * 0 (default) refines, as above; 1 runs an iteration in which
 * some factorizing scenario's max |F| is below refineBelow in FP64 for all its scenarios (factorization and solves),
 * and the other iterations in FP32 without refinement, so the last steps follow the FP64 trajectory at the cost of an
 * FP64 factorization instead of refinement solves.  olfgpu_last_fp64_iterations reads how many iterations of the last
 * solve ran in FP64 under policy 1. */
int olfgpu_set_mixed_precision_policy(int64_t context, int policy);
int olfgpu_last_fp64_iterations(int64_t context, int* iterations);
int olfgpu_last_fp64_refactors(int64_t context, unsigned char* flagged, int* count);

/*
 * Schedule of the Newton iterations (no counterpart in the reference, which launches per dependency step and per
 * level and reads norms back every iteration): schedule 0 launches one kernel per wide dependency level over all
 * lanes and the narrow levels (<= 48 tasks) of each phase in one launch of tiles of lanesPerTile (1, 2 or 4; 0: one
 * launch per level throughout), captured as one CUDA graph per Newton iteration;
 * schedule 1 runs the whole Newton loop in one persistent launch, one CTA per tile of lanesPerTile (1, 2, 4 or 8)
 * lanes with `threads` (256 or 512) threads; schedule 2 runs each factorization and each solve as one cooperative
 * launch over all lanes whose CTAs meet at a grid barrier between dependency levels (tile arguments ignored);
 * schedule 3 is schedule 0 with the narrow factorization levels run in shared memory, one CTA of 256 threads per
 * lane holding every LU block those levels produce (lanesPerTile then only sets the solves' narrow-level tiles; plans
 * whose narrow levels do not fit, and deferred-L plans, fall back to schedule 0); schedule 4 is schedule 3 with the
 * solves' narrow levels (the forward tail and the backward head) in shared memory as well, one CTA per lane holding
 * those rows' solution entries (lanesPerTile ignored); schedule -1 lets the next solve time every candidate on its
 * batch and keep the fastest (the autotuner).  olfgpu_get_schedule reports the schedule in force and, after an
 * autotuned solve, up to maxResults timings {schedule, lanesPerTile, threads, ms} into results (nResults receives
 * their count).
 */
int olfgpu_set_schedule(int64_t context, int schedule, int lanesPerTile, int threads);
int olfgpu_get_schedule(int64_t context, int* schedule, int* lanesPerTile, int* threads, int maxResults,
                        double* results, int* nResults);

/*
 * BatchSolveNative.solveBatchContext (batch_solve_jni.cu:84-394; BatchSolveNative.java:106-125).
 *   x0Base [n]: the start state of every scenario (ignored where x0Full is given), x0Full [nScenarios][n] or null;
 *   targetBase [n], baseRowMode [n]; rowModeEntries (scenario, row, mode) triples; disabled [nScenarios][nElements]
 *   bytes (element order: closed branches, open branches, shunts; BatchSolveNative.java:81-83);
 *   targetOverrideIndex (flat scenario * n + row) / targetOverrideValue;
 *   maxIter, tol (||F||inf stopping threshold), reactiveLimitTol, maxOuter (reactive-limit outer iterations),
 *   maxPqPvSwitch.
 * out [nScenarios][n + 3]: per scenario the final state x, the Newton iterations of its last solve, ||F||inf and the
 * status (batch_solve_jni.cu:308-337).
 */
int olfgpu_solve_batch_context(int64_t context, const double* x0Base, const double* x0Full, const double* targetBase,
                               const int* baseRowMode, int nRowModeEntries, const int* rowModeEntries,
                               int nScenarios, int nElements, const unsigned char* disabled, int nTargetOverrides,
                               const int* targetOverrideIndex, const double* targetOverrideValue, int maxIter,
                               double tol, double reactiveLimitTol, int maxOuter, int maxPqPvSwitch, double* out);

/*
 * BatchSolveNative.solveBatchContext with the reference's full argument list, in its order (batch_solve_jni.cu:84-100;
 * BatchSolveNative.java:106-125): every Java array argument is a pointer and its length (null or length 0 when the
 * caller has none), so a JNI shim forwards each one as it comes.  Supported beyond olfgpu_solve_batch_context:
 *   convEpsPerEq > 0: OLF's stopping criterion ||F||2 < sqrt(convEpsPerEq^2 n) (newton_iteration.cu:105,241-250)
 *     instead of ||F||inf < tol;
 *   stateVectorScalingMode 0 NONE or 2 MAX_VOLTAGE_CHANGE with maxDv, maxDphi and varType [n] (0 BUS_V, 1 BUS_PHI;
 *     state_vector_scaling.cu:53-97); 1 LINE_SEARCH is rejected;
 *   skipReactiveLimitsPhase != 0: this solve runs without the reactive-limit outer loop;
 *   x0PerScenario [nScenarios * n] (the reference's x0Full).
 * slackDistTol and rejectSlackDistributionFailure drive the distributed-slack outer loop (olfgpu_create_batch_context_full).
 * Rejected with an error naming the argument when non-empty (families this engine does not model): the distributed-
 * slack overrides and anchor shifts, the reactive-limit target-V / delta / capability-curve overrides, the shunt and
 * closed-branch parameter overrides, the reactive-limit seed state, the zero-impedance branch lists (and
 * nBaseClosedZeroImpedanceBranches != 0), and pauseAtEnded != 0.  out [nScenarios][n + 3] as
 * olfgpu_solve_batch_context.
 */
int olfgpu_solve_batch_context_full(
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
    int zeroImpedanceBranchOpenScenarioElementLength, int pauseAtEnded, double* out);

/*
 * ReactiveLimitsNative.setBatchRealisticCheck (reactive_limits_jni.cu:172-195; realistic_voltage_check.cu:23-44):
 * rowChecked [n] marks the voltage rows OLF's realistic-voltage check reads; a converged scenario with a checked
 * voltage outside [minV, maxV] ends UNREALISTIC_STATE (status 2), its state kept.  enabled = 0 (or rowChecked null)
 * clears the check.  The level and cooperative schedules apply it.
 */
int olfgpu_set_realistic_check(int64_t context, const unsigned char* rowChecked, double minV, double maxV, int enabled);

/*
 * Mixed precision (no counterpart in the reference): in an iteration where a scenario's max |F| is below refineBelow
 * (olfgpu_set_mixed_precision_controls), the scenario refines its FP32 solve (FP64 residual, correction solve) until
 * the correction's max |d| falls to correctionBound or below (default 1e-11), at most refinementSteps times: its last
 * Newton step is then FP64-accurate.  With olfgpu_set_fp64_restart enabled (the default), a scenario whose mixed-
 * precision solve fails (diverged, iteration budget, failed linear solve) restarts once with FP64 factorizations and
 * solves from its start, so it ends as the FP64 engine ends it (level and cooperative schedules, no reactive limits).
 */
int olfgpu_set_refinement_bound(int64_t context, double correctionBound);
int olfgpu_set_fp64_restart(int64_t context, int enable);

/*
 * Statistics of the context's last solve (no counterpart in the reference's API; its OLF_GPU_PHASE_TIME trace prints
 * similar counters, batch_solve_jni.cu:338-391): device milliseconds of its Newton iterations (CUDA events on the
 * context's stream), the batched iterations run, and per scenario the Newton iterations summed over all its solves
 * (totalIterations [nScenarios], may be null).
 */
int olfgpu_last_solve_stats(int64_t context, float* deviceMs, int* batchedIterations, int* totalIterations);

/*
 * Phase timing (diagnostics; no counterpart in the reference): with enable = 1 the level schedule launches every
 * Newton iteration phase by phase between CUDA events on the context's stream instead of replaying its graphs (same
 * kernels, same order).  olfgpu_last_phase_times writes, for the last solve, the milliseconds of {fill, test,
 * factorization, solves, refinement, step} summed over its iterations, then the iterations run and the lanes that
 * factorized summed over them (out8 [8]).
 */
int olfgpu_set_phase_timing(int64_t context, int enable);
int olfgpu_last_phase_times(int64_t context, double* out8);

/*
 * Device-resident start states (no counterpart in the reference): while x0FullDevice is set (non-null), every solve
 * of the context takes its per-scenario start states from that device array [nScenarios][n] on the context's GPU
 * (e.g. a learned start predicted on the device) instead of the host x0Full argument; null switches back.  The array
 * must stay valid and unchanged while a solve runs.
 */
int olfgpu_set_device_start(int64_t context, const double* x0FullDevice);

/*
 * Fallback start (no counterpart in the reference): with enable = 1, a solve given both x0Full (e.g. learned starts)
 * and x0Base first keeps, per scenario, whichever of its x0Full row and x0Base has the smaller initial max |F|; then
 * every scenario whose solve from its x0Full row ends DIVERGED, MAX_ITERATION_REACHED or LINEAR_SOLVE_FAILED restarts
 * once from x0Base, inside the same batch (its result, iterations and status are those of the restarted solve; total
 * iterations count both).  Not available with reactive limits.  olfgpu_last_fallbacks writes per scenario 0 (its own
 * start), 1 (restarted from x0Base after failing) or 2 (x0Base chosen before iterating) into fellBack [nScenarios]
 * (may be null), and the count of non-zero entries.
 */
int olfgpu_set_fallback_start(int64_t context, int enable);
/* Fallback mode (no counterpart in the reference): a scenario that converged from its own x0Full row with max |F|
 * above polishRatio * tol (default
 * 1e-2; 0 switches it off) takes one more Newton step.  A state that met the tolerance may lie anywhere in its ball
 * (on a 9,241-bus grid up to 1.5e-8 from the solution at max |F| just under 1e-8), so a scenario that converged from
 * another start than the reference's base start is brought next to the solution, where the base-start trajectory's
 * converged state also lies.  Its iteration count includes the step. */
int olfgpu_set_start_polish(int64_t context, double polishRatio);

/* Device-resident Newton loop (level schedules 0, 3, 4, 5; no counterpart in the reference, whose driver loop reads
 * the lane counts on the host every iteration): with enable = 1 a solve runs its whole Newton loop as ONE graph launch.
 * A conditional WHILE node runs an iteration per pass, and conditional IF / WHILE nodes take the host loop's decisions
 * between the iteration's phases (lanes left, lanes factorizing, refinement steps, FP64 refactor, scoring).  Small
 * kernels set them from the lane counts.  The iteration counter caps the loop as the host loop does.  Results are
 * identical to the host-driven loop. */
int olfgpu_set_device_loop(int64_t context, int enable);
int olfgpu_last_fallbacks(int64_t context, unsigned char* fellBack, int* count);

/*
 * Uneven batching across grids (no counterpart in the reference, whose GpuBatchedAcSecurityAnalysis runs one network
 * per batch).  olfgpu_stage_batch_context validates a request and uploads its inputs exactly as
 * olfgpu_solve_batch_context does, without running it.  A multi-grid context groups batch contexts of different
 * structures on one device and one precision; olfgpu_solve_multi_context runs every member's staged batch through ONE
 * persistent launch (one CTA per tile of lanesPerTile lanes of any member, the whole Newton loop with reactive limits
 * inside; captured with the result gathers in a CUDA graph) and writes member i's results into outs[i]
 * ([nScenarios_i][n_i + 3], as olfgpu_solve_batch_context; null skips the copy); deviceMs receives the device time
 * from the first install to the last result.  Members' olfgpu_last_solve_stats report their per-scenario iterations
 * afterwards.  olfgpu_set_multi_schedule fixes the tile (lanesPerTile 1, 2, 4 or 8; threads 256 or 512; order 0 as
 * given, 1 the grids with the most buses first), or lanesPerTile 0: ONE graph launch whose branches are the members'
 * device-resident Newton loops (olfgpu_set_device_loop) under their own level schedules, which run concurrently on the
 * device (any plan, outer loop and precision policy a member supports alone).  With lanesPerTile -1 the next solve
 * times every candidate and keeps the fastest.  olfgpu_get_multi_schedule reports the schedule in force and the
 * timings {lanesPerTile, threads, order, ms} of the last autotune.
 */
int olfgpu_stage_batch_context(int64_t context, const double* x0Base, const double* x0Full, const double* targetBase,
                               const int* baseRowMode, int nRowModeEntries, const int* rowModeEntries,
                               int nScenarios, int nElements, const unsigned char* disabled, int nTargetOverrides,
                               const int* targetOverrideIndex, const double* targetOverrideValue, int maxIter,
                               double tol, double reactiveLimitTol, int maxOuter, int maxPqPvSwitch);
int olfgpu_create_multi_context(int nContexts, const int64_t* contexts, int64_t* multiOut);
int olfgpu_destroy_multi_context(int64_t multi);
int olfgpu_set_multi_schedule(int64_t multi, int lanesPerTile, int threads, int order);
int olfgpu_get_multi_schedule(int64_t multi, int* lanesPerTile, int* threads, int* order, int maxResults,
                              double* results, int* nResults);
int olfgpu_solve_multi_context(int64_t multi, double* const* outs, float* deviceMs);

/*
 * Test surface of the engine (the role BatchedLuNative plays for the reference's LU, BatchedLuNative.java:121-125):
 * the Jacobian values in the reference-compatible CSR layout and the mismatch of each scenario at the states xFull
 * [nScenarios][n], through the engine's fill; and a batched linear solve J z = rhs through the engine's block LU
 * (precision 0 FP64, 1 FP32), csrVals [nScenarios][nnz], rhs and out [nScenarios][n].
 */
int olfgpu_debug_fill(int64_t context, const double* xFull, const double* targetBase, const int* baseRowMode,
                      const unsigned char* disabled, double* jacobianOut, double* mismatchOut);
int olfgpu_debug_linear_solve(int64_t context, const double* csrVals, const double* rhs, int precision, double* out);

/*
 * Post-contingency violation screening of the context's last solve on the device (sa/olf_gpu_violations.cu:160-361;
 * GpuViolationScreen.java).  Branch limits: nElem limited elements (elemId: closed branch e, or open branch nCb + e),
 * each with the limit groups [groupPtr[r], groupPtr[r + 1]) (groupSide 1 / 2; groupQty 0 current I = hypot(p, q) / v,
 * 1 active power |P|, 2 apparent power S), each group with thresholds limThreshold[limPtr[g] .. limPtr[g + 1]) in the
 * order the caller reports them.  Bus limits: busVRow (-1 none), busHigh / busLow (NaN: no limit); realistic != 0 also
 * flags the buses outside [minV, maxV].  A limit is a candidate once its value exceeds the threshold relaxed by band
 * (relative); a group's later thresholds stop being candidates once one is exceeded beyond the band; an outaged branch
 * yields nothing.  records [nScenarios][capacity] receives each scenario's candidate ids, sorted (branch limit l: l;
 * bus i high: nLimits + 2i, low: nLimits + 2i + 1, realistic: nLimits + 2 nBus + i), counts [nScenarios] their count
 * (above capacity: truncated).  The host re-tests candidates exactly; the screen never decides.
 */
int olfgpu_screen_violations(int64_t context, int nElem, const int* elemId, const int* groupPtr, const int* groupSide,
                             const int* groupQty, const int* limPtr, const double* limThreshold, int nBus,
                             const int* busVRow, const double* busHigh, const double* busLow, int realistic,
                             double minV, double maxV, double band, int capacity, int* records, int* counts);

/*
 * BatchedLuNative.factorizeAndSolveTransposed (BatchedLuNative.java:121-125; lu/transposed_solve.cuh:1-30): one block-LU
 * factorization of each scenario's J (csrVals [nScenarios][nnz], the reference-compatible CSR layout), then both
 * J x = rhs and the transposed (adjoint) system J^T y = rhsTransposed on the same factors, the latter as two more
 * triangular sweeps (U^T forward, L^T backward).  rhs / rhsTransposed and solution / solutionTransposed are
 * [nScenarios][n]; a null right-hand side skips its solve.  precision 0 FP64, 1 FP32 factors.
 */
int olfgpu_linear_solve_transposed(int64_t context, const double* csrVals, const double* rhs,
                                   const double* rhsTransposed, int precision, double* solution,
                                   double* solutionTransposed);

/*
 * Learned warm start (no counterpart in the reference): kernels of a message-passing graph network over the bus
 * graph, BF16 weights and activations with FP32 accumulation, on caller-owned device buffers, enqueued on `stream`.
 * Row-major matrices; M rows = samples x buses.
 *   gemm:     Y = [A1 | A2] . W (+ bias), z = relu ? max(Y, 0) : Y (saved to saveZ if given), out = z (+ residual);
 *             shapes (K1, K2, N) in {(16,0,64), (64,0,128), (64,64,64), (64,0,16), (128,0,64)}; fifth-generation
 *             tensor cores (tcgen05.mma, FP32 accumulators in tensor memory, 128-row tiles).  Its completion wait is
 *             bounded; olfgpu_gnn_tc_timeouts reads how many tiles gave up waiting since the library was loaded
 *             (synchronises the device; always 0 on a working GPU).
 *   gemm_dw:  dW = [A1 | A2]^T dZ and db = column sums of dZ, summed over at most maxChunks row chunks in a fixed order
 *             (partial holds maxChunks * (K * N + N) floats); shapes (16,0,64), (64,0,128), (64,64,64), (64,0,16).
 *   copy_cols: dst[r, dstCol0 + c] (+)= src[r, srcCol0 + c], FP32.
 *   message_forward:  agg[b, i] = sum over directed edges e = (j -> i) not in sample b's outaged branch of
 *             relu(P[b, j] + Q[b, i] + C[e] + bmsg), PQ rows = [P | Q] (128 BF16), agg rows 64 BF16.
 *   message_backward: dPQ (FP32) and dC (FP32, summed over samples) of the same, by recomputation.
 *   edge_project (C = Es . We) and its backward; relu_grad; adam (FP32 master weights, BF16 copy and transpose);
 *   mse (loss partials and its gradient).
 * olfgpu_gnn_last_error() reports the calling thread's last failure of these functions.
 */
const char* olfgpu_gnn_last_error(void);
int olfgpu_gnn_tc_timeouts(int* count);
int olfgpu_gnn_gemm(int M, int K1, int K2, int N, const void* A1, const void* A2, const void* W, const float* bias,
                    int relu, const void* residual, void* outBf16, float* outF32, int ldo, void* saveZ, void* stream);
int olfgpu_gnn_gemm_dw(int M, int K1, int K2, int N, const void* A1, const void* A2, const void* dZ, float* dW,
                       float* db, float* partial, int maxChunks, void* stream);
int olfgpu_gnn_message_forward(int B, int nb, const int* inPtr, const int* inEdge, const int* edgeSrc,
                               const int* edgeBranch, const int* outage, const void* PQ, const float* C,
                               const float* bmsg, void* agg, void* stream);
int olfgpu_gnn_message_backward(int B, int nb, int nEdges, const int* inPtr, const int* inEdge, const int* outPtr,
                                const int* outEdge, const int* edgeSrc, const int* edgeDst, const int* edgeBranch,
                                const int* outage, const void* PQ, const float* C, const float* bmsg,
                                const float* dAgg, float* dPQ, float* dC, void* stream);
int olfgpu_gnn_edge_project(int nEdges, const float* Es, const float* We, float* C, void* stream);
int olfgpu_gnn_edge_project_backward(int nEdges, const float* Es, const float* dC, float* dWe, float* dbmsg,
                                     void* stream);
int olfgpu_gnn_relu_grad(long long count, int N, int ldd, const float* dOut, const void* z, void* dz, float* dzF32,
                         void* stream);
int olfgpu_gnn_adam(int count, int K, int N, float* w, const float* grad, float* m, float* v, float lr, float beta1,
                    float beta2, float eps, int step, void* wBf16, void* wTBf16, void* stream);
int olfgpu_gnn_mse(int M, int ldo, const float* out, const float* target, float* dOut, float* partial, void* stream);
int olfgpu_gnn_copy_cols(int M, int ncols, const float* src, int lds, int srcCol0, float* dst, int ldd, int dstCol0,
                         int accumulate, void* stream);
/*
 * Learned start states on the device (no counterpart in the reference): x0 [nScenarios][2 nb] (device) from the network's output pred
 * [nScenarios * nb][ldPred] (columns 0, 1: normalised dVm, dVa), de-normalised by stdVm / stdVa and added to the base
 * state xBase [2 nb]; rows flagged in identity [2 nb] take target [2 nb].  All pointers are device memory.
 */
int olfgpu_gnn_compose_start(int nScenarios, int nb, const float* pred, int ldPred, double stdVm, double stdVa,
                             const double* xBase, const unsigned char* identity, const double* target, double* x0,
                             void* stream);

/*
 * Learned-start inference restricted to the buses an outage can reach (no counterpart in the reference): a
 * message-passing layer only moves
 * information one hop, so after L layers a sample differs from the outage-free sample only within L hops of its
 * outaged branch.  The compact rows (sample rowSample[r], bus rowNode[r]) hold those buses; rowOf [nSamples * nb]
 * maps (sample, bus) to its row or -1, and a neighbour outside the rows reads the outage-free sample's PQbase row
 * (identical there).  olfgpu_gnn_message_forward_compact is olfgpu_gnn_message_forward on those rows, with the same
 * edges, order and arithmetic; olfgpu_gnn_compose_start_compact writes every scenario's start from the outage-free
 * prediction predBase [nb][ldPred], then its rows from predRows [R][ldPred].  olfgpu_gnn_compact_inputs builds the
 * rows' node inputs x [R][16] (BF16) from the outage-free inputs xBase [nb][16]: at an end of the scenario's outaged
 * branch o (branchFrom[o], branchTo[o]) column nFeat is 1 and the next two hold flows[o][0..1] (float32), negated at
 * the to end; it also sets rowOf[rowSample[r] * nb + rowNode[r]] = r (the caller fills rowOf with -1 first).  Device
 * pointers throughout.
 */
int olfgpu_gnn_message_forward_compact(int R, int nb, const int* rowNode, const int* rowSample, const int* rowOf,
                                       const int* inPtr, const int* inEdge, const int* edgeSrc, const int* edgeBranch,
                                       const int* outage, const void* PQ, const void* PQbase, const float* C,
                                       const float* bmsg, void* agg, void* stream);
int olfgpu_gnn_compact_inputs(int R, int nb, int nFeat, const int* rowNode, const int* rowSample, const int* outage,
                              const int* branchFrom, const int* branchTo, const void* xBase, const float* flows, void* x,
                              int* rowOf, void* stream);
int olfgpu_gnn_compose_start_compact(int nScenarios, int nb, const float* predBase, const float* predRows, int ldPred,
                                     int R, const int* rowNode, const int* rowSample, double stdVm, double stdVa,
                                     const double* xBase, const unsigned char* identity, const double* target,
                                     double* x0, void* stream);

/*
 * Batched linear solve J z = rhs that allocates no memory (this entry point has no counterpart in the reference).
 * It is for callers that cannot allocate device memory while they solve: a host whose GPU memory is reserved up front
 * and handed out by someone else (a JVM or service that sized its pools at start-up), or a code path that must not
 * call cudaMalloc / cudaFree because those calls synchronise the whole device.  The caller passes device buffers:
 * csrValsDevice [nScenarios][nnz] (the reference-compatible CSR layout of olfgpu_structure_export), rhsDevice and
 * outDevice [nScenarios][n]; precision 0 factors in FP64, 1 in FP32.  The work is enqueued on `stream` (a
 * cudaStream_t, null for the legacy default stream) and the call returns without waiting for it.
 * Scratch: one fixed 64 MiB device array inside the library, which every GPU that loads the library holds until the
 * process exits; a batch whose Jacobian, factors and work vectors do not fit is rejected with an error naming the
 * largest batch that fits.  The structure must already be on the current device (creating a batch context on it
 * uploads it).  The first call on each device looks up the array's address (set-up, no allocation), and so does the
 * first call after the device's CUDA context was re-created (cudaDeviceReset); make that first call before any stream
 * capture.  All calls share the one array and it keeps the previous call's contents (what must start at zero is
 * cleared on every call): calls whose work overlaps on the GPU race, so order them on one stream.  A scenario whose
 * factorization meets a (near-)singular 2x2 pivot gets NaN in every entry of its outDevice row.
 */
int olfgpu_linear_solve_noalloc(int64_t structure, int nScenarios, const double* csrValsDevice,
                                const double* rhsDevice, double* outDevice, int precision, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* OLFGPU_B200_H */
