// JNI layer of the engine: the native methods of the reference's Java facades for the batched AC Newton-Raphson path
// (StructureNative, BatchSolveNative, NewtonSettingsNative, ReactiveLimitsNative, DistributedSlackNative, DriverNative,
// BatchReadbackNative),
// with the reference's symbol names and argument lists (native/cuda/jni/*_jni.cu), forwarded to the C ABI of
// include/olfgpu_b200.h.  Built as lib/libolfgpu.so, the name the Java side loads (GpuNativeLoader.java:32).
//
// Java arrays are read with Get*ArrayRegion (never written back); results are new Java arrays.  A C ABI failure
// becomes a java/lang/RuntimeException whose message carries olfgpu_last_error() and the call returns 0 / null, as the
// reference's JNI layer reports native failures (structure_jni.cu:128-137, batch_solve_jni.cu:302-306).  A handle of 0
// is a no-op on destroy.  Per-scenario problems are status codes in the result rows, never exceptions.
#include "jni.h"

#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/olfgpu_b200.h"

namespace {

#define OLF_JNI(pkg, cls, m) Java_com_powsybl_openloadflow_##pkg##_##cls##_##m

void throwRuntime(JNIEnv* env, const std::string& what) {
    jclass cls = olfjni_FindClass(env, "java/lang/RuntimeException");
    if (cls) olfjni_ThrowNew(env, cls, what.c_str());
}

// rc != 0: the C ABI call failed; raise its reason in Java.  Returns whether the call succeeded.
bool ok(JNIEnv* env, int rc, const char* what) {
    if (rc == 0) return true;
    throwRuntime(env, std::string(what) + " failed: " + olfgpu_last_error());
    return false;
}

jsize lengthOf(JNIEnv* env, jarray a) { return a ? olfjni_GetArrayLength(env, a) : 0; }

std::vector<jint> ints(JNIEnv* env, jintArray a) {
    std::vector<jint> v(lengthOf(env, a));
    if (!v.empty()) olfjni_GetIntArrayRegion(env, a, 0, static_cast<jsize>(v.size()), v.data());
    return v;
}

std::vector<jdouble> doubles(JNIEnv* env, jdoubleArray a) {
    std::vector<jdouble> v(lengthOf(env, a));
    if (!v.empty()) olfjni_GetDoubleArrayRegion(env, a, 0, static_cast<jsize>(v.size()), v.data());
    return v;
}

std::vector<jbyte> bytes(JNIEnv* env, jbyteArray a) {
    std::vector<jbyte> v(lengthOf(env, a));
    if (!v.empty()) olfjni_GetByteArrayRegion(env, a, 0, static_cast<jsize>(v.size()), v.data());
    return v;
}

template <typename T>
const T* ptr(const std::vector<T>& v) {
    return v.empty() ? nullptr : v.data();
}

template <typename T>
int len(const std::vector<T>& v) {
    return static_cast<int>(v.size());
}

// NewtonSettingsNative.setLinearSolverSettings is process-wide in the reference (gLinearSolver); kept here so
// readLinearSolverSettings returns what was set.  The engine has its own block-LU plan (minimum degree with a dense
// front), which every structure this layer creates uses whatever batchedLuOrdering says.
struct LinearSolverSettings {
    int reorder = 0, matching = 0, pivotType = 0;
    double pivotThreshold = 0.0;
    int refinementBaseSteps = 0, refinementMaxSteps = 0;
    double refinementTolerance = 0.0;
    int batchedLuOrdering = 0;
    bool splitLongRows = false;
};
LinearSolverSettings gSettings;

// NewtonSettingsNative.setBatchX0Seeds per context: (local scenario * n + row, value) pairs written over the tiled
// base state of the next solve that is given no full per-scenario state, and consumed by that solve either way
// (scenario_install.cu:57-74).
struct X0Seeds {
    std::vector<jint> index;
    std::vector<jdouble> value;
};
std::mutex gSeedsMutex;
std::map<jlong, X0Seeds> gSeeds;

X0Seeds takeSeeds(jlong handle) {
    std::lock_guard<std::mutex> lock(gSeedsMutex);
    X0Seeds out;
    auto it = gSeeds.find(handle);
    if (it != gSeeds.end()) {
        out = std::move(it->second);
        gSeeds.erase(it);
    }
    return out;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------------------------------------------
// StructureNative (structure_jni.cu:7-180)
// ---------------------------------------------------------------------------------------------------------------
JNIEXPORT jlong JNICALL OLF_JNI(ac_equations_vector_gpu, StructureNative, createStructure)(
    JNIEnv* env, jclass, jint n, jdoubleArray jClosedBranchParameters, jintArray jClosedBranchIndices,
    jdoubleArray jOpenBranchParameters, jintArray jOpenBranchIndices, jdoubleArray jShuntParameters,
    jintArray jShuntIndices, jdoubleArray jHvdcAcEmulationParameters, jintArray jHvdcAcEmulationIndices,
    jintArray jDistrQElement, jintArray jDistrQSide, jdoubleArray jDistrQWeight, jintArray jDistrQRow,
    jintArray jDistrQKind, jdoubleArray jZeroImpedanceBranchParameters, jintArray jZeroImpedanceBranchIndices,
    jintArray jDistrRhoRow, jintArray jDistrRhoColumn, jdoubleArray jDistrRhoCoefficient, jintArray jDistrShuntBRow,
    jintArray jDistrShuntBColumn, jdoubleArray jDistrShuntBCoefficient, jintArray jClosedBranchPhaseControlSide,
    jdoubleArray jLoadModelParameters, jintArray jLoadModelIndices, jintArray jReactiveRelocationGroupStart,
    jintArray jReactiveRelocationCandidateRows, jintArray jOpenBranchAlternateReactiveDestination,
    jintArray jZeroImpedanceBranchAlternateReactiveDestination, jintArray jReactiveRelocationDependentBaseGroup,
    jintArray jReactiveRelocationBaseTargetRow, jintArray jReactiveRelocationDependentGroupOfRow,
    jintArray jIdentityRows) {
    const auto cbP = doubles(env, jClosedBranchParameters);
    const auto cbI = ints(env, jClosedBranchIndices);
    const auto obP = doubles(env, jOpenBranchParameters);
    const auto obI = ints(env, jOpenBranchIndices);
    const auto shP = doubles(env, jShuntParameters);
    const auto shI = ints(env, jShuntIndices);
    const auto hvP = doubles(env, jHvdcAcEmulationParameters);
    const auto hvI = ints(env, jHvdcAcEmulationIndices);
    const auto dqE = ints(env, jDistrQElement);
    const auto dqS = ints(env, jDistrQSide);
    const auto dqW = doubles(env, jDistrQWeight);
    const auto dqR = ints(env, jDistrQRow);
    const auto dqK = ints(env, jDistrQKind);
    const auto zP = doubles(env, jZeroImpedanceBranchParameters);
    const auto zI = ints(env, jZeroImpedanceBranchIndices);
    const auto drR = ints(env, jDistrRhoRow);
    const auto drC = ints(env, jDistrRhoColumn);
    const auto drK = doubles(env, jDistrRhoCoefficient);
    const auto dbR = ints(env, jDistrShuntBRow);
    const auto dbC = ints(env, jDistrShuntBColumn);
    const auto dbK = doubles(env, jDistrShuntBCoefficient);
    const auto pcs = ints(env, jClosedBranchPhaseControlSide);
    const auto lmP = doubles(env, jLoadModelParameters);
    const auto lmI = ints(env, jLoadModelIndices);
    const auto rrG = ints(env, jReactiveRelocationGroupStart);
    const auto rrC = ints(env, jReactiveRelocationCandidateRows);
    const auto obA = ints(env, jOpenBranchAlternateReactiveDestination);
    const auto zA = ints(env, jZeroImpedanceBranchAlternateReactiveDestination);
    const auto rrB = ints(env, jReactiveRelocationDependentBaseGroup);
    const auto rrT = ints(env, jReactiveRelocationBaseTargetRow);
    const auto rrD = ints(env, jReactiveRelocationDependentGroupOfRow);
    const auto idr = ints(env, jIdentityRows);
    int64_t h = 0;
    const int rc = olfgpu_create_structure_full(
        n, ptr(cbP), len(cbP), ptr(cbI), len(cbI), ptr(obP), len(obP), ptr(obI), len(obI), ptr(shP), len(shP),
        ptr(shI), len(shI), ptr(hvP), len(hvP), ptr(hvI), len(hvI), ptr(dqE), len(dqE), ptr(dqS), len(dqS), ptr(dqW),
        len(dqW), ptr(dqR), len(dqR), ptr(dqK), len(dqK), ptr(zP), len(zP), ptr(zI), len(zI), ptr(drR), len(drR),
        ptr(drC), len(drC), ptr(drK), len(drK), ptr(dbR), len(dbR), ptr(dbC), len(dbC), ptr(dbK), len(dbK), ptr(pcs),
        len(pcs), ptr(lmP), len(lmP), ptr(lmI), len(lmI), ptr(rrG), len(rrG), ptr(rrC), len(rrC), ptr(obA), len(obA),
        ptr(zA), len(zA), ptr(rrB), len(rrB), ptr(rrT), len(rrT), ptr(rrD), len(rrD), ptr(idr), len(idr),
        16 | 3 /* minimum degree toward a shallow elimination tree, dense-front block-LU plan: the engine's fastest */, &h);
    return ok(env, rc, "GPU structure creation") ? static_cast<jlong>(h) : 0;
}

JNIEXPORT void JNICALL OLF_JNI(ac_equations_vector_gpu, StructureNative, destroyStructure)(JNIEnv*, jclass,
                                                                                         jlong handle) {
    if (handle) olfgpu_destroy_structure(handle);
}

JNIEXPORT jint JNICALL OLF_JNI(ac_equations_vector_gpu, StructureNative, recommendBatchSize)(JNIEnv*, jclass,
                                                                                           jlong handle, jint maxCap,
                                                                                           jint mode) {
    int batch = 1;
    if (olfgpu_recommend_batch_size(handle, maxCap, mode, &batch) != 0) batch = 1;   // a failed query: the safest
    return batch;
}

// ---------------------------------------------------------------------------------------------------------------
// BatchSolveNative (batch_solve_jni.cu:29-465)
// ---------------------------------------------------------------------------------------------------------------
JNIEXPORT jlong JNICALL OLF_JNI(ac_solver_gpu, BatchSolveNative, createBatchContext)(
    JNIEnv* env, jclass, jlong structureHandle, jint nScenarios, jint mode, jintArray jReactiveLimitVoltageRow,
    jdoubleArray jReactiveLimitMinQ, jdoubleArray jReactiveLimitMaxQ, jdoubleArray jReactiveLimitLoadQ,
    jdoubleArray jReactiveLimitTargetV, jbyteArray jReactiveLimitFlags, jdoubleArray jRowSlope,
    jintArray jDistributedSlackBusPhiRow, jdoubleArray jDistributedSlackBusFactor, jint slackBusPhiRow,
    jdouble slackBusTargetP, jdoubleArray jDistributedSlackBusBaseTargetP, jdoubleArray jDistributedSlackBusMaxDelta,
    jdoubleArray jDistributedSlackBusMinDelta, jint distributedSlackFactorMode,
    jdoubleArray jDistributedSlackBusMarginUp, jdoubleArray jDistributedSlackBusMarginDown, jdouble slackBusMarginUp,
    jdouble slackBusMarginDown) {
    const auto vr = ints(env, jReactiveLimitVoltageRow);
    const auto mn = doubles(env, jReactiveLimitMinQ);
    const auto mx = doubles(env, jReactiveLimitMaxQ);
    const auto lq = doubles(env, jReactiveLimitLoadQ);
    const auto tv = doubles(env, jReactiveLimitTargetV);
    const auto fl = bytes(env, jReactiveLimitFlags);
    const auto sl = doubles(env, jRowSlope);
    const auto dsR = ints(env, jDistributedSlackBusPhiRow);
    const auto dsF = doubles(env, jDistributedSlackBusFactor);
    const auto dsB = doubles(env, jDistributedSlackBusBaseTargetP);
    const auto dsX = doubles(env, jDistributedSlackBusMaxDelta);
    const auto dsN = doubles(env, jDistributedSlackBusMinDelta);
    const auto dsU = doubles(env, jDistributedSlackBusMarginUp);
    const auto dsD = doubles(env, jDistributedSlackBusMarginDown);
    int64_t h = 0;
    const int rc = olfgpu_create_batch_context_full(
        structureHandle, nScenarios, mode, ptr(vr), len(vr), ptr(mn), len(mn), ptr(mx), len(mx), ptr(lq), len(lq),
        ptr(tv), len(tv), reinterpret_cast<const signed char*>(ptr(fl)), len(fl), ptr(sl), len(sl), ptr(dsR), len(dsR),
        ptr(dsF), len(dsF), slackBusPhiRow, slackBusTargetP, ptr(dsB), len(dsB), ptr(dsX), len(dsX), ptr(dsN),
        len(dsN), distributedSlackFactorMode, ptr(dsU), len(dsU), ptr(dsD), len(dsD), slackBusMarginUp,
        slackBusMarginDown, &h);
    if (!ok(env, rc, "GPU batched context creation")) return 0;
    // the narrow levels of every phase in shared memory: the engine's fastest schedule for the dense-front plan
    if (!ok(env, olfgpu_set_schedule(h, 4, 0, 256), "GPU batched context creation")) {
        olfgpu_destroy_batch_context(h);
        return 0;
    }
    return static_cast<jlong>(h);
}

JNIEXPORT void JNICALL OLF_JNI(ac_solver_gpu, BatchSolveNative, destroyBatchContext)(JNIEnv*, jclass, jlong handle) {
    if (!handle) return;
    takeSeeds(handle);
    olfgpu_destroy_batch_context(handle);
}

JNIEXPORT void JNICALL OLF_JNI(ac_solver_gpu, BatchSolveNative, setBatchStatesToHost)(JNIEnv*, jclass, jlong handle,
                                                                                    jboolean statesToHost) {
    if (handle) olfgpu_set_states_to_host(handle, statesToHost == JNI_TRUE ? 1 : 0);
}

JNIEXPORT jintArray JNICALL OLF_JNI(ac_solver_gpu, BatchSolveNative, readBatchHandedBackSlots)(JNIEnv* env, jclass,
                                                                                             jlong handle) {
    if (!handle) return nullptr;
    int count = 0;
    if (!ok(env, olfgpu_read_handed_back_slots(handle, nullptr, 0, &count), "readBatchHandedBackSlots")) return nullptr;
    std::vector<int> slots(count);
    if (!ok(env, olfgpu_read_handed_back_slots(handle, slots.data(), count, &count), "readBatchHandedBackSlots")) {
        return nullptr;
    }
    jintArray arr = olfjni_NewIntArray(env, count);
    if (arr && count) olfjni_SetIntArrayRegion(env, arr, 0, count, slots.data());
    return arr;
}

JNIEXPORT void JNICALL OLF_JNI(ac_solver_gpu, BatchSolveNative, beginBatchInstall)(JNIEnv* env, jclass, jlong handle,
                                                                                 jintArray jBankSlots) {
    if (!handle) return;
    const auto slots = ints(env, jBankSlots);
    ok(env, olfgpu_begin_batch_install(handle, ptr(slots), len(slots)), "beginBatchInstall");
}

JNIEXPORT jobjectArray JNICALL OLF_JNI(ac_solver_gpu, BatchSolveNative, solveBatchContext)(
    JNIEnv* env, jclass, jlong handle, jdoubleArray jx0Base, jdoubleArray jtargetBase, jintArray jrowModeEntries,
    jintArray jbaseRowMode, jobjectArray jdisabledMask, jintArray jtargetOverrideIndex,
    jdoubleArray jtargetOverrideValue, jintArray jDistributedSlackOverrideBus,
    jdoubleArray jDistributedSlackOverrideFactorDelta, jdoubleArray jDistributedSlackOverrideBaseTargetPDelta,
    jdoubleArray jDistributedSlackOverrideMaxDelta, jdoubleArray jDistributedSlackOverrideMinDelta,
    jdoubleArray jDistributedSlackBusAnchorShift, jdoubleArray jSlackBusAnchorShift,
    jintArray jReactiveLimitTargetVOverrideScenarioEntry, jdoubleArray jReactiveLimitTargetVOverrideValue,
    jintArray jReactiveLimitDeltaOverrideScenarioEntry, jdoubleArray jReactiveLimitDeltaOverrideValues,
    jintArray jReactiveCapabilityCurveOverrideScenarioCurve, jdoubleArray jReactiveCapabilityCurveOverrideStepScale,
    jint maxIter, jdouble tol, jdouble reactiveLimitTol, jdouble slackDistTol, jdouble convEpsPerEq,
    jint stateVectorScalingMode, jdouble maxDv, jdouble maxDphi, jintArray jvarType, jdoubleArray jx0Full,
    jintArray jShuntOvSlotElem, jdoubleArray jShuntOvGb, jintArray jReactiveLimitsSeedState, jintArray jR1OvSlotElem,
    jdoubleArray jR1OvVal, jint maxOuterProductive, jint maxPqPvSwitch, jint rejectSlackDistributionFailure,
    jint skipReactiveLimitsPhase, jint nBaseClosedZeroImpedanceBranches,
    jintArray jZeroImpedanceBranchCloseScenarioElement, jintArray jZeroImpedanceBranchOpenScenarioElement,
    jint pauseAtEnded) {
    int n = 0, nElements = 0, bank = 0, installed = 0;
    if (!ok(env, olfgpu_context_info(handle, &n, &nElements, &bank, &installed, nullptr, nullptr),
            "GPU batched Newton-Raphson")) {
        return nullptr;
    }
    const auto x0 = doubles(env, jx0Base);
    const auto tg = doubles(env, jtargetBase);
    const auto rme = ints(env, jrowModeEntries);
    const auto brm = ints(env, jbaseRowMode);
    const auto toi = ints(env, jtargetOverrideIndex);
    const auto tov = doubles(env, jtargetOverrideValue);
    const auto a1 = ints(env, jDistributedSlackOverrideBus);
    const auto a2 = doubles(env, jDistributedSlackOverrideFactorDelta);
    const auto a3 = doubles(env, jDistributedSlackOverrideBaseTargetPDelta);
    const auto a4 = doubles(env, jDistributedSlackOverrideMaxDelta);
    const auto a5 = doubles(env, jDistributedSlackOverrideMinDelta);
    const auto a6 = doubles(env, jDistributedSlackBusAnchorShift);
    const auto a7 = doubles(env, jSlackBusAnchorShift);
    const auto a8 = ints(env, jReactiveLimitTargetVOverrideScenarioEntry);
    const auto a9 = doubles(env, jReactiveLimitTargetVOverrideValue);
    const auto a10 = ints(env, jReactiveLimitDeltaOverrideScenarioEntry);
    const auto a11 = doubles(env, jReactiveLimitDeltaOverrideValues);
    const auto a12 = ints(env, jReactiveCapabilityCurveOverrideScenarioCurve);
    const auto a13 = doubles(env, jReactiveCapabilityCurveOverrideStepScale);
    const auto vt = ints(env, jvarType);
    auto xf = doubles(env, jx0Full);
    const auto so = ints(env, jShuntOvSlotElem);
    const auto sg = doubles(env, jShuntOvGb);
    const auto rs = ints(env, jReactiveLimitsSeedState);
    const auto r1 = ints(env, jR1OvSlotElem);
    const auto rv = doubles(env, jR1OvVal);
    const auto zc = ints(env, jZeroImpedanceBranchCloseScenarioElement);
    const auto zo = ints(env, jZeroImpedanceBranchOpenScenarioElement);
    // the disabled mask, one boolean row per installed scenario (a shorter row is padded with false), one region copy
    // per row: a jboolean is an unsigned byte holding 0 or 1, the mask's own encoding (batch_solve_jni.cu:216-228)
    const int nS = lengthOf(env, jdisabledMask);
    std::vector<unsigned char> dis(static_cast<size_t>(nS) * nElements, 0);
    for (int s = 0; s < nS; s++) {
        jobject row = olfjni_GetObjectArrayElement(env, jdisabledMask, s);
        const int rl = row ? olfjni_GetArrayLength(env, row) : 0;
        const int k = rl < nElements ? rl : nElements;
        if (k > 0) olfjni_GetBooleanArrayRegion(env, row, 0, k, dis.data() + static_cast<size_t>(s) * nElements);
        if (row) olfjni_DeleteLocalRef(env, row);
    }
    // start seeds (setBatchX0Seeds) over the tiled base state when no full per-scenario state is given; consumed
    // by this solve either way
    const X0Seeds seeds = takeSeeds(handle);
    if (xf.empty() && !seeds.index.empty()) {
        if (static_cast<int>(x0.size()) != n) {
            throwRuntime(env, "GPU batched Newton-Raphson failed: x0Base must hold n values to take start seeds");
            return nullptr;
        }
        xf.resize(static_cast<size_t>(nS) * n);
        for (int s2 = 0; s2 < nS; s2++) std::memcpy(&xf[static_cast<size_t>(s2) * n], x0.data(), sizeof(double) * n);
        for (size_t k = 0; k < seeds.index.size(); k++) {
            const jint idx = seeds.index[k];
            if (idx < 0 || static_cast<int64_t>(idx) >= static_cast<int64_t>(nS) * n) {
                throwRuntime(env, "GPU batched Newton-Raphson failed: setBatchX0Seeds index " + std::to_string(idx) +
                                      " outside the " + std::to_string(nS) + " installed scenarios");
                return nullptr;
            }
            xf[idx] = seeds.value[k];
        }
    }
    std::vector<double> out(static_cast<size_t>(nS) * (n + 3));
    const int rc = olfgpu_solve_batch_context_full(
        handle, ptr(x0), len(x0), ptr(tg), len(tg), ptr(rme), len(rme), ptr(brm), len(brm), ptr(dis), nS, nElements,
        ptr(toi), len(toi), ptr(tov), len(tov), ptr(a1), len(a1), ptr(a2), len(a2), ptr(a3), len(a3), ptr(a4), len(a4),
        ptr(a5), len(a5), ptr(a6), len(a6), ptr(a7), len(a7), ptr(a8), len(a8), ptr(a9), len(a9), ptr(a10), len(a10),
        ptr(a11), len(a11), ptr(a12), len(a12), ptr(a13), len(a13), maxIter, tol, reactiveLimitTol, slackDistTol,
        convEpsPerEq, stateVectorScalingMode, maxDv, maxDphi, ptr(vt), len(vt), ptr(xf), len(xf), ptr(so), len(so),
        ptr(sg), len(sg), ptr(rs), len(rs), ptr(r1), len(r1), ptr(rv), len(rv), maxOuterProductive, maxPqPvSwitch,
        rejectSlackDistributionFailure, skipReactiveLimitsPhase, nBaseClosedZeroImpedanceBranches, ptr(zc), len(zc),
        ptr(zo), len(zo), pauseAtEnded, out.data());
    if (!ok(env, rc, "GPU batched Newton-Raphson")) return nullptr;
    // the row width follows setBatchStatesToHost: [x(n), iterations, ||F||inf, status] or the three last alone
    int statesToHost = 1;
    if (olfgpu_states_to_host(handle, &statesToHost) != 0) statesToHost = 1;
    const int width = statesToHost ? n + 3 : 3;
    jclass rowClass = olfjni_FindClass(env, "[D");
    // a null allocation means the Java heap is exhausted and an OutOfMemoryError is pending: return and let it surface
    jobjectArray result = olfjni_NewObjectArray(env, nS, rowClass, nullptr);
    if (!result) return nullptr;
    for (int j = 0; j < nS; j++) {
        jdoubleArray row = olfjni_NewDoubleArray(env, width);
        if (!row) return nullptr;
        olfjni_SetDoubleArrayRegion(env, row, 0, width, out.data() + static_cast<size_t>(j) * width);
        olfjni_SetObjectArrayElement(env, result, j, row);
        olfjni_DeleteLocalRef(env, row);
    }
    return result;
}

// ---------------------------------------------------------------------------------------------------------------
// NewtonSettingsNative (newton_settings_jni.cu:11-43)
// ---------------------------------------------------------------------------------------------------------------
JNIEXPORT void JNICALL OLF_JNI(ac_solver_gpu, NewtonSettingsNative, setLinearSolverSettings)(
    JNIEnv*, jclass, jint reorder, jint matching, jint pivotType, jdouble pivotThreshold,
    jint iterativeRefinementBaseSteps, jint iterativeRefinementMaxSteps, jdouble iterativeRefinementTolerance,
    jint batchedLuOrdering, jboolean batchedLuSplitLongRows) {
    gSettings.reorder = reorder;
    gSettings.matching = matching;
    gSettings.pivotType = pivotType;
    gSettings.pivotThreshold = pivotThreshold;
    gSettings.refinementBaseSteps = iterativeRefinementBaseSteps;
    gSettings.refinementMaxSteps = iterativeRefinementMaxSteps;
    gSettings.refinementTolerance = iterativeRefinementTolerance;
    gSettings.batchedLuOrdering = batchedLuOrdering;
    gSettings.splitLongRows = batchedLuSplitLongRows == JNI_TRUE;
}

JNIEXPORT jdoubleArray JNICALL OLF_JNI(ac_solver_gpu, NewtonSettingsNative, readLinearSolverSettings)(JNIEnv* env,
                                                                                                    jclass) {
    const double v[9] = {static_cast<double>(gSettings.reorder), static_cast<double>(gSettings.matching),
                         static_cast<double>(gSettings.pivotType), gSettings.pivotThreshold,
                         static_cast<double>(gSettings.refinementBaseSteps),
                         static_cast<double>(gSettings.refinementMaxSteps), gSettings.refinementTolerance,
                         static_cast<double>(gSettings.batchedLuOrdering), gSettings.splitLongRows ? 1.0 : 0.0};
    jdoubleArray out = olfjni_NewDoubleArray(env, 9);
    if (out) olfjni_SetDoubleArrayRegion(env, out, 0, 9, v);
    return out;
}

// ---------------------------------------------------------------------------------------------------------------
// ReactiveLimitsNative (reactive_limits_jni.cu:118-195)
// ---------------------------------------------------------------------------------------------------------------
JNIEXPORT void JNICALL OLF_JNI(ac_outerloop_gpu, ReactiveLimitsNative, setBatchReactiveLimitStrongestPvKeys)(
    JNIEnv* env, jclass, jlong handle, jdoubleArray jNomV, jintArray jPRow, jdoubleArray jStaticP, jintArray jIdRank) {
    if (!handle || !jNomV || !jPRow || !jStaticP || !jIdRank) return;
    const auto nv = doubles(env, jNomV);
    const auto pr = ints(env, jPRow);
    const auto sp = doubles(env, jStaticP);
    const auto ir = ints(env, jIdRank);
    if (nv.size() != pr.size() || nv.size() != sp.size() || nv.size() != ir.size()) {
        throwRuntime(env, "setBatchReactiveLimitStrongestPvKeys: array length != nReactiveLimitEntries");
        return;
    }
    ok(env, olfgpu_set_reactive_limit_strongest_pv_keys(handle, ptr(nv), ptr(pr), ptr(sp), ptr(ir), len(nv)),
       "setBatchReactiveLimitStrongestPvKeys");
}

JNIEXPORT void JNICALL OLF_JNI(ac_outerloop_gpu, ReactiveLimitsNative, setBatchRealisticCheck)(
    JNIEnv* env, jclass, jlong handle, jbyteArray jRowChecked, jdouble minV, jdouble maxV, jint enabled,
    jint fixingLoop) {
    (void)fixingLoop;   // the realistic-voltage fixing loop is not modelled: the check alone
    if (!handle) return;
    int n = 0;
    if (!ok(env, olfgpu_context_info(handle, &n, nullptr, nullptr, nullptr, nullptr, nullptr), "setBatchRealisticCheck")) {
        return;
    }
    if (!enabled || !jRowChecked) {
        ok(env, olfgpu_set_realistic_check(handle, nullptr, minV, maxV, 0), "setBatchRealisticCheck");
        return;
    }
    const auto rc = bytes(env, jRowChecked);
    if (len(rc) != n) {
        throwRuntime(env, "setBatchRealisticCheck: array length != n");
        return;
    }
    ok(env, olfgpu_set_realistic_check(handle, reinterpret_cast<const unsigned char*>(rc.data()), minV, maxV, 1),
       "setBatchRealisticCheck");
}

// ---------------------------------------------------------------------------------------------------------------
// DriverNative (driver_jni.cu:11-18), BatchReadbackNative (batch_readback_jni.cu:13-45, 103-118)
// ---------------------------------------------------------------------------------------------------------------
JNIEXPORT void JNICALL OLF_JNI(ac_solver_gpu, DriverNative, setBatchOuterLoops)(JNIEnv* env, jclass, jlong handle,
                                                                              jboolean distributedSlackOuterLoop,
                                                                              jboolean reactiveLimitsOuterLoop) {
    if (!handle) return;
    ok(env, olfgpu_set_outer_loops(handle, distributedSlackOuterLoop == JNI_TRUE ? 1 : 0,
                                   reactiveLimitsOuterLoop == JNI_TRUE ? 1 : 0),
       "setBatchOuterLoops");
}

JNIEXPORT jint JNICALL OLF_JNI(ac_solver_gpu, BatchReadbackNative, readBatchNewtonLoopIterations)(JNIEnv*, jclass,
                                                                                                jlong handle) {
    int it = 0;
    return handle && olfgpu_context_info(handle, nullptr, nullptr, nullptr, nullptr, &it, nullptr) == 0 ? it : -1;
}

JNIEXPORT jlong JNICALL OLF_JNI(ac_solver_gpu, BatchReadbackNative, readBatchSolveCount)(JNIEnv*, jclass,
                                                                                       jlong handle) {
    int64_t count = 0;
    return handle && olfgpu_context_info(handle, nullptr, nullptr, nullptr, nullptr, nullptr, &count) == 0 ? count
                                                                                                          : -1;
}

}  // extern "C"

namespace {

// The bank slots whose rows the per-scenario readbacks return, in row order: the last solve's (its handed-back
// slots), or the whole bank before any solve (batch_readback_jni.cu reads the installed slots the same way).  n
// receives the row width.  False (a Java exception pending) on a failure.
bool readbackSlots(JNIEnv* env, jlong handle, const char* what, std::vector<int>& slots, int& n) {
    int count = 0, nS = 0;
    if (!ok(env, olfgpu_context_info(handle, &n, nullptr, &nS, nullptr, nullptr, nullptr), what)) return false;
    if (!ok(env, olfgpu_read_handed_back_slots(handle, nullptr, 0, &count), what)) return false;
    if (count == 0) {
        slots.resize(nS);
        for (int j = 0; j < nS; j++) slots[j] = j;
        return true;
    }
    slots.resize(count);
    return ok(env, olfgpu_read_handed_back_slots(handle, slots.data(), count, &count), what);
}

}  // namespace

extern "C" {

// BatchReadbackNative.readBatchTargets (batch_readback_jni.cu:13-24): [slots x n] targets as the last solve ended.
JNIEXPORT jdoubleArray JNICALL OLF_JNI(ac_solver_gpu, BatchReadbackNative, readBatchTargets)(JNIEnv* env, jclass,
                                                                                           jlong handle) {
    if (!handle) return nullptr;
    std::vector<int> slots;
    int n = 0;
    if (!readbackSlots(env, handle, "readBatchTargets", slots, n)) return nullptr;
    std::vector<double> host(slots.size() * static_cast<size_t>(n));
    if (!ok(env, olfgpu_read_batch_targets(handle, len(slots), ptr(slots), host.data()), "readBatchTargets")) {
        return nullptr;
    }
    jdoubleArray out = olfjni_NewDoubleArray(env, static_cast<jsize>(host.size()));
    if (out && !host.empty()) olfjni_SetDoubleArrayRegion(env, out, 0, static_cast<jsize>(host.size()), host.data());
    return out;
}

// BatchReadbackNative.readBatchRowModes (batch_readback_jni.cu:26-45): [slots x n] row modes as the last solve ended.
JNIEXPORT jintArray JNICALL OLF_JNI(ac_solver_gpu, BatchReadbackNative, readBatchRowModes)(JNIEnv* env, jclass,
                                                                                         jlong handle) {
    if (!handle) return nullptr;
    std::vector<int> slots;
    int n = 0;
    if (!readbackSlots(env, handle, "readBatchRowModes", slots, n)) return nullptr;
    std::vector<int> host(slots.size() * static_cast<size_t>(n));
    if (!ok(env, olfgpu_read_batch_row_modes(handle, len(slots), ptr(slots), host.data()), "readBatchRowModes")) {
        return nullptr;
    }
    jintArray out = olfjni_NewIntArray(env, static_cast<jsize>(host.size()));
    if (out && !host.empty()) olfjni_SetIntArrayRegion(env, out, 0, static_cast<jsize>(host.size()), host.data());
    return out;
}


// ---------------------------------------------------------------------------------------------------------------
// The rest of the native methods the SPI path (GpuNewtonRaphson.java) and the batched SA (GpuBatchChunkSolver.java)
// call on every run, so that the Java side links against this library: settings this engine applies, the reference's
// own answer for a context without the feature (null read-backs, ignored anchors), and an exception naming the input
// where a caller hands in data of a family this engine does not model.
// ---------------------------------------------------------------------------------------------------------------

// NewtonSettingsNative.setBatchX0Seeds (newton_settings_jni.cu:42-63): start values over the base state of the next
// solve given no full per-scenario state (flat index local scenario * n + row); null or empty clears them.
JNIEXPORT void JNICALL OLF_JNI(ac_solver_gpu, NewtonSettingsNative, setBatchX0Seeds)(JNIEnv* env, jclass,
                                                                                   jlong handle, jintArray jIdx,
                                                                                   jdoubleArray jVal) {
    if (!handle) return;
    X0Seeds seeds;
    if (jIdx && jVal) {
        seeds.index = ints(env, jIdx);
        seeds.value = doubles(env, jVal);
        if (seeds.index.size() != seeds.value.size()) {
            throwRuntime(env, "setBatchX0Seeds failed: index and value arrays differ in length");
            return;
        }
    }
    std::lock_guard<std::mutex> lock(gSeedsMutex);
    if (seeds.index.empty()) gSeeds.erase(handle);
    else gSeeds[handle] = std::move(seeds);
}

// NewtonSettingsNative.setBatchRowCriteria / setBatchRowCriteriaAlternate (newton_settings_jni.cu:80-120): null
// clears the per-row stopping thresholds, which this engine never holds (its test is OLF's infinity-norm or 2-norm
// rule); thresholds (OLF's PerEquationTypeStoppingCriteria) are refused.
JNIEXPORT void JNICALL OLF_JNI(ac_solver_gpu, NewtonSettingsNative, setBatchRowCriteria)(
    JNIEnv* env, jclass, jlong handle, jdoubleArray jFixedVariableRowMaxMismatch, jdoubleArray jEquationRowMaxMismatch) {
    if (!handle || !jFixedVariableRowMaxMismatch || !jEquationRowMaxMismatch) return;
    throwRuntime(env, "setBatchRowCriteria failed: per-equation-type stopping criteria are not supported by this engine");
}

JNIEXPORT void JNICALL OLF_JNI(ac_solver_gpu, NewtonSettingsNative, setBatchRowCriteriaAlternate)(
    JNIEnv* env, jclass, jlong handle, jdoubleArray jAlternateRowMaxMismatch, jintArray jSelector) {
    if (!handle || !jAlternateRowMaxMismatch || !jSelector) return;
    throwRuntime(env,
                 "setBatchRowCriteriaAlternate failed: per-equation-type stopping criteria are not supported by this engine");
}

// NewtonSettingsNative.setBatchActiveRowCounts: the active equation count of OLF's 2-norm threshold per scenario.
// Every row of the families this engine models is active, so null, or a count of n for every scenario, is what it
// already uses; a smaller count (islanded buses, rho/a1 identities) is refused.
JNIEXPORT void JNICALL OLF_JNI(ac_solver_gpu, NewtonSettingsNative, setBatchActiveRowCounts)(JNIEnv* env, jclass,
                                                                                           jlong handle,
                                                                                           jintArray jActive) {
    if (!handle || !jActive) return;
    int n = 0;
    if (!ok(env, olfgpu_context_info(handle, &n, nullptr, nullptr, nullptr, nullptr, nullptr), "setBatchActiveRowCounts")) {
        return;
    }
    for (jint a : ints(env, jActive)) {
        if (a != n) {
            throwRuntime(env, "setBatchActiveRowCounts failed: an active equation count below n (islanded buses or "
                              "rho/a1 identities) is not supported by this engine");
            return;
        }
    }
}

// NewtonSettingsNative.setBatchFrozenRows: the rows an islanding outage froze; null or empty clears (islanding
// outages are not batched by this engine, so there are none to hold).
JNIEXPORT void JNICALL OLF_JNI(ac_solver_gpu, NewtonSettingsNative, setBatchFrozenRows)(JNIEnv* env, jclass,
                                                                                      jlong handle, jintArray jSlotRow) {
    if (!handle || lengthOf(env, jSlotRow) == 0) return;
    throwRuntime(env, "setBatchFrozenRows failed: islanding outages are not supported by this engine");
}

// NewtonSettingsNative.setBatchLineSearch: the LINE_SEARCH state-vector scaling is not modelled (NONE and
// MAX_VOLTAGE_CHANGE are); the Java side calls this only for that mode.
JNIEXPORT void JNICALL OLF_JNI(ac_solver_gpu, NewtonSettingsNative, setBatchLineSearch)(JNIEnv* env, jclass,
                                                                                      jlong handle, jint, jdouble) {
    if (!handle) return;
    throwRuntime(env, "setBatchLineSearch failed: LINE_SEARCH state-vector scaling is not supported by this engine");
}

// NewtonSettingsNative.setBatchLoopTraceSlot: the reference's print-only outer-loop trace channel; nothing to print
// here, and a trace never changes a result.
JNIEXPORT void JNICALL OLF_JNI(ac_solver_gpu, NewtonSettingsNative, setBatchLoopTraceSlot)(JNIEnv*, jclass, jlong,
                                                                                         jint) {}

// DistributedSlackNative.setBatchDistributedSlackGeneratorAnchors (distributed_slack_jni.cu:26-42): per scenario and
// participating GENERATOR; this engine's participants are buses (olfgpu_create_batch_context_full), so only null or
// empty arrays fit its zero generators.
JNIEXPORT void JNICALL OLF_JNI(ac_outerloop_gpu, DistributedSlackNative, setBatchDistributedSlackGeneratorAnchors)(
    JNIEnv* env, jclass, jlong handle, jdoubleArray jAnchor, jdoubleArray jStart, jdoubleArray jSeedAnchor) {
    if (!handle) return;
    if (lengthOf(env, jAnchor) || lengthOf(env, jStart) || lengthOf(env, jSeedAnchor)) {
        throwRuntime(env, "setBatchDistributedSlackGeneratorAnchors failed: per-generator distributed-slack "
                          "participants are not supported by this engine (its participants are buses)");
    }
}

// DistributedSlackNative.setBatchSlackOnlyAnchor (distributed_slack_jni.cu:12-19): the reference installs it only
// for a slack-only distribution and ignores it otherwise; this engine never runs one.
JNIEXPORT void JNICALL OLF_JNI(ac_outerloop_gpu, DistributedSlackNative, setBatchSlackOnlyAnchor)(JNIEnv*, jclass,
                                                                                                jlong, jdoubleArray) {}

// ReactiveLimitsNative.setBatchForcedTargetQPre (reactive_limits_jni.cu:108-116): ignored without forced-target-Q
// entries, as in the reference; this engine has none.
JNIEXPORT void JNICALL OLF_JNI(ac_outerloop_gpu, ReactiveLimitsNative, setBatchForcedTargetQPre)(JNIEnv*, jclass,
                                                                                               jlong, jdoubleArray) {}

// ReactiveLimitsNative.setBatchReactiveLimitSeedTargetQ (reactive_limits_jni.cu:368-376): per-scenario seeded target
// Q of the entries (a strategy pair's continuation); null or empty clears, values are refused.
JNIEXPORT void JNICALL OLF_JNI(ac_outerloop_gpu, ReactiveLimitsNative, setBatchReactiveLimitSeedTargetQ)(
    JNIEnv* env, jclass, jlong handle, jdoubleArray jTargets) {
    if (!handle || lengthOf(env, jTargets) == 0) return;
    throwRuntime(env, "setBatchReactiveLimitSeedTargetQ failed: seeded reactive-limit targets are not supported by "
                      "this engine");
}

// ReactiveLimitsNative.readBatchReactiveLimitsFinalState (reactive_limits_jni.cu:407-427): [slots x entries] of
// limit type | switch count << 3, the last solve's slots; null without reactive-limit entries.
JNIEXPORT jintArray JNICALL OLF_JNI(ac_outerloop_gpu, ReactiveLimitsNative, readBatchReactiveLimitsFinalState)(
    JNIEnv* env, jclass, jlong handle) {
    if (!handle) return nullptr;
    int nRl = 0;
    if (!ok(env, olfgpu_read_reactive_limits_state(handle, 0, nullptr, nullptr, &nRl),
            "readBatchReactiveLimitsFinalState") || nRl == 0) {
        return nullptr;
    }
    std::vector<int> slots;
    int n = 0;
    if (!readbackSlots(env, handle, "readBatchReactiveLimitsFinalState", slots, n)) return nullptr;
    std::vector<int> host(slots.size() * static_cast<size_t>(nRl));
    if (!ok(env, olfgpu_read_reactive_limits_state(handle, len(slots), ptr(slots), host.data(), nullptr),
            "readBatchReactiveLimitsFinalState")) {
        return nullptr;
    }
    jintArray out = olfjni_NewIntArray(env, static_cast<jsize>(host.size()));
    if (out && !host.empty()) olfjni_SetIntArrayRegion(env, out, 0, static_cast<jsize>(host.size()), host.data());
    return out;
}

// BatchReadbackNative read-backs of what this engine does not track: the reference answers null for a context
// without per-generator distributed-slack participants (batch_readback_jni.cu:64-79), without a slack-only
// distribution (:50-62) or its retained share (:138-150), without the per-pass statistics (:81-101) and without the
// last converged state (:121-136), and its callers take null as "none" (GpuNewtonRaphson.java:381 then counts the
// solve's own iterations).
JNIEXPORT jdoubleArray JNICALL OLF_JNI(ac_solver_gpu, BatchReadbackNative, readBatchDistributedSlackGeneratorMove)(
    JNIEnv*, jclass, jlong) {
    return nullptr;
}

JNIEXPORT jdoubleArray JNICALL OLF_JNI(ac_solver_gpu, BatchReadbackNative, readBatchSlackRetainedShare)(JNIEnv*,
                                                                                                      jclass, jlong) {
    return nullptr;
}

JNIEXPORT jdoubleArray JNICALL OLF_JNI(ac_solver_gpu, BatchReadbackNative, readBatchSlackAbsorbed)(JNIEnv*, jclass,
                                                                                                jlong) {
    return nullptr;
}

JNIEXPORT jintArray JNICALL OLF_JNI(ac_solver_gpu, BatchReadbackNative, readBatchOuterLoopStats)(JNIEnv*, jclass,
                                                                                              jlong) {
    return nullptr;
}

JNIEXPORT jdoubleArray JNICALL OLF_JNI(ac_solver_gpu, BatchReadbackNative, readBatchLastConvergedState)(JNIEnv*,
                                                                                                     jclass, jlong,
                                                                                                     jint) {
    return nullptr;
}

}  // extern "C"
