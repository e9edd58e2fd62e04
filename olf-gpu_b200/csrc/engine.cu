// Batched Newton-Raphson engine: device copy of a structure, batch contexts and the solve driver.
#include "engine.hpp"

#include <algorithm>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>

namespace olfb200 {

// ---------------------------------------------------------------------------------------------------------------
// Device copy of a structure
// ---------------------------------------------------------------------------------------------------------------
std::shared_ptr<DeviceNet> uploadNet(const Structure& s) {
    auto d = std::make_shared<DeviceNet>();
    OLF_CUDA(cudaGetDevice(&d->device));
    const BlockPlan& p = s.plan;
    const int nb = s.nb;
    auto aBlock = [&](int i, int j) {
        auto b = p.aCol.begin() + p.aPtr[i], e = p.aCol.begin() + p.aPtr[i + 1];
        auto it = std::lower_bound(b, e, j);
        if (it == e || *it != j) throw std::runtime_error("A block lookup miss");
        return static_cast<int>(it - p.aCol.begin());
    };
    // incident closed-branch sides per node, sorted by (neighbour, element)
    std::vector<std::vector<Side>> sides(nb);
    for (int e = 0; e < s.ncb; e++) {
        const int* ix = &s.cbIx[static_cast<size_t>(e) * CB_INDICES];
        const int i = s.colNode[ix[4]] >> 1, j = s.colNode[ix[6]] >> 1;
        if (i == j) throw std::runtime_error("closed branch " + std::to_string(e) + " has both ends on one bus");
        sides[i].push_back(Side{e, 0, j, aBlock(i, j)});
        sides[j].push_back(Side{e, 1, i, aBlock(j, i)});
    }
    std::vector<int> sidePtr(nb + 1, 0);
    std::vector<Side> sideAll;
    for (int i = 0; i < nb; i++) {
        std::sort(sides[i].begin(), sides[i].end(), [](const Side& a, const Side& b) {
            return a.neighbour != b.neighbour ? a.neighbour < b.neighbour : a.element < b.element;
        });
        sideAll.insert(sideAll.end(), sides[i].begin(), sides[i].end());
        sidePtr[i + 1] = static_cast<int>(sideAll.size());
    }
    std::vector<double2> trig(s.ncb);
    for (int e = 0; e < s.ncb; e++) {
        const double ksi = s.cbPar[static_cast<size_t>(e) * CB_PARAMS + 5];
        trig[e] = make_double2(std::sin(ksi), std::cos(ksi));
    }
    std::vector<std::vector<int>> shOf(nb);
    for (int e = 0; e < s.nsh; e++) shOf[s.colNode[s.shIx[static_cast<size_t>(e) * SH_INDICES + 2]] >> 1].push_back(e);
    std::vector<int> shPtr(nb + 1, 0), shList;
    for (int i = 0; i < nb; i++) {
        shList.insert(shList.end(), shOf[i].begin(), shOf[i].end());
        shPtr[i + 1] = static_cast<int>(shList.size());
    }
    std::vector<std::vector<int2>> obOf(nb);
    for (int e = 0; e < s.nob; e++) {
        const int* ix = &s.obIx[static_cast<size_t>(e) * OB_INDICES];
        if (ix[4] >= 0) obOf[s.colNode[ix[4]] >> 1].push_back(make_int2(e, 0));
        else if (ix[5] >= 0) obOf[s.colNode[ix[5]] >> 1].push_back(make_int2(e, 1));
    }
    std::vector<int> obPtr(nb + 1, 0);
    std::vector<int2> obList;
    for (int i = 0; i < nb; i++) {
        obList.insert(obList.end(), obOf[i].begin(), obOf[i].end());
        obPtr[i + 1] = static_cast<int>(obList.size());
    }
    // factorization tasks
    const int nLu = p.nU + p.nL;
    std::vector<Task> task(nLu);
    for (int k = 0; k < nb; k++) {
        for (int t = p.uPtr[k]; t < p.uPtr[k + 1]; t++) {
            task[t] = Task{p.luToA[t], p.opPtr[t], p.opPtr[t + 1], t == p.uPtr[k] ? -2 : -1};
        }
        for (int t = p.lPtr[k]; t < p.lPtr[k + 1]; t++) {
            const int id = p.nU + t;
            task[id] = Task{p.luToA[id], p.opPtr[id], p.opPtr[id + 1], p.uPtr[k]};
        }
    }
    // dense front: a front block's level task applies its updates from before the front and stores the partial sum
    // (diag -3: no inversion, no scaling); the dense front kernel finishes it
    for (int id : p.frontBlocks)
        if (id >= 0) task[id] = Task{p.luToA[id], p.opPtr[id], p.opOuterEnd[id], -3};
    // L blocks by row position (for the forward solve), ascending column position
    std::vector<std::vector<int2>> lr(nb);
    for (int k = 0; k < nb; k++)
        for (int t = p.lPtr[k]; t < p.lPtr[k + 1]; t++) lr[p.lRow[t]].push_back(make_int2(p.nU + t, k));
    std::vector<int> lrowPtr(nb + 1, 0);
    std::vector<int2> lrow;
    for (int i = 0; i < nb; i++) {
        lrow.insert(lrow.end(), lr[i].begin(), lr[i].end());
        lrowPtr[i + 1] = static_cast<int>(lrow.size());
    }
    // CSR slot -> A block entry
    d->csrToA.assign(s.nnz, -1);
    for (int r = 0; r < s.n; r++) {
        const int nr = s.colNode[r];
        for (int k = s.rowPtr[r]; k < s.rowPtr[r + 1]; k++) {
            const int nc = s.colNode[s.colIdx[k]];
            d->csrToA[k] = aBlock(nr >> 1, nc >> 1) * 4 + (nr & 1) * 2 + (nc & 1);
        }
    }
    d->csrToAD.upload(d->csrToA);
    d->nodeCol.upload(s.nodeCol);
    d->sidePtr.upload(sidePtr);
    d->side.upload(sideAll);
    d->cbPar.upload(s.cbPar);
    d->cbTrig.upload(trig);
    d->aPtr.upload(p.aPtr);
    d->aCol.upload(p.aCol);
    d->aDiag.upload(p.aDiag);
    d->shPtr.upload(shPtr);
    d->shList.upload(shList);
    d->shPar.upload(s.shPar);
    d->obPtr.upload(obPtr);
    d->obList.upload(obList);
    d->obPar.upload(s.obPar);
    d->task.upload(task);
    std::vector<int4> ops(p.opL.size());
    for (size_t q = 0; q < ops.size(); q++) ops[q] = make_int4(p.opL[q], p.opU[q], p.opD[q], 0);
    d->levelTask.upload(p.levelTask);
    d->perm.upload(p.perm);
    d->iperm.upload(p.iperm);
    d->lrowPtr.upload(lrowPtr);
    // forward-solve row ends: a dense-front row's level task stops at its first front column (the dense front solve
    // applies the rest); lrow lists ascend in column
    std::vector<int> lrowEnd(nb);
    for (int i = 0; i < nb; i++) {
        int q = lrowPtr[i + 1];
        if (i >= p.frontStart) {
            q = lrowPtr[i];
            while (q < lrowPtr[i + 1] && lrow[q].y < p.frontStart) q++;
        }
        lrowEnd[i] = q;
    }
    d->lrowEnd.upload(lrowEnd);
    d->lrow.upload(lrow);
    d->uPtr.upload(p.uPtr);
    d->uCol.upload(p.uCol);
    d->fwdPos.upload(p.fwdLevelPos);
    d->bwdPos.upload(p.bwdLevelPos);
    d->levelPtr = p.levelPtr;
    d->fwdPtr = p.fwdLevelPtr;
    d->bwdPtr = p.bwdLevelPtr;
    // split factor of each level (a power of two <= 16): enough threads per task that each walks at most ~12
    // updates of a factorization task, ~8 blocks of a solve row.  Measured on the 9,241-bus / 500-outage batch
    // (FP64 step): at most 4 -> 18.3 ms, 2 -> 23.4 ms, 8 -> 16.6 ms, 12 / 8 -> 16.5 ms, 16 -> 17.4 ms: fewer, longer
    // threads cost fewer waves and smaller reductions, until a task's walk becomes the level's critical path.
    auto splitOf = [](int longest, int walk) {
        int P = 1;
        while (P < 16 && (longest + P - 1) / P > walk) P *= 2;
        return P;
    };
    std::vector<int> lrowLen(nb, 0);
    for (int i = 0; i < nb; i++) lrowLen[i] = lrowPtr[i + 1] - lrowPtr[i];
    d->levelSplit.assign(p.levelPtr.size() - 1, 1);
    for (size_t l = 0; l + 1 < p.levelPtr.size(); l++) {
        int m = 0;
        for (int q = p.levelPtr[l]; q < p.levelPtr[l + 1]; q++) {
            const int t = p.levelTask[q];
            m = std::max(m, p.opPtr[t + 1] - p.opPtr[t]);
        }
        d->levelSplit[l] = splitOf(m, 12);
    }
    d->fwdSplit.assign(p.fwdLevelPtr.size() - 1, 1);
    for (size_t l = 0; l + 1 < p.fwdLevelPtr.size(); l++) {
        int m = 0;
        for (int q = p.fwdLevelPtr[l]; q < p.fwdLevelPtr[l + 1]; q++) m = std::max(m, lrowLen[p.fwdLevelPos[q]]);
        d->fwdSplit[l] = splitOf(m, 8);
    }
    // longest update list per level (the persistent kernel sizes its per-level split from it)
    std::vector<int> levelLongest(p.levelPtr.size() - 1, 0), fwdLongest(p.fwdLevelPtr.size() - 1, 0),
        bwdLongest(p.bwdLevelPtr.size() - 1, 0);
    for (size_t l = 0; l + 1 < p.levelPtr.size(); l++)
        for (int q = p.levelPtr[l]; q < p.levelPtr[l + 1]; q++) {
            const int t = p.levelTask[q];
            levelLongest[l] = std::max(levelLongest[l], p.opPtr[t + 1] - p.opPtr[t]);
        }
    for (size_t l = 0; l + 1 < p.fwdLevelPtr.size(); l++)
        for (int q = p.fwdLevelPtr[l]; q < p.fwdLevelPtr[l + 1]; q++)
            fwdLongest[l] = std::max(fwdLongest[l], lrowLen[p.fwdLevelPos[q]]);
    for (size_t l = 0; l + 1 < p.bwdLevelPtr.size(); l++)
        for (int q = p.bwdLevelPtr[l]; q < p.bwdLevelPtr[l + 1]; q++) {
            const int i = p.bwdLevelPos[q];
            bwdLongest[l] = std::max(bwdLongest[l], p.uPtr[i + 1] - p.uPtr[i] - 1);
        }
    d->levelPtrD.upload(p.levelPtr);
    d->levelLongestD.upload(levelLongest);
    d->fwdPtrD.upload(p.fwdLevelPtr);
    d->fwdLongestD.upload(fwdLongest);
    d->bwdPtrD.upload(p.bwdLevelPtr);
    d->bwdLongestD.upload(bwdLongest);
    d->persistent.nLevels = static_cast<int>(p.levelPtr.size()) - 1;
    d->persistent.nFwd = static_cast<int>(p.fwdLevelPtr.size()) - 1;
    d->persistent.nBwd = static_cast<int>(p.bwdLevelPtr.size()) - 1;
    d->persistent.levelPtr = d->levelPtrD.as<int>();
    d->persistent.levelLongest = d->levelLongestD.as<int>();
    d->persistent.fwdPtr = d->fwdPtrD.as<int>();
    d->persistent.fwdLongest = d->fwdLongestD.as<int>();
    d->persistent.fwdPos = d->fwdPos.as<int>();
    d->persistent.bwdPtr = d->bwdPtrD.as<int>();
    d->persistent.bwdLongest = d->bwdLongestD.as<int>();
    d->persistent.bwdPos = d->bwdPos.as<int>();
    // the narrow levels: the factorization / forward tail and the backward head whose levels hold <= NARROW tasks
    constexpr int NARROW = 48;
    auto countOf = [](const std::vector<int>& ptr, size_t l) { return ptr[l + 1] - ptr[l]; };
    // (a dense-front plan ends with the front's assembly level, wide whatever the tree above it: it stays a level
    // launch after the range)
    d->factorTo = static_cast<int>(p.levelPtr.size()) - 1 - (p.frontF > 0 ? 1 : 0);
    d->factorFrom = d->factorTo;
    while (d->factorFrom > 0 && countOf(p.levelPtr, d->factorFrom - 1) <= NARROW) d->factorFrom--;
    // the shared-memory region: the narrow factorization levels before factorTo whose blocks fit REGION_BYTES (FP64,
    // one lane: two CTAs per SM); every block they produce gets a slot, in level order, and every update its operands'
    // slots in ops.w (slot + 1 of the L block in the low 16 bits, of the U block in the high 16 bits, 0 outside).
    // Deferred-L plans keep the range launches (their updates also read the pivot's inverse).
    constexpr size_t REGION_BYTES = 110 * 1024;
    d->regionFrom = d->factorTo;
    if (!p.deferredL) {
        d->regionFrom = d->factorFrom;
        while (d->regionFrom < d->factorTo &&
               static_cast<size_t>(p.levelPtr[d->factorTo] - p.levelPtr[d->regionFrom]) * 32 > REGION_BYTES) {
            d->regionFrom++;
        }
    }
    for (int l = d->regionFrom; l < d->factorTo; l++) {   // one round of the CTA per level
        if (p.levelPtr[l + 1] - p.levelPtr[l] > REGION_THREADS) d->regionFrom = l + 1;
    }
    d->regionBase = p.levelPtr[d->regionFrom];
    d->regionSlots = p.levelPtr[d->factorTo] - d->regionBase;
    if (d->regionSlots > 0) {
        std::vector<int> slotOf(nLu, -1);
        for (int k = 0; k < d->regionSlots; k++) slotOf[p.levelTask[d->regionBase + k]] = k;
        for (size_t q = 0; q < ops.size(); q++) {
            ops[q].w = (slotOf[p.opL[q]] + 1) | ((slotOf[p.opU[q]] + 1) << 16);
        }
        // per slot: (task, end of its updates, first update with an operand in the region, pivot code: -2 pivot,
        // -1 / -3 stored as summed, >= 0 the inverted pivot's block outside the region, <= -4 its slot -4 - code).
        // A slot task's updates with both operands outside the region go first (each group in ascending pivot
        // order): the prefix kernel applies them, coalesced over the lanes, before the region starts.
        std::vector<int4> rtask(d->regionSlots);
        for (int k = 0; k < d->regionSlots; k++) {
            const int t = p.levelTask[d->regionBase + k];
            const Task& tk = task[t];
            std::stable_partition(ops.begin() + tk.opBegin, ops.begin() + tk.opEnd,
                                  [](const int4& o) { return o.w == 0; });
            int mid = tk.opBegin;
            while (mid < tk.opEnd && ops[mid].w == 0) mid++;
            int diag = tk.diag;
            if (diag >= 0 && slotOf[diag] >= 0) diag = -4 - slotOf[diag];
            rtask[k] = make_int4(t, tk.opEnd, mid, diag);
        }
        d->regionTask.upload(rtask);
        // the limit for the largest region any plan can have (one process may hold several structures)
        OLF_CUDA(prepareRegion(static_cast<int>(REGION_BYTES / 32), static_cast<int>(REGION_BYTES / 32)));
    }
    d->ops.upload(ops);
    // (a solve range up to 256 rows per level measured slower: a tile walked the backward sweep's wide middle levels at
    // 1 ms per solve, against 0.8 ms as level launches)
    d->fwdFrom = static_cast<int>(p.fwdLevelPtr.size()) - 1;
    while (d->fwdFrom > 0 && countOf(p.fwdLevelPtr, d->fwdFrom - 1) <= NARROW) d->fwdFrom--;
    d->bwdUntil = 0;
    while (d->bwdUntil < static_cast<int>(p.bwdLevelPtr.size()) - 1 && countOf(p.bwdLevelPtr, d->bwdUntil) <= NARROW) {
        d->bwdUntil++;
    }
    // shared-memory solve regions: slot k of the forward tail holds position fwdLevelPos[fwdRegionBase + k], of the
    // backward head position bwdLevelPos[k]; each L / U entry of a region row carries its column's slot + 1 (0: a
    // column outside the region, final in global memory before the region's launch).  Both fit far below the default
    // 48 KB of shared memory on these grids; a larger one is left to the level launches.
    {
        constexpr int SOLVE_REGION_SLOTS = 2048;
        const int nFwd = static_cast<int>(p.fwdLevelPtr.size()) - 1;
        d->fwdRegionBase = p.fwdLevelPtr[d->fwdFrom];
        d->fwdRegionSlots = p.fwdLevelPtr[nFwd] - d->fwdRegionBase;
        d->bwdRegionSlots = p.bwdLevelPtr[d->bwdUntil];
        if (d->fwdRegionSlots > SOLVE_REGION_SLOTS) d->fwdRegionSlots = 0;
        if (d->bwdRegionSlots > SOLVE_REGION_SLOTS) d->bwdRegionSlots = 0;
        std::vector<int> slot(nb, -1);
        std::vector<int> lrowSlot(std::max<size_t>(lrow.size(), 1), 0), uSlot(std::max<size_t>(p.nU, 1), 0);
        for (int k = 0; k < d->fwdRegionSlots; k++) slot[p.fwdLevelPos[d->fwdRegionBase + k]] = k;
        // a forward-tail row's entries whose columns lie outside the region go first (each group in ascending column):
        // solvePrefixKernel applies them, coalesced over the lanes, before the region starts at fwdRegionStart[k]
        std::vector<int> fwdStart(std::max(d->fwdRegionSlots, 1), 0);
        for (int k = 0; k < d->fwdRegionSlots; k++) {
            const int i = p.fwdLevelPos[d->fwdRegionBase + k];
            std::stable_partition(lrow.begin() + lrowPtr[i], lrow.begin() + lrowEnd[i],
                                  [&](const int2& e) { return slot[e.y] < 0; });
            int q = lrowPtr[i];
            while (q < lrowEnd[i] && slot[lrow[q].y] < 0) q++;
            fwdStart[k] = q;
            for (q = lrowPtr[i]; q < lrowEnd[i]; q++) lrowSlot[q] = slot[lrow[q].y] + 1;
        }
        d->lrow.upload(lrow);
        d->fwdRegionStart.upload(fwdStart);
        std::fill(slot.begin(), slot.end(), -1);
        for (int k = 0; k < d->bwdRegionSlots; k++) slot[p.bwdLevelPos[k]] = k;
        for (int k = 0; k < d->bwdRegionSlots; k++) {
            const int i = p.bwdLevelPos[k];
            for (int q = p.uPtr[i] + 1; q < p.uPtr[i + 1]; q++) uSlot[q] = slot[p.uCol[q]] + 1;
        }
        d->lrowSlot.upload(lrowSlot);
        d->uSlot.upload(uSlot);
    }
    d->bwdSplit.assign(p.bwdLevelPtr.size() - 1, 1);
    for (size_t l = 0; l + 1 < p.bwdLevelPtr.size(); l++) {
        int m = 0;
        for (int q = p.bwdLevelPtr[l]; q < p.bwdLevelPtr[l + 1]; q++) {
            const int i = p.bwdLevelPos[q];
            m = std::max(m, p.uPtr[i + 1] - p.uPtr[i] - 1);
        }
        d->bwdSplit[l] = splitOf(m, 8);
    }
    d->levelSplitD.upload(d->levelSplit);
    d->fwdSplitD.upload(d->fwdSplit);
    d->bwdSplitD.upload(d->bwdSplit);
    d->coop = CoopPlan{static_cast<int>(p.levelPtr.size()) - 1, static_cast<int>(p.fwdLevelPtr.size()) - 1,
                       static_cast<int>(p.bwdLevelPtr.size()) - 1, d->levelPtrD.as<int>(), d->levelSplitD.as<int>(),
                       d->fwdPtrD.as<int>(), d->fwdPos.as<int>(), d->fwdSplitD.as<int>(), d->bwdPtrD.as<int>(),
                       d->bwdPos.as<int>(), d->bwdSplitD.as<int>()};
    DevNet& v = d->view;
    v.n = s.n;
    v.nb = nb;
    v.nA = static_cast<int>(p.aCol.size());
    v.nLu = nLu;
    v.nU = p.nU;
    v.deferredL = p.deferredL ? 1 : 0;
    v.frontStart = p.frontStart;
    v.frontF = p.frontF;
    if (p.frontF > 0) {
        d->frontBlocks.upload(p.frontBlocks);
        OLF_CUDA(prepareDenseFront(MAX_FRONT));   // the largest front: the limit serves every structure
    }
    v.frontBlocks = d->frontBlocks.as<int>();
    v.ncb = s.ncb;
    v.nob = s.nob;
    v.nsh = s.nsh;
    v.nElements = s.nElements;
    v.nodeCol = d->nodeCol.as<int>();
    v.sidePtr = d->sidePtr.as<int>();
    v.side = d->side.as<Side>();
    v.cbPar = d->cbPar.as<double>();
    v.cbTrig = d->cbTrig.as<double2>();
    v.aPtr = d->aPtr.as<int>();
    v.aCol = d->aCol.as<int>();
    v.aDiag = d->aDiag.as<int>();
    v.shPtr = d->shPtr.as<int>();
    v.shList = d->shList.as<int>();
    v.shPar = d->shPar.as<double>();
    v.obPtr = d->obPtr.as<int>();
    v.obList = d->obList.as<int2>();
    v.obPar = d->obPar.as<double>();
    v.task = d->task.as<Task>();
    v.ops = d->ops.as<int4>();
    v.levelTask = d->levelTask.as<int>();
    v.perm = d->perm.as<int>();
    v.iperm = d->iperm.as<int>();
    v.lrowPtr = d->lrowPtr.as<int>();
    v.lrowEnd = d->lrowEnd.as<int>();
    v.lrow = d->lrow.as<int2>();
    v.uPtr = d->uPtr.as<int>();
    v.uCol = d->uCol.as<int>();
    OLF_CUDA(cudaDeviceSynchronize());
    // the uploads above are pageable cudaMemcpy calls, whose DMA may still be in flight when they return; the
    // contexts' non-blocking streams would not wait for it
    OLF_CUDA(cudaDeviceSynchronize());
    return d;
}

// ---------------------------------------------------------------------------------------------------------------
// Batch context
// ---------------------------------------------------------------------------------------------------------------
BatchContext::~BatchContext() {
    if (graph) cudaGraphExecDestroy(graph);
    if (graphSolve) cudaGraphExecDestroy(graphSolve);
    for (cudaGraphExec_t gx : {graphFactor, graphResidual, graphCorrect, graph64, graphStep})
        if (gx) cudaGraphExecDestroy(gx);
    if (hostActive) cudaFreeHost(hostActive);
    if (countReady) cudaEventDestroy(countReady);
    if (hostBitsPinned) cudaFreeHost(hostBitsPinned);
    if (stream) cudaStreamDestroy(stream);
}

DevBatch BatchContext::batch() const {
    DevBatch b{};
    b.S = S;
    b.nS = nS;
    b.x = x.as<double>();
    b.target = target.as<double>();
    b.mode = mode.as<int8_t>();
    b.F = F.as<double>();
    b.J = J.as<double>();
    b.lu64 = lu64.as<double>();
    b.lu32 = lu32.as<float>();
    b.w64 = w64.as<double>();
    b.w32 = w32.as<float>();
    b.dx = dx.as<double>();
    b.res = res.as<double>();
    b.qbuf = qbuf.as<double>();
    b.disabled = disabled.as<uint32_t>();
    b.norm = norm.as<unsigned long long>();
    b.iter = iter.as<int>();
    b.status = status.as<int>();
    b.outer = outer.as<int>();
    b.totalIter = totalIter.as<int>();
    b.trouble = trouble.as<int>();
    b.normOut = normOut.as<double>();
    b.active = active.as<int8_t>();
    b.pending = pending.as<int8_t>();
    b.precision64 = precision64.as<int8_t>();
    b.nActive = nActive.as<int>();
    b.fallbackX = stage.as<double>();        // the staged base start x0Base
    b.nFallback = net->host.n;
    b.fallbackOn = fallbackStart && hasX0Base && hasX0Full ? 1 : 0;
    b.fallbackLeft = fallbackLeft.as<int8_t>();
    b.fellBack = fellBack.as<int8_t>();
    b.growthLimit = growthLimit;
    b.laneMask = nullptr;
    b.resNorm = resNorm.as<unsigned long long>();
    return b;
}

BatchContext* createContext(std::shared_ptr<NetStructure> net, int nScenarios, int mode, int nRl, const int* voltageRow,
                            const double* minQ, const double* maxQ, const double* loadQ, const double* targetV,
                            const double* nomV, const int* pRow, const double* staticP, const int* idRank) {
    if (nScenarios <= 0) throw std::runtime_error("nScenarios must be positive");
    if (mode != MODE_UBATCH && mode != MODE_ROBUST && mode != MODE_BATCHED_LU) {
        throw std::runtime_error("unknown linear-solve mode " + std::to_string(mode));
    }
    auto ctx = std::make_unique<BatchContext>();
    ctx->net = net;
    OLF_CUDA(cudaGetDevice(&ctx->device));
    if (!net->dev || net->dev->device != ctx->device) net->dev = uploadNet(net->host);
    const Structure& s = net->host;
    const DevNet& v = net->dev->view;
    ctx->nS = nScenarios;
    ctx->S = (nScenarios + 31) / 32 * 32;
    const size_t S = ctx->S, n = s.n;
    OLF_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    OLF_CUDA(cudaMallocHost(&ctx->hostActive, 4 * sizeof(int)));
    OLF_CUDA(cudaEventCreateWithFlags(&ctx->countReady, cudaEventDisableTiming));
    ctx->x.alloc(n * S * 8);
    ctx->target.alloc(n * S * 8);
    ctx->mode.alloc(n * S);
    ctx->F.alloc(n * S * 8);
    ctx->J.alloc(static_cast<size_t>(v.nA) * 4 * S * 8);
    ctx->w64.alloc(static_cast<size_t>(v.nb) * 2 * S * 8);
    ctx->w32.alloc(static_cast<size_t>(v.nb) * 2 * S * 4);
    ctx->dx.alloc(n * S * 8);
    ctx->res.alloc(n * S * 8);
    ctx->qbuf.alloc(n * S * 8);
    ctx->disabled.alloc(static_cast<size_t>(std::max(v.nElements, 1)) * (S / 32) * 4);
    ctx->norm.alloc(S * 8);
    ctx->iter.alloc(S * 4);
    ctx->status.alloc(S * 4);
    ctx->outer.alloc(S * 4);
    ctx->totalIter.alloc(S * 4);
    ctx->trouble.alloc(S * 4);
    ctx->normOut.alloc(S * 8);
    ctx->active.alloc(S);
    ctx->pending.alloc(S);
    ctx->precision64.alloc(S);
    ctx->fallbackLeft.alloc(S);
    ctx->resNorm.alloc(S * 8);
    ctx->fellBack.alloc(S);
    ctx->nActive.alloc(16);
    ctx->out.alloc(static_cast<size_t>(nScenarios) * (n + 3) * 8);
    ctx->stage.alloc(n * 8 * 2 + n * 4);
    ctx->cfg.maxIter = 15;
    ctx->cfg.tol = 1e-8;
    ctx->cfg.rlTol = 1e-4;
    ctx->cfg.maxOuter = 20;
    ctx->cfg.maxSwitch = 3;
    ctx->cfg.refinementSteps = 1;
    ctx->cfg.growthLimit = ctx->growthLimit;
    ctx->cfg.refineBelow = ctx->refineBelow;
    if (nRl > 0) {
        for (int i = 0; i < nRl; i++) {
            if (voltageRow[i] < 0 || voltageRow[i] >= s.n) throw std::runtime_error("bad reactiveLimitVoltageRow");
            if (pRow[i] >= s.n) throw std::runtime_error("bad reactiveLimit pRow");
        }
        auto up = [&](DeviceBuffer& d, const void* src, size_t bytes) {
            d.alloc(bytes);
            OLF_CUDA(cudaMemcpy(d.p, src, bytes, cudaMemcpyHostToDevice));
        };
        up(ctx->rlVoltageRow, voltageRow, nRl * 4);
        up(ctx->rlMinQ, minQ, nRl * 8);
        up(ctx->rlMaxQ, maxQ, nRl * 8);
        up(ctx->rlLoadQ, loadQ, nRl * 8);
        up(ctx->rlTargetV, targetV, nRl * 8);
        up(ctx->rlNomV, nomV, nRl * 8);
        up(ctx->rlPRow, pRow, nRl * 4);
        up(ctx->rlStaticP, staticP, nRl * 8);
        up(ctx->rlIdRank, idRank, nRl * 4);
        ctx->rlLimitType.alloc(nRl * S);
        ctx->rlSwitchCount.alloc(nRl * S);
        ctx->rlPassSwitched.alloc(nRl * S);
        ctx->rlSavedMode.alloc(nRl * S);
        ctx->rlSavedTarget.alloc(nRl * S * 8);
        ctx->rlRemainingPv.alloc(S * 4);
        ctx->rlSwitched.alloc(S * 4);
        DevRl& r = ctx->rl;
        r.nRl = nRl;
        r.voltageRow = ctx->rlVoltageRow.as<int>();
        r.minQ = ctx->rlMinQ.as<double>();
        r.maxQ = ctx->rlMaxQ.as<double>();
        r.loadQ = ctx->rlLoadQ.as<double>();
        r.targetV = ctx->rlTargetV.as<double>();
        r.nomV = ctx->rlNomV.as<double>();
        r.pRow = ctx->rlPRow.as<int>();
        r.staticP = ctx->rlStaticP.as<double>();
        r.idRank = ctx->rlIdRank.as<int>();
        r.limitType = ctx->rlLimitType.as<int8_t>();
        r.switchCount = ctx->rlSwitchCount.as<int8_t>();
        r.passSwitched = ctx->rlPassSwitched.as<int8_t>();
        r.savedMode = ctx->rlSavedMode.as<int8_t>();
        r.savedTarget = ctx->rlSavedTarget.as<double>();
        r.remainingPv = ctx->rlRemainingPv.as<int>();
        r.switched = ctx->rlSwitched.as<int>();
    }
    OLF_CUDA(cudaDeviceSynchronize());   // the reactive-limit uploads (pageable) have landed
    return ctx.release();
}

namespace {

// base vector [n] -> every lane; padding lanes get the same values (they never iterate)
__global__ void tileKernel(const double* base, double* out, int n, int S) {
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (size_t)n * S) return;
    out[tid] = base[tid / S];
}

__global__ void tileModeKernel(const int* base, int8_t* out, int n, int S) {
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (size_t)n * S) return;
    out[tid] = (int8_t)base[tid / S];
}

// scenario-major [nS][n] -> lane-interleaved [n][S] through 32x32 shared tiles
// Start selection of the fallback mode: the per-lane max |F| of the fill just run moves to out[s] (NaN stays NaN)
// and the accumulator is cleared for the Newton loop.
__global__ void takeNormKernel(DevBatch b, double* out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.S) return;
    out[s] = __longlong_as_double((long long)b.norm[s]);
    b.norm[s] = 0ull;
}

// Keeps, per lane, the start with the smaller initial max |F|: x holds the base start, `saved` the lane's own start.
// A lane that keeps the base start is marked (fellBack = 2) and not restarted again on failure.
__global__ void chooseStartKernel(DevBatch b, const double* saved, const double* normOwn, const double* normBase, int n) {
    const size_t S = b.S;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (size_t)n * S) return;
    const int s = (int)(tid % S);
    if (s >= b.nS) return;
    const bool own = normOwn[s] <= normBase[s];      // false when the own start's mismatch is NaN
    if (own) {
        b.x[tid] = saved[tid];
    } else if (tid < S) {
        b.fellBack[s] = 2;
        b.fallbackLeft[s] = 0;
    }
}

__global__ void toLanesKernel(const double* in, double* out, int n, int nS, int S) {
    __shared__ double tile[32][33];
    const int r0 = blockIdx.x * 32, s0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int s = s0 + k, r = r0 + threadIdx.x;
        if (s < nS && r < n) tile[k][threadIdx.x] = in[(size_t)s * n + r];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, s = s0 + threadIdx.x;
        if (r < n && s < nS) out[(size_t)r * S + s] = tile[threadIdx.x][k];
    }
}

// lane-interleaved state -> scenario-major results [nS][n + 3]
__global__ void resultsKernel(const double* x, const int* iter, const double* normOut, const int* status, double* out,
                              int n, int nS, int S) {
    __shared__ double tile[32][33];
    const int r0 = blockIdx.x * 32, s0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, s = s0 + threadIdx.x;
        if (r < n && s < S) tile[k][threadIdx.x] = x[(size_t)r * S + s];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int s = s0 + k, r = r0 + threadIdx.x;
        if (s < nS && r < n) out[(size_t)s * (n + 3) + r] = tile[threadIdx.x][k];
    }
    if (blockIdx.x == 0 && threadIdx.y == 0) {
        const int s = s0 + threadIdx.x;
        if (s < nS) {
            out[(size_t)s * (n + 3) + n] = (double)iter[s];
            out[(size_t)s * (n + 3) + n + 1] = normOut[s];
            out[(size_t)s * (n + 3) + n + 2] = (double)status[s];
        }
    }
}

__global__ void targetOverrideKernel(const int* idx, const double* val, int count, double* target, int n, int S) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int s = idx[k] / n, r = idx[k] % n;
    target[(size_t)r * S + s] = val[k];
}

__global__ void rowModeOverrideKernel(const int* triples, int count, int8_t* mode, int S) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    mode[(size_t)triples[3 * k + 1] * S + triples[3 * k]] = (int8_t)triples[3 * k + 2];
}

__global__ void laneInitKernel(DevBatch b) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.S) return;
    const bool live = s < b.nS;
    b.iter[s] = 0;
    b.status[s] = live ? ST_RUNNING : ST_REJECTED;
    b.active[s] = live ? 1 : 0;
    b.pending[s] = 0;
    b.outer[s] = 0;
    b.totalIter[s] = 0;
    b.trouble[s] = 0;
    b.norm[s] = 0ull;
    b.normOut[s] = 0.0;
    b.precision64[s] = 0;
    b.fallbackLeft[s] = live && b.fallbackOn ? 1 : 0;
    b.fellBack[s] = 0;
    if (s == 0) *b.nActive = b.nS;
}

// lanes still iterating after the batched-iteration cap (newton_iteration.cu:410-429) are REJECTED
__global__ void capKernel(DevBatch b) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.S || !b.active[s]) return;
    b.status[s] = ST_REJECTED;
    b.active[s] = 0;
}

void outageBits(BatchContext& ctx, const unsigned char* disabled, int nS, int nElements) {
    const int words = ctx.S / 32;
    const int nE = ctx.net->host.nElements;
    const size_t count = static_cast<size_t>(std::max(nE, 1)) * words;
    if (!ctx.hostBitsPinned) OLF_CUDA(cudaMallocHost(&ctx.hostBitsPinned, count * 4));
    OLF_CUDA(cudaStreamSynchronize(ctx.stream));   // the previous upload from the staging has completed
    uint32_t* bits = ctx.hostBitsPinned;
    std::memset(bits, 0, count * 4);
    if (disabled) {
        const int cols = std::min(nElements, nE);
        for (int s = 0; s < nS; s++) {
            const unsigned char* row = disabled + static_cast<size_t>(s) * nElements;
            int e = 0;
            // skip zero runs eight bytes at a time
            for (; e + 8 <= cols; e += 8) {
                uint64_t w;
                std::memcpy(&w, row + e, 8);
                if (!w) continue;
                for (int k = 0; k < 8; k++)
                    if (row[e + k]) bits[static_cast<size_t>(e + k) * words + (s >> 5)] |= 1u << (s & 31);
            }
            for (; e < cols; e++)
                if (row[e]) bits[static_cast<size_t>(e) * words + (s >> 5)] |= 1u << (s & 31);
        }
    }
    OLF_CUDA(cudaMemcpyAsync(ctx.disabled.p, bits, count * 4, cudaMemcpyHostToDevice, ctx.stream));
}

namespace {

cudaGraphExec_t captureInto(cudaStream_t st, const std::function<void()>& body) {
    cudaGraph_t g;
    cudaGraphExec_t x = nullptr;
    OLF_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    body();
    OLF_CUDA(cudaStreamEndCapture(st, &g));
    OLF_CUDA(cudaGraphInstantiate(&x, g, 0));
    cudaGraphDestroy(g);
    return x;
}

void dropGraph(cudaGraphExec_t& g) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
}

// The lanes flagged for an FP64 refactor (mixed precision), as a batch view whose LU kernels see only them.
DevBatch fp64View(BatchContext& ctx) {
    const size_t S = ctx.S;
    if (!ctx.lu64.p) ctx.lu64.alloc(static_cast<size_t>(ctx.net->dev->view.nLu) * 4 * S * 8);
    DevBatch b = ctx.batch();
    b.lu64 = ctx.lu64.as<double>();
    b.laneMask = ctx.precision64.as<int8_t>();
    return b;
}

}  // namespace

void captureIteration(BatchContext& ctx) {
    const int key = ctx.narrowLanes * 100000 + (ctx.regionFactor ? 50000 : 0) + (ctx.regionSolve ? 20000 : 0) +
                    ctx.precision * 1000 +
                    ctx.refinementSteps * 10 +
                    (ctx.rl.nRl > 0 && ctx.cfg.reactiveLimits ? 1 : 0);
    if (ctx.graph && ctx.graphKey == key) return;
    dropGraph(ctx.graph);
    dropGraph(ctx.graphSolve);
    dropGraph(ctx.graphFactor);
    dropGraph(ctx.graphResidual);
    dropGraph(ctx.graphCorrect);
    dropGraph(ctx.graph64);
    dropGraph(ctx.graphStep);
    const DeviceNet& dn = *ctx.net->dev;
    const DevNet& net = dn.view;
    const size_t S = ctx.S;
    const bool mixed = ctx.precision == 1;
    if (mixed && !ctx.lu32.p) ctx.lu32.alloc(static_cast<size_t>(net.nLu) * 4 * S * 4);
    if (!mixed && !ctx.lu64.p) ctx.lu64.alloc(static_cast<size_t>(net.nLu) * 4 * S * 8);
    const DevBatch b = ctx.batch();
    const bool rl = ctx.rl.nRl > 0 && ctx.cfg.reactiveLimits;
    cudaStream_t st = ctx.stream;
    const Hybrid hy = ctx.hybrid();
    const Hybrid* hp = ctx.useHybrid() ? &hy : nullptr;
    const int nLevels = static_cast<int>(dn.levelPtr.size()) - 1;
    // part 1: fill, test, reactive limits, lane counts
    ctx.graph = captureInto(st, [&] {
        launchIterationStart(b, st);
        launchFill(net, b, true, rl, st);
        launchTest(net, b, ctx.cfg, rl ? ctx.rl.remainingPv : nullptr, st);
        if (rl) launchReactiveLimits(net, b, ctx.rl, ctx.cfg, st);
        launchCountSolving(b, mixed ? ctx.cfg.refineBelow : -1.0, st);
    });
    if (!mixed) {
        // part 2 (FP64): factorization, solves, step
        ctx.graphSolve = captureInto(st, [&] {
            launchFactor(net, b, dn.levelPtr.data(), dn.levelSplit.data(), nLevels, false, hp, st);
            launchSolve(net, b, dn.fwd(), dn.bwd(), false, false, hp, st);
            launchStep(net, b, false, st);
        });
    } else {
        ctx.graphFactor = captureInto(st, [&] {
            launchFactor(net, b, dn.levelPtr.data(), dn.levelSplit.data(), nLevels, true, hp, st);
            launchCountFp64(b, st);
        });
        ctx.graphSolve = captureInto(st, [&] { launchSolve(net, b, dn.fwd(), dn.bwd(), true, false, hp, st); });
        if (ctx.refinementSteps > 0) {
            // one refinement step: the FP64 residual and its check, then (when a lane needs it) the correction solve
            ctx.graphResidual = captureInto(st, [&] {
                launchResidual(net, b, st);
                launchResidualCheck(net, b, REFINE_RESIDUAL * ctx.cfg.tol, ctx.cfg.refineBelow, st);
            });
            ctx.graphCorrect = captureInto(st, [&] { launchSolve(net, b, dn.fwd(), dn.bwd(), true, true, hp, st); });
        }
        ctx.graphStep = captureInto(st, [&] { launchStep(net, b, false, st); });
    }
    ctx.graphKey = key;
}

// Mixed precision: the FP64 refactor and solve of the flagged lanes (captured on first use: it allocates the FP64
// factors).
void launchFp64Redo(BatchContext& ctx) {
    if (!ctx.graph64) {
        const DeviceNet& dn = *ctx.net->dev;
        const DevBatch b64 = fp64View(ctx);
        const Hybrid hy = ctx.hybrid();
        const Hybrid* hp = ctx.useHybrid() ? &hy : nullptr;
        cudaStream_t st = ctx.stream;
        ctx.graph64 = captureInto(st, [&] {
            launchFactor(dn.view, b64, dn.levelPtr.data(), dn.levelSplit.data(),
                         static_cast<int>(dn.levelPtr.size()) - 1, false, hp, st);
            launchSolve(dn.view, b64, dn.fwd(), dn.bwd(), false, false, hp, st);
        });
    }
    OLF_CUDA(cudaGraphLaunch(ctx.graph64, ctx.stream));
}

// One Newton iteration launched phase by phase with CUDA events between the phases (the same kernels in the same
// order as the two captured graphs); the phase times and the lanes that factorized accumulate in the context.
// Returns false when no lane is left iterating.
// The factorization / one solve of an iteration under the context's schedule (level launches or cooperative sweeps).
void factorPhase(BatchContext& ctx, const DevBatch& b, bool fp32) {
    const DeviceNet& dn = *ctx.net->dev;
    if (ctx.schedule == SCHEDULE_COOP) {
        OLF_CUDA(launchFactorCoop(dn.view, b, dn.coop, fp32, ctx.stream));
        launchDenseFront(dn.view, b, fp32, ctx.stream);
        return;
    }
    const Hybrid hy = ctx.hybrid();
    launchFactor(dn.view, b, dn.levelPtr.data(), dn.levelSplit.data(), static_cast<int>(dn.levelPtr.size()) - 1, fp32,
                 ctx.useHybrid() ? &hy : nullptr, ctx.stream);
}

void solvePhase(BatchContext& ctx, const DevBatch& b, bool fp32, bool fromResidual) {
    const DeviceNet& dn = *ctx.net->dev;
    if (ctx.schedule == SCHEDULE_COOP) {
        OLF_CUDA(launchSolveCoop(dn.view, b, dn.coop, fp32, fromResidual, ctx.stream));
        return;
    }
    const Hybrid hy = ctx.hybrid();
    launchSolve(dn.view, b, dn.fwd(), dn.bwd(), fp32, fromResidual, ctx.useHybrid() ? &hy : nullptr, ctx.stream);
}

// The refinement steps of a mixed-precision iteration, launched directly: FP64 residual, its per-lane check, and the
// correction solve only while some lane's residual is above the bound.
void refinementSteps(BatchContext& ctx, const DevBatch& b) {
    const DeviceNet& dn = *ctx.net->dev;
    cudaStream_t st = ctx.stream;
    for (int r = 0; r < ctx.refinementSteps; r++) {
        launchResidual(dn.view, b, st);
        launchResidualCheck(dn.view, b, REFINE_RESIDUAL * ctx.cfg.tol, ctx.cfg.refineBelow, st);
        OLF_CUDA(cudaMemcpyAsync(ctx.hostActive + 2, static_cast<int*>(ctx.nActive.p) + 2, 4, cudaMemcpyDeviceToHost,
                                 st));
        OLF_CUDA(cudaStreamSynchronize(st));
        if (ctx.hostActive[2] <= 0) break;
        solvePhase(ctx, b, true, true);
    }
}

// One Newton iteration's factorization, solves, refinement, FP64 refactor and step with cooperative sweeps (the
// cooperative launches are not captured in graphs).
void coopIteration(BatchContext& ctx) {
    const DeviceNet& dn = *ctx.net->dev;
    const bool mixed = ctx.precision == 1;
    cudaStream_t st = ctx.stream;
    const DevBatch b = ctx.batch();
    factorPhase(ctx, b, mixed);
    if (mixed) {
        launchCountFp64(b, st);
        OLF_CUDA(cudaMemcpyAsync(ctx.hostActive + 3, static_cast<int*>(ctx.nActive.p) + 3, 4, cudaMemcpyDeviceToHost,
                                 st));
        OLF_CUDA(cudaEventRecord(ctx.countReady, st));
    }
    solvePhase(ctx, b, mixed, false);
    if (mixed) {
        if (ctx.hostActive[2] > 0) refinementSteps(ctx, b);
        OLF_CUDA(cudaEventSynchronize(ctx.countReady));
        if (ctx.hostActive[3] > 0) {
            const DevBatch b64 = fp64View(ctx);
            factorPhase(ctx, b64, false);
            solvePhase(ctx, b64, false, false);
        }
    }
    launchStep(dn.view, b, false, st);
}

bool phaseTimedIteration(BatchContext& ctx) {
    const DeviceNet& dn = *ctx.net->dev;
    const DevNet& net = dn.view;
    const bool mixed = ctx.precision == 1;
    const bool rl = ctx.rl.nRl > 0 && ctx.cfg.reactiveLimits;
    const DevBatch b = ctx.batch();
    cudaStream_t st = ctx.stream;
    cudaEvent_t ev[7];
    for (auto& e : ev) OLF_CUDA(cudaEventCreate(&e));
    OLF_CUDA(cudaEventRecord(ev[0], st));
    launchIterationStart(b, st);
    launchFill(net, b, true, rl, st);
    OLF_CUDA(cudaEventRecord(ev[1], st));
    launchTest(net, b, ctx.cfg, rl ? ctx.rl.remainingPv : nullptr, st);
    if (rl) launchReactiveLimits(net, b, ctx.rl, ctx.cfg, st);
    launchCountSolving(b, mixed ? ctx.cfg.refineBelow : -1.0, st);
    OLF_CUDA(cudaEventRecord(ev[2], st));
    OLF_CUDA(cudaMemcpyAsync(ctx.hostActive, ctx.nActive.p, 12, cudaMemcpyDeviceToHost, st));
    OLF_CUDA(cudaStreamSynchronize(st));
    float ms[6] = {0, 0, 0, 0, 0, 0};
    OLF_CUDA(cudaEventElapsedTime(&ms[0], ev[0], ev[1]));
    OLF_CUDA(cudaEventElapsedTime(&ms[1], ev[1], ev[2]));
    const bool live = ctx.hostActive[0] > 0;
    const int solving = ctx.hostActive[1];
    if (live && solving > 0) {
        OLF_CUDA(cudaEventRecord(ev[2], st));
        factorPhase(ctx, b, mixed);
        if (mixed) launchCountFp64(b, st);
        OLF_CUDA(cudaEventRecord(ev[3], st));
        solvePhase(ctx, b, mixed, false);
        OLF_CUDA(cudaEventRecord(ev[4], st));
        if (mixed) {
            // refinement steps (in iterations with a lane below the threshold) and the FP64 refactor of flagged lanes
            if (ctx.hostActive[2] > 0) refinementSteps(ctx, b);
            OLF_CUDA(cudaMemcpyAsync(ctx.hostActive + 3, static_cast<int*>(ctx.nActive.p) + 3, 4,
                                     cudaMemcpyDeviceToHost, st));
            OLF_CUDA(cudaStreamSynchronize(st));
            if (ctx.hostActive[3] > 0) {
                const DevBatch b64 = fp64View(ctx);
                factorPhase(ctx, b64, false);
                solvePhase(ctx, b64, false, false);
            }
        }
        OLF_CUDA(cudaEventRecord(ev[5], st));
        launchStep(net, b, false, st);
        OLF_CUDA(cudaEventRecord(ev[6], st));
        OLF_CUDA(cudaEventSynchronize(ev[6]));
        for (int i = 2; i < 6; i++) OLF_CUDA(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]));
        ctx.phaseLanes += solving;
    }
    for (int i = 0; i < 6; i++) ctx.phaseMs[i] += ms[i];
    if (live) ctx.phaseIterations++;
    for (auto& e : ev) cudaEventDestroy(e);
    return live;
}

}  // namespace

namespace {

// Host inputs of a solve copied to the device (staging and persistent override buffers); no kernel runs here.
void uploadInputs(BatchContext& ctx, const SolveRequest& req) {
    const int n = ctx.net->host.n;
    cudaStream_t st = ctx.stream;
    double* stageX = ctx.stage.as<double>();
    double* stageT = stageX + n;
    int* stageM = reinterpret_cast<int*>(stageT + n);
    ctx.hasX0Base = req.x0Base != nullptr;
    ctx.hasX0Full = req.x0Full != nullptr || ctx.deviceStart != nullptr;
    ctx.fullSrc = ctx.deviceStart ? ctx.deviceStart : ctx.full.as<double>();
    if (req.x0Full && !ctx.deviceStart) {
        if (ctx.full.bytes < static_cast<size_t>(ctx.nS) * n * 8) ctx.full.alloc(static_cast<size_t>(ctx.nS) * n * 8);
        ctx.fullSrc = ctx.full.as<double>();
        OLF_CUDA(cudaMemcpyAsync(ctx.full.p, req.x0Full, static_cast<size_t>(ctx.nS) * n * 8, cudaMemcpyHostToDevice, st));
    }
    if (req.x0Base) OLF_CUDA(cudaMemcpyAsync(stageX, req.x0Base, n * 8, cudaMemcpyHostToDevice, st));
    OLF_CUDA(cudaMemcpyAsync(stageT, req.targetBase, n * 8, cudaMemcpyHostToDevice, st));
    OLF_CUDA(cudaMemcpyAsync(stageM, req.baseRowMode, n * 4, cudaMemcpyHostToDevice, st));
    ctx.nTargetOverrides = req.nTargetOverrides;
    if (req.nTargetOverrides > 0) {
        if (ctx.ovIdx.bytes < static_cast<size_t>(req.nTargetOverrides) * 4) {
            ctx.ovIdx.alloc(req.nTargetOverrides * 4);
            ctx.ovVal.alloc(req.nTargetOverrides * 8);
        }
        OLF_CUDA(cudaMemcpyAsync(ctx.ovIdx.p, req.targetOverrideIndex, req.nTargetOverrides * 4, cudaMemcpyHostToDevice, st));
        OLF_CUDA(cudaMemcpyAsync(ctx.ovVal.p, req.targetOverrideValue, req.nTargetOverrides * 8, cudaMemcpyHostToDevice, st));
    }
    ctx.nRowModeEntries = req.nRowModeEntries;
    if (req.nRowModeEntries > 0) {
        if (ctx.rowModeE.bytes < static_cast<size_t>(req.nRowModeEntries) * 12) ctx.rowModeE.alloc(req.nRowModeEntries * 12);
        OLF_CUDA(cudaMemcpyAsync(ctx.rowModeE.p, req.rowModeEntries, req.nRowModeEntries * 12, cudaMemcpyHostToDevice, st));
    }
    outageBits(ctx, req.disabled, ctx.nS, req.nElements);
}

// Device-side install of the uploaded inputs: every lane gets the base vectors, then the per-scenario overrides; lane
// state and reactive-limit state reset.  Repeatable (the autotuner reinstalls the same batch for every candidate).
void installLanes(BatchContext& ctx) {
    const int n = ctx.net->host.n;
    const size_t S = ctx.S;
    cudaStream_t st = ctx.stream;
    double* stageX = ctx.stage.as<double>();
    double* stageT = stageX + n;
    int* stageM = reinterpret_cast<int*>(stageT + n);
    const unsigned blocksAll = static_cast<unsigned>((static_cast<size_t>(n) * S + 255) / 256);
    if (ctx.hasX0Base) tileKernel<<<blocksAll, 256, 0, st>>>(stageX, ctx.x.as<double>(), n, ctx.S);
    if (ctx.hasX0Full) {
        dim3 blk(32, 8), grd((n + 31) / 32, (ctx.nS + 31) / 32);
        toLanesKernel<<<grd, blk, 0, st>>>(ctx.fullSrc, ctx.x.as<double>(), n, ctx.nS, ctx.S);
    }
    tileKernel<<<blocksAll, 256, 0, st>>>(stageT, ctx.target.as<double>(), n, ctx.S);
    tileModeKernel<<<blocksAll, 256, 0, st>>>(stageM, ctx.mode.as<int8_t>(), n, ctx.S);
    if (ctx.nTargetOverrides > 0) {
        targetOverrideKernel<<<(ctx.nTargetOverrides + 255) / 256, 256, 0, st>>>(
            ctx.ovIdx.as<int>(), ctx.ovVal.as<double>(), ctx.nTargetOverrides, ctx.target.as<double>(), n, ctx.S);
    }
    if (ctx.nRowModeEntries > 0) {
        rowModeOverrideKernel<<<(ctx.nRowModeEntries + 255) / 256, 256, 0, st>>>(ctx.rowModeE.as<int>(),
                                                                                ctx.nRowModeEntries,
                                                                                ctx.mode.as<int8_t>(), ctx.S);
    }
    laneInitKernel<<<(ctx.S + 127) / 128, 128, 0, st>>>(ctx.batch());
    if (ctx.rl.nRl > 0) {
        OLF_CUDA(cudaMemsetAsync(ctx.rlLimitType.p, 0, ctx.rlLimitType.bytes, st));
        OLF_CUDA(cudaMemsetAsync(ctx.rlSwitchCount.p, 0, ctx.rlSwitchCount.bytes, st));
        OLF_CUDA(cudaMemsetAsync(ctx.rlPassSwitched.p, 0, ctx.rlPassSwitched.bytes, st));
    }
}

int roundCap(const BatchContext& ctx) {
    const int solves = ctx.fallbackStart && ctx.hasX0Base && ctx.hasX0Full ? 2 : 1;   // a fallback restart: 2 solves
    return ctx.cfg.reactiveLimits ? (ctx.cfg.maxOuter + 1) * (ctx.cfg.maxIter + 1) : solves * (ctx.cfg.maxIter + 1);
}

// The Newton iterations under the context's schedule; returns the batched iterations run (level launches) or 0.
// Fallback mode, before the first iteration: each lane starts from whichever of its own start (x0Full) and the base
// start (x0Base) has the smaller max |F| (two mismatch-only fills over all lanes).
void selectStarts(BatchContext& ctx) {
    const DeviceNet& dn = *ctx.net->dev;
    cudaStream_t st = ctx.stream;
    const int n = ctx.net->host.n;
    const size_t all = static_cast<size_t>(n) * ctx.S;
    const DevBatch b = ctx.batch();
    double* saved = ctx.dx.as<double>();             // free until the first solve
    double* normOwn = ctx.res.as<double>();          // [S] scratch at the head of the residual buffer
    double* normBase = normOwn + ctx.S;
    OLF_CUDA(cudaMemsetAsync(ctx.norm.p, 0, ctx.norm.bytes, st));
    launchFill(dn.view, b, false, false, st);
    takeNormKernel<<<(ctx.S + 127) / 128, 128, 0, st>>>(b, normOwn);
    OLF_CUDA(cudaMemcpyAsync(saved, ctx.x.p, all * 8, cudaMemcpyDeviceToDevice, st));
    tileKernel<<<static_cast<unsigned>((all + 255) / 256), 256, 0, st>>>(ctx.stage.as<double>(), ctx.x.as<double>(), n,
                                                                         ctx.S);
    launchFill(dn.view, b, false, false, st);
    takeNormKernel<<<(ctx.S + 127) / 128, 128, 0, st>>>(b, normBase);
    chooseStartKernel<<<static_cast<unsigned>((all + 255) / 256), 256, 0, st>>>(b, saved, normOwn, normBase, n);
}

int runIterations(BatchContext& ctx) {
    cudaStream_t st = ctx.stream;
    const DeviceNet& dn = *ctx.net->dev;
    const bool mixed = ctx.precision == 1;
    const size_t S = ctx.S;
    if (mixed && !ctx.lu32.p) ctx.lu32.alloc(static_cast<size_t>(dn.view.nLu) * 4 * S * 4);
    if (!mixed && !ctx.lu64.p) ctx.lu64.alloc(static_cast<size_t>(dn.view.nLu) * 4 * S * 8);
    const int cap = roundCap(ctx);
    if (ctx.fallbackStart && ctx.hasX0Base && ctx.hasX0Full) selectStarts(ctx);
    if (ctx.schedule == SCHEDULE_PERSISTENT) {
        if (dn.view.frontF > 0) throw std::runtime_error("the persistent schedule does not run dense-front plans");
        PersistentPlan plan = dn.persistent;
        plan.maxRounds = cap;
        launchPersistent(dn.view, ctx.batch(), ctx.rl, ctx.cfg, plan, ctx.lanesPerTile, ctx.threads, mixed, st);
        OLF_CUDA(cudaGetLastError());
        return 0;
    }
    captureIteration(ctx);
    if (ctx.phaseTiming) {
        for (double& v : ctx.phaseMs) v = 0.0;
        ctx.phaseLanes = 0;
        ctx.phaseIterations = 0;
    }
    int k = 0;
    for (; k < cap; k++) {
        if (ctx.phaseTiming) {
            if (!phaseTimedIteration(ctx)) {
                k++;
                break;
            }
            continue;
        }
        OLF_CUDA(cudaGraphLaunch(ctx.graph, st));
        OLF_CUDA(cudaMemcpyAsync(ctx.hostActive, ctx.nActive.p, 12, cudaMemcpyDeviceToHost, st));
        OLF_CUDA(cudaStreamSynchronize(st));
        if (ctx.hostActive[0] <= 0) {
            k++;
            break;
        }
        // no lane factorizes this iteration (only restarts pending): skip the factor / solve graphs
        if (ctx.hostActive[1] <= 0) continue;
        if (ctx.schedule == SCHEDULE_COOP) {
            coopIteration(ctx);
            continue;
        }
        if (!mixed) {
            OLF_CUDA(cudaGraphLaunch(ctx.graphSolve, st));
            continue;
        }
        // mixed: FP32 factorization, then (while the FP32 solves run) the count of lanes flagged for FP64
        OLF_CUDA(cudaGraphLaunch(ctx.graphFactor, st));
        OLF_CUDA(cudaMemcpyAsync(ctx.hostActive + 3, static_cast<int*>(ctx.nActive.p) + 3, 4, cudaMemcpyDeviceToHost,
                                 st));
        OLF_CUDA(cudaEventRecord(ctx.countReady, st));
        OLF_CUDA(cudaGraphLaunch(ctx.graphSolve, st));
        if (ctx.graphResidual && ctx.hostActive[2] > 0) {
            for (int r = 0; r < ctx.refinementSteps; r++) {
                OLF_CUDA(cudaGraphLaunch(ctx.graphResidual, st));
                OLF_CUDA(cudaMemcpyAsync(ctx.hostActive + 2, static_cast<int*>(ctx.nActive.p) + 2, 4,
                                         cudaMemcpyDeviceToHost, st));
                OLF_CUDA(cudaStreamSynchronize(st));
                if (ctx.hostActive[2] <= 0) break;   // every lane's FP32 solve already meets the residual bound
                OLF_CUDA(cudaGraphLaunch(ctx.graphCorrect, st));
            }
        }
        OLF_CUDA(cudaEventSynchronize(ctx.countReady));
        if (ctx.hostActive[3] > 0) launchFp64Redo(ctx);
        OLF_CUDA(cudaGraphLaunch(ctx.graphStep, st));
    }
    capKernel<<<(ctx.S + 127) / 128, 128, 0, st>>>(ctx.batch());
    return k;
}

// Times every candidate schedule on the installed batch and keeps the fastest (the batch is reinstalled before each).
void autotune(BatchContext& ctx) {
    struct Candidate { int schedule, lanes, threads; };
    std::vector<Candidate> cands;
    for (int narrow : {0, 1, 2, 4}) cands.push_back({SCHEDULE_LEVELS, narrow, 256});
    if (ctx.net->dev->regionSlots > 0) {
        for (int narrow : {0, 2}) cands.push_back({SCHEDULE_LEVELS_SHARED, narrow, 256});
    }
    if (ctx.net->dev->fwdRegionSlots > 0 || ctx.net->dev->bwdRegionSlots > 0) {
        cands.push_back({SCHEDULE_LEVELS_SHARED_ALL, 0, 256});
    }
    cands.push_back({SCHEDULE_COOP, 0, 512});
    if (ctx.net->dev->view.frontF == 0) {   // the persistent tiles do not run dense-front plans
        for (int lanes : {2, 4})
            for (int threads : {256, 512}) cands.push_back({SCHEDULE_PERSISTENT, lanes, threads});
    }
    cudaEvent_t e0, e1;
    OLF_CUDA(cudaEventCreate(&e0));
    OLF_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    Candidate pick = cands[0];
    ctx.tuning.clear();
    auto apply = [&](const Candidate& c) {
        ctx.regionFactor = c.schedule == SCHEDULE_LEVELS_SHARED || c.schedule == SCHEDULE_LEVELS_SHARED_ALL;
        ctx.regionSolve = c.schedule == SCHEDULE_LEVELS_SHARED_ALL;
        ctx.schedule = ctx.regionFactor ? SCHEDULE_LEVELS : c.schedule;
        if (ctx.schedule == SCHEDULE_LEVELS) {
            ctx.narrowLanes = c.lanes;
        } else {
            ctx.lanesPerTile = c.lanes;
            ctx.threads = c.threads;
        }
    };
    for (const Candidate& c : cands) {
        apply(c);
        installLanes(ctx);
        OLF_CUDA(cudaEventRecord(e0, ctx.stream));
        runIterations(ctx);
        OLF_CUDA(cudaEventRecord(e1, ctx.stream));
        OLF_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        OLF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        ctx.tuning.push_back({c.schedule, c.lanes, c.threads, ms});
        if (ms < best) {
            best = ms;
            pick = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    apply(pick);
    ctx.autotunePending = false;
}

}  // namespace

void stageRequest(BatchContext& ctx, const SolveRequest& req) {
    OLF_CUDA(cudaSetDevice(ctx.device));
    const Structure& s = ctx.net->host;
    const int n = s.n;
    if (req.nScenarios != ctx.nS) {
        throw std::runtime_error("scenario count " + std::to_string(req.nScenarios) + " does not match the context's " +
                                 std::to_string(ctx.nS));
    }
    if (!req.x0Base && !req.x0Full && !ctx.deviceStart) throw std::runtime_error("no start state");
    if (!req.targetBase || !req.baseRowMode) throw std::runtime_error("no base targets or row modes");
    if (req.maxIter < 1) throw std::runtime_error("maxIter must be >= 1");
    for (int r = 0; r < n; r++) {
        const int m = req.baseRowMode[r];
        if (m != MODE_FIXED_VARIABLE && m != MODE_EQUATION && m != MODE_BUS_TARGET_Q) {
            throw std::runtime_error("unsupported row mode " + std::to_string(m) + " at row " + std::to_string(r));
        }
    }
    for (int k = 0; k < req.nRowModeEntries; k++) {
        const int* t = req.rowModeEntries + 3 * k;
        if (t[0] < 0 || t[0] >= ctx.nS || t[1] < 0 || t[1] >= n) {
            throw std::runtime_error("rowMode entry outside the installed slots or the rows");
        }
        if (t[2] != MODE_FIXED_VARIABLE && t[2] != MODE_EQUATION && t[2] != MODE_BUS_TARGET_Q) {
            throw std::runtime_error("unsupported row mode " + std::to_string(t[2]));
        }
    }
    for (int k = 0; k < req.nTargetOverrides; k++) {
        if (req.targetOverrideIndex[k] < 0 || req.targetOverrideIndex[k] >= ctx.nS * n) {
            throw std::runtime_error("target override index out of range");
        }
    }
    if (ctx.fallbackStart && ctx.rl.nRl > 0) {
        throw std::runtime_error("the fallback start is not available with reactive limits");
    }
    Settings cfg = ctx.cfg;
    cfg.maxIter = req.maxIter;
    cfg.tol = req.tol;
    cfg.rlTol = req.reactiveLimitTol;
    cfg.maxOuter = req.maxOuter;
    cfg.maxSwitch = req.maxPqPvSwitch;
    cfg.reactiveLimits = ctx.rl.nRl > 0 ? 1 : 0;
    cfg.mixed = ctx.precision;
    cfg.refinementSteps = ctx.refinementSteps;
    cfg.refineBelow = ctx.refineBelow;
    cfg.growthLimit = ctx.growthLimit;
    if (std::memcmp(&cfg, &ctx.cfg, sizeof(Settings)) != 0 && ctx.graph) {
        // the level-launch graph bakes the settings in
        cudaGraphExecDestroy(ctx.graph);
        ctx.graph = nullptr;
    }
    ctx.cfg = cfg;
    uploadInputs(ctx, req);
    ctx.staged = true;
}

void solveBatch(BatchContext& ctx, const SolveRequest& req, double* out) {
    stageRequest(ctx, req);
    const int n = ctx.net->host.n;
    cudaStream_t st = ctx.stream;
    if (ctx.autotunePending) autotune(ctx);
    cudaEvent_t e0, e1;
    OLF_CUDA(cudaEventCreate(&e0));
    OLF_CUDA(cudaEventCreate(&e1));
    OLF_CUDA(cudaEventRecord(e0, st));
    installLanes(ctx);
    ctx.lastIterations = runIterations(ctx);
    dim3 blk(32, 8), grd((n + 31) / 32, (ctx.nS + 31) / 32);
    resultsKernel<<<grd, blk, 0, st>>>(ctx.x.as<double>(), ctx.iter.as<int>(), ctx.normOut.as<double>(),
                                       ctx.status.as<int>(), ctx.out.as<double>(), n, ctx.nS, ctx.S);
    OLF_CUDA(cudaEventRecord(e1, st));
    if (out) {
        OLF_CUDA(cudaMemcpyAsync(out, ctx.out.p, static_cast<size_t>(ctx.nS) * (n + 3) * 8, cudaMemcpyDeviceToHost, st));
    }
    OLF_CUDA(cudaStreamSynchronize(st));
    OLF_CUDA(cudaEventElapsedTime(&ctx.lastMs, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    OLF_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------------------------------------------
// Several grids in one persistent launch
// ---------------------------------------------------------------------------------------------------------------
MultiContext::~MultiContext() {
    if (graph) cudaGraphExecDestroy(graph);
    for (cudaEvent_t e : ready) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
    if (hostItems) cudaFreeHost(hostItems);
}

MultiContext* createMultiContext(const std::vector<BatchContext*>& members) {
    if (members.empty()) throw std::runtime_error("a multi-grid context needs at least one batch context");
    const int device = members[0]->device;
    for (const BatchContext* c : members) {
        if (!c) throw std::runtime_error("null batch context");
        if (c->device != device) throw std::runtime_error("the batch contexts of a multi-grid launch share one device");
        if (c->net->dev->view.frontF > 0) {
            throw std::runtime_error("a multi-grid launch runs persistent tiles, which do not run dense-front plans");
        }
    }
    for (size_t i = 0; i < members.size(); i++)
        for (size_t j = i + 1; j < members.size(); j++)
            if (members[i] == members[j]) throw std::runtime_error("a batch context appears twice");
    OLF_CUDA(cudaSetDevice(device));
    auto m = std::make_unique<MultiContext>();
    m->members = members;
    m->device = device;
    OLF_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    m->ready.resize(members.size());
    for (auto& e : m->ready) OLF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    m->itemsDev.alloc(members.size() * sizeof(MultiItem));
    OLF_CUDA(cudaMallocHost(&m->hostItems, members.size() * sizeof(MultiItem)));
    return m.release();
}

namespace {

int tilesOf(const BatchContext& c, int lanes) { return (c.nS + lanes - 1) / lanes; }

// Member order of the launch: as given, or the grids with the most buses first (their tiles run longest, so they
// are dispatched first and the small grids' tiles fill the tail).
std::vector<int> launchOrder(const MultiContext& m, int order) {
    std::vector<int> idx(m.members.size());
    for (size_t i = 0; i < idx.size(); i++) idx[i] = static_cast<int>(i);
    if (order == 1) {
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
            return m.members[a]->net->host.n > m.members[b]->net->host.n;
        });
    }
    return idx;
}

// Lanes of every member reset to their staged inputs, then the one launch (and the members' result gathers).
void runMulti(MultiContext& m, bool fp32) {
    cudaStream_t st = m.stream;
    for (size_t i = 0; i < m.members.size(); i++) {
        BatchContext& c = *m.members[i];
        installLanes(c);
        OLF_CUDA(cudaEventRecord(m.ready[i], c.stream));
        OLF_CUDA(cudaStreamWaitEvent(st, m.ready[i], 0));
    }
    const std::vector<int> idx = launchOrder(m, m.order);
    int tile = 0;
    for (size_t k = 0; k < idx.size(); k++) {
        BatchContext& c = *m.members[idx[k]];
        MultiItem& it = m.hostItems[k];
        it.net = c.net->dev->view;
        it.b = c.batch();
        it.rl = c.rl;
        it.cfg = c.cfg;
        it.plan = c.net->dev->persistent;
        it.plan.maxRounds = roundCap(c);
        it.tileBegin = tile;
        tile += tilesOf(c, m.lanesPerTile);
    }
    OLF_CUDA(cudaMemcpyAsync(m.itemsDev.p, m.hostItems, m.members.size() * sizeof(MultiItem), cudaMemcpyHostToDevice,
                             st));
    const int key = (m.lanesPerTile * 1024 + m.threads) * 2 + (fp32 ? 1 : 0);
    if (!m.graph || m.graphKey != key) {
        if (m.graph) cudaGraphExecDestroy(m.graph);
        m.graph = nullptr;
        cudaGraph_t g;
        OLF_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        launchMulti(m.itemsDev.as<MultiItem>(), static_cast<int>(m.members.size()), tile, m.lanesPerTile, m.threads,
                    fp32, st);
        for (BatchContext* c : m.members) {
            const int n = c->net->host.n;
            dim3 blk(32, 8), grd((n + 31) / 32, (c->nS + 31) / 32);
            resultsKernel<<<grd, blk, 0, st>>>(c->x.as<double>(), c->iter.as<int>(), c->normOut.as<double>(),
                                               c->status.as<int>(), c->out.as<double>(), n, c->nS, c->S);
        }
        OLF_CUDA(cudaStreamEndCapture(st, &g));
        OLF_CUDA(cudaGraphInstantiate(&m.graph, g, 0));
        cudaGraphDestroy(g);
        m.graphKey = key;
    }
    OLF_CUDA(cudaGraphLaunch(m.graph, st));
}

void autotuneMulti(MultiContext& m, bool fp32) {
    cudaEvent_t e0, e1;
    OLF_CUDA(cudaEventCreate(&e0));
    OLF_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    MultiTuning pick{};
    m.tuning.clear();
    for (int lanes : {1, 2, 4, 8})
        for (int threads : {256, 512})
            for (int order : {0, 1}) {
                m.lanesPerTile = lanes;
                m.threads = threads;
                m.order = order;
                OLF_CUDA(cudaEventRecord(e0, m.stream));
                runMulti(m, fp32);
                OLF_CUDA(cudaEventRecord(e1, m.stream));
                OLF_CUDA(cudaEventSynchronize(e1));
                float ms = 0.f;
                OLF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                m.tuning.push_back({lanes, threads, order, ms});
                if (ms < best) {
                    best = ms;
                    pick = m.tuning.back();
                }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    m.lanesPerTile = pick.lanesPerTile;
    m.threads = pick.threads;
    m.order = pick.order;
    m.autotunePending = false;
}

}  // namespace

void solveMulti(MultiContext& m, double* const* outs) {
    OLF_CUDA(cudaSetDevice(m.device));
    const int precision = m.members[0]->precision;
    for (BatchContext* c : m.members) {
        if (!c->staged) throw std::runtime_error("every batch context of a multi-grid launch must be staged first");
        if (c->precision != precision) {
            throw std::runtime_error("the batch contexts of a multi-grid launch share one precision");
        }
    }
    const bool fp32 = precision == 1;
    for (BatchContext* c : m.members) {
        const size_t lu = static_cast<size_t>(c->net->dev->view.nLu) * 4 * c->S;
        if (fp32 && !c->lu32.p) c->lu32.alloc(lu * 4);
        if (!fp32 && !c->lu64.p) c->lu64.alloc(lu * 8);
    }
    if (m.autotunePending) autotuneMulti(m, fp32);
    cudaStream_t st = m.stream;
    cudaEvent_t e0, e1;
    OLF_CUDA(cudaEventCreate(&e0));
    OLF_CUDA(cudaEventCreate(&e1));
    // the members' installs run on their own streams after e0: time from before them
    OLF_CUDA(cudaEventRecord(e0, st));
    for (BatchContext* c : m.members) OLF_CUDA(cudaStreamWaitEvent(c->stream, e0, 0));
    runMulti(m, fp32);
    OLF_CUDA(cudaEventRecord(e1, st));
    for (size_t i = 0; i < m.members.size(); i++) {
        BatchContext& c = *m.members[i];
        if (outs && outs[i]) {
            OLF_CUDA(cudaMemcpyAsync(outs[i], c.out.p, static_cast<size_t>(c.nS) * (c.net->host.n + 3) * 8,
                                     cudaMemcpyDeviceToHost, st));
        }
    }
    OLF_CUDA(cudaStreamSynchronize(st));
    OLF_CUDA(cudaEventElapsedTime(&m.lastMs, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (BatchContext* c : m.members) {
        c->lastIterations = 0;
        c->lastMs = m.lastMs;
    }
    OLF_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------------------------------------------
// Test surface
// ---------------------------------------------------------------------------------------------------------------
void debugFill(BatchContext& ctx, const double* xFull, const double* targetBase, const int* baseRowMode,
               const unsigned char* disabled, double* jOut, double* fOut) {
    OLF_CUDA(cudaSetDevice(ctx.device));
    const Structure& s = ctx.net->host;
    const DeviceNet& dn = *ctx.net->dev;
    const int n = s.n;
    const size_t S = ctx.S;
    cudaStream_t st = ctx.stream;
    DeviceBuffer full;
    full.alloc(static_cast<size_t>(ctx.nS) * n * 8);
    // stream-ordered: a pageable cudaMemcpy may return before its DMA lands, and ctx.stream does not wait for it
    OLF_CUDA(cudaMemcpyAsync(full.p, xFull, static_cast<size_t>(ctx.nS) * n * 8, cudaMemcpyHostToDevice, st));
    dim3 blk(32, 8), grd((n + 31) / 32, (ctx.nS + 31) / 32);
    toLanesKernel<<<grd, blk, 0, st>>>(full.as<double>(), ctx.x.as<double>(), n, ctx.nS, ctx.S);
    double* stageT = ctx.stage.as<double>() + n;
    int* stageM = reinterpret_cast<int*>(stageT + n);
    OLF_CUDA(cudaMemcpyAsync(stageT, targetBase, n * 8, cudaMemcpyHostToDevice, st));
    OLF_CUDA(cudaMemcpyAsync(stageM, baseRowMode, n * 4, cudaMemcpyHostToDevice, st));
    const unsigned blocksAll = static_cast<unsigned>((static_cast<size_t>(n) * S + 255) / 256);
    tileKernel<<<blocksAll, 256, 0, st>>>(stageT, ctx.target.as<double>(), n, ctx.S);
    tileModeKernel<<<blocksAll, 256, 0, st>>>(stageM, ctx.mode.as<int8_t>(), n, ctx.S);
    outageBits(ctx, disabled, ctx.nS, s.nElements);
    const DevBatch b = ctx.batch();
    laneInitKernel<<<(ctx.S + 127) / 128, 128, 0, st>>>(b);
    launchFill(dn.view, b, true, false, st);
    OLF_CUDA(cudaStreamSynchronize(st));
    OLF_CUDA(cudaGetLastError());
    std::vector<double> J(ctx.J.bytes / 8), F(static_cast<size_t>(n) * S);
    OLF_CUDA(cudaMemcpy(J.data(), ctx.J.p, ctx.J.bytes, cudaMemcpyDeviceToHost));
    OLF_CUDA(cudaMemcpy(F.data(), ctx.F.p, F.size() * 8, cudaMemcpyDeviceToHost));
    for (int sc = 0; sc < ctx.nS; sc++) {
        for (int k = 0; k < s.nnz; k++) {
            const int a = dn.csrToA[k];
            jOut[static_cast<size_t>(sc) * s.nnz + k] = J[static_cast<size_t>(a) * S + sc];
        }
        for (int r = 0; r < n; r++) fOut[static_cast<size_t>(sc) * n + r] = F[static_cast<size_t>(r) * S + sc];
    }
}

void debugLinearSolve(BatchContext& ctx, const double* csrVals, const double* rhs, int precision, double* out) {
    OLF_CUDA(cudaSetDevice(ctx.device));
    const Structure& s = ctx.net->host;
    const DeviceNet& dn = *ctx.net->dev;
    const DevNet& net = dn.view;
    const int n = s.n;
    const size_t S = ctx.S;
    cudaStream_t st = ctx.stream;
    const bool fp32 = precision == 1;
    if (fp32 && !ctx.lu32.p) ctx.lu32.alloc(static_cast<size_t>(net.nLu) * 4 * S * 4);
    if (!fp32 && !ctx.lu64.p) ctx.lu64.alloc(static_cast<size_t>(net.nLu) * 4 * S * 8);
    std::vector<double> J(ctx.J.bytes / 8, 0.0), F(static_cast<size_t>(n) * S, 0.0);
    for (int sc = 0; sc < ctx.nS; sc++) {
        for (int k = 0; k < s.nnz; k++) {
            J[static_cast<size_t>(dn.csrToA[k]) * S + sc] = csrVals[static_cast<size_t>(sc) * s.nnz + k];
        }
        for (int r = 0; r < n; r++) F[static_cast<size_t>(r) * S + sc] = -rhs[static_cast<size_t>(sc) * n + r];
    }
    OLF_CUDA(cudaMemcpyAsync(ctx.J.p, J.data(), ctx.J.bytes, cudaMemcpyHostToDevice, ctx.stream));
    OLF_CUDA(cudaMemcpyAsync(ctx.F.p, F.data(), F.size() * 8, cudaMemcpyHostToDevice, ctx.stream));
    const DevBatch b = ctx.batch();
    laneInitKernel<<<(ctx.S + 127) / 128, 128, 0, st>>>(b);
    launchFactor(net, b, dn.levelPtr.data(), dn.levelSplit.data(), static_cast<int>(dn.levelPtr.size()) - 1, fp32,
                 nullptr, st);
    launchSolve(net, b, dn.fwd(), dn.bwd(), fp32, false, nullptr, st);
    OLF_CUDA(cudaStreamSynchronize(st));
    OLF_CUDA(cudaGetLastError());
    std::vector<double> dx(static_cast<size_t>(n) * S);
    OLF_CUDA(cudaMemcpy(dx.data(), ctx.dx.p, dx.size() * 8, cudaMemcpyDeviceToHost));
    for (int sc = 0; sc < ctx.nS; sc++)
        for (int r = 0; r < n; r++) out[static_cast<size_t>(sc) * n + r] = dx[static_cast<size_t>(r) * S + sc];
}

}  // namespace olfb200
