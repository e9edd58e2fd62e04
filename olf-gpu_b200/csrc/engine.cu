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
// Subtree bins of the wide levels
// ---------------------------------------------------------------------------------------------------------------
// The elimination tree's parent of position k is the first column of its U row after the diagonal; the tasks of
// position k (its U row and L column) update from pivots in k's subtree only, and its forward solve reads only k's
// descendants, so a subtree is independent of every other.  A subtree qualifies when all its tasks sit below the narrow
// factorization levels, all its positions below the narrow forward tail and at or above the backward head (the
// shared-memory regions keep those), and it holds no dense-front position.  From the roots down, a qualifying subtree
// whose work (block updates + tasks) fits the cap becomes a bin member; any other root turns into a top position and
// its children are examined.  Members are packed into bins of at most the cap (largest first).  The cap is the
// qualifying work over SUBTREE_BINS: enough bins that bins x lane groups fill the GPU at a few hundred lanes.
constexpr int SUBTREE_BINS = 96;
constexpr int SUBTREE_PHASES = 6;   // bins of the remaining forest, phase after phase
constexpr int NARROW = 48;   // a level of at most this many tasks (positions) is narrow

// The shared-memory factorization region: the narrow levels below factorTo, from the top of the tree down, while each
// fits one round of the region's CTA (at most REGION_THREADS tasks) and their blocks fit REGION_BYTES (FP64, one lane:
// two CTAs per SM).  (Taking the moderately wide levels under them too, up to REGION_THREADS tasks, as far as the
// slots reach, measured the same step time on the shallow-tree plan with a third fewer launches: not kept.)
constexpr size_t REGION_BYTES = 110 * 1024;

int regionStart(const BlockPlan& p, const NarrowBounds& nbd) {
    if (p.deferredL) return nbd.factorTo;   // (deferred-L updates also read the pivot's inverse: range launches)
    int from = nbd.factorTo;
    while (from > nbd.factorFrom && p.levelPtr[from] - p.levelPtr[from - 1] <= REGION_THREADS &&
           static_cast<size_t>(p.levelPtr[nbd.factorTo] - p.levelPtr[from - 1]) * 32 <= REGION_BYTES) {
        from--;
    }
    return from;
}

NarrowBounds binBounds(const BlockPlan& p) {
    NarrowBounds nbd = narrowBounds(p);
    nbd.factorFrom = std::min(nbd.factorFrom, regionStart(p, nbd));   // the bins stop where the region starts
    return nbd;
}

NarrowBounds narrowBounds(const BlockPlan& p) {
    auto countOf = [](const std::vector<int>& ptr, size_t l) { return ptr[l + 1] - ptr[l]; };
    NarrowBounds nbd{};
    // (a dense-front plan ends with the front's assembly level, wide whatever the tree above it: it stays a level
    // launch after the range)
    nbd.factorTo = static_cast<int>(p.levelPtr.size()) - 1 - (p.frontF > 0 ? 1 : 0);
    nbd.factorFrom = nbd.factorTo;
    while (nbd.factorFrom > 0 && countOf(p.levelPtr, nbd.factorFrom - 1) <= NARROW) nbd.factorFrom--;
    nbd.fwdFrom = static_cast<int>(p.fwdLevelPtr.size()) - 1;
    while (nbd.fwdFrom > 0 && countOf(p.fwdLevelPtr, nbd.fwdFrom - 1) <= NARROW) nbd.fwdFrom--;
    nbd.bwdUntil = 0;
    while (nbd.bwdUntil < static_cast<int>(p.bwdLevelPtr.size()) - 1 && countOf(p.bwdLevelPtr, nbd.bwdUntil) <= NARROW) {
        nbd.bwdUntil++;
    }
    return nbd;
}

namespace {

// Bins of subtrees of the elimination forest, phase after phase: a phase takes, from the roots of the forest of
// positions no earlier phase took, every subtree whose root may start one (eligible: monotone, every descendant of an
// eligible root is eligible) and whose weight fits the phase's cap (the remaining weight over SUBTREE_BINS); a root
// that may not, or does not fit, stays out and its children are examined.  Subtrees are packed into bins of at most
// the cap, largest first.  Returns the positions of each bin and the bins of each phase.
struct Forest {
    std::vector<int> parent;
    std::vector<std::vector<int>> children;
};

void binForest(const Forest& fo, const std::vector<long long>& weight, const std::vector<char>& eligible,
               std::vector<std::vector<int>>& binPos, std::vector<int>& phasePtr, std::vector<int>& binOf) {
    const int nb = static_cast<int>(fo.parent.size());
    binOf.assign(nb, -1);
    binPos.clear();
    phasePtr = {0};
    for (int phase = 0; phase < SUBTREE_PHASES; phase++) {
        std::vector<long long> sub(nb, 0);
        for (int k = 0; k < nb; k++) sub[k] = binOf[k] < 0 ? weight[k] : 0;
        for (int k = 0; k < nb; k++)   // children precede their parent (child < parent)
            if (fo.parent[k] >= 0 && binOf[k] < 0) sub[fo.parent[k]] += sub[k];
        long long total = 0;
        for (int k = 0; k < nb; k++)
            if (binOf[k] < 0 && eligible[k] && (fo.parent[k] < 0 || !eligible[fo.parent[k]])) total += sub[k];
        if (total == 0) break;
        const long long cap = std::max<long long>(1, total / SUBTREE_BINS);
        std::vector<int> members, queue;
        for (int k = 0; k < nb; k++)
            if (fo.parent[k] < 0) queue.push_back(k);
        while (!queue.empty()) {
            const int r = queue.back();
            queue.pop_back();
            if (binOf[r] >= 0) continue;
            if (eligible[r] && sub[r] <= cap) {
                if (sub[r] > 0) members.push_back(r);
            } else {
                for (int c : fo.children[r]) queue.push_back(c);
            }
        }
        if (members.empty()) break;
        std::sort(members.begin(), members.end(), [&](int x, int y) { return sub[x] != sub[y] ? sub[x] > sub[y] : x < y; });
        const int first = static_cast<int>(binPos.size());
        std::vector<long long> binWork;
        for (int r : members) {
            size_t k = 0;
            while (k < binWork.size() && binWork[k] + sub[r] > cap) k++;
            if (k == binWork.size()) {
                binWork.push_back(0);
                binPos.emplace_back();
            }
            binWork[k] += sub[r];
            // the remaining subtree of r
            std::vector<int> stack{r};
            while (!stack.empty()) {
                const int q = stack.back();
                stack.pop_back();
                if (binOf[q] >= 0) continue;
                binOf[q] = first + static_cast<int>(k);
                binPos[first + k].push_back(q);
                for (int c : fo.children[q]) stack.push_back(c);
            }
        }
        phasePtr.push_back(static_cast<int>(binPos.size()));
    }
}

}  // namespace

SubtreeBinsHost planSubtreeBins(const BlockPlan& p, const NarrowBounds& nbd) {
    SubtreeBinsHost h;
    const int nb = p.nb;
    if (p.deferredL || nb < 64) return h;
    const int nLu = p.nU + p.nL;
    Forest fo;
    fo.parent.assign(nb, -1);
    fo.children.assign(nb, {});
    std::vector<int> fl(nb, -1), bl(nb, -1);
    h.posOf.assign(nLu, -1);
    for (int k = 0; k < nb; k++) {
        if (p.uPtr[k + 1] - p.uPtr[k] > 1) fo.parent[k] = p.uCol[p.uPtr[k] + 1];
        for (int t = p.uPtr[k]; t < p.uPtr[k + 1]; t++) h.posOf[t] = k;
        for (int t = p.lPtr[k]; t < p.lPtr[k + 1]; t++) h.posOf[p.nU + t] = k;
    }
    for (int k = 0; k < nb; k++)
        if (fo.parent[k] >= 0) fo.children[fo.parent[k]].push_back(k);
    for (size_t l = 0; l + 1 < p.fwdLevelPtr.size(); l++)
        for (int q = p.fwdLevelPtr[l]; q < p.fwdLevelPtr[l + 1]; q++) fl[p.fwdLevelPos[q]] = static_cast<int>(l);
    for (size_t l = 0; l + 1 < p.bwdLevelPtr.size(); l++)
        for (int q = p.bwdLevelPtr[l]; q < p.bwdLevelPtr[l + 1]; q++) bl[p.bwdLevelPos[q]] = static_cast<int>(l);
    auto wide = [&](int id) { return p.level[id] < nbd.factorFrom; };
    // factorization: a position weighs its wide-level tasks (block updates + 1 each); any root may start a bin (a
    // wide task only reads wide blocks of its subtree).  Forward: positions of the wide forward levels (the forward
    // level grows towards the roots); backward: positions of the wide backward levels (it grows towards the leaves),
    // never a dense-front position (the dense front solves those).
    std::vector<long long> wf(nb, 0), ws(nb, 0);
    std::vector<char> anyRoot(nb, 1), fwdOk(nb, 0), bwdOk(nb, 0);
    for (int k = 0; k < nb; k++) {
        auto add = [&](int id) {
            if (wide(id)) wf[k] += p.opPtr[id + 1] - p.opPtr[id] + 1;
        };
        for (int t = p.uPtr[k]; t < p.uPtr[k + 1]; t++) add(t);
        for (int t = p.lPtr[k]; t < p.lPtr[k + 1]; t++) add(p.nU + t);
        ws[k] = (p.uPtr[k + 1] - p.uPtr[k]) + (p.lPtr[k + 1] - p.lPtr[k]);
        fwdOk[k] = fl[k] >= 0 && fl[k] < nbd.fwdFrom;
        bwdOk[k] = k < p.frontStart && bl[k] >= nbd.bwdUntil;
    }
    std::vector<std::vector<int>> fBins, wBins, bBins;
    std::vector<int> fBinOf, wBinOf, bBinOf;
    binForest(fo, wf, anyRoot, fBins, h.phasePtr, fBinOf);
    binForest(fo, ws, fwdOk, wBins, h.fwdPhasePtr, wBinOf);
    binForest(fo, ws, bwdOk, bBins, h.bwdPhasePtr, bBinOf);
    if (fBins.empty() || wBins.empty() || bBins.empty()) return SubtreeBinsHost{};
    auto groupInto = [](std::vector<std::pair<int, int>>& v, std::vector<int>& all, std::vector<int>& off,
                        std::vector<int>& ptr) {
        std::sort(v.begin(), v.end());
        for (size_t q = 0; q < v.size(); q++) {
            if (q > 0 && v[q].first != v[q - 1].first) off.push_back(static_cast<int>(all.size()));
            all.push_back(v[q].second);
        }
        off.push_back(static_cast<int>(all.size()));
        ptr.push_back(static_cast<int>(off.size()) - 1);
    };
    h.levPtr = {0};
    h.levOff = {0};
    h.fwdPtr = {0};
    h.fwdOff = {0};
    h.bwdPtr = {0};
    h.bwdOff = {0};
    h.taskBin.assign(nLu, -1);
    for (size_t b = 0; b < fBins.size(); b++) {
        std::vector<std::pair<int, int>> tk;
        for (int k : fBins[b]) {
            for (int t = p.uPtr[k]; t < p.uPtr[k + 1]; t++)
                if (wide(t)) tk.push_back({p.level[t], t});
            for (int t = p.lPtr[k]; t < p.lPtr[k + 1]; t++)
                if (wide(p.nU + t)) tk.push_back({p.level[p.nU + t], p.nU + t});
        }
        for (auto& e : tk) h.taskBin[e.second] = static_cast<int>(b);
        groupInto(tk, h.task, h.levOff, h.levPtr);
    }
    for (auto& bin : wBins) {
        std::vector<std::pair<int, int>> v;
        for (int k : bin) v.push_back({fl[k], k});
        groupInto(v, h.fwdPos, h.fwdOff, h.fwdPtr);
    }
    for (auto& bin : bBins) {
        std::vector<std::pair<int, int>> v;
        for (int k : bin) v.push_back({bl[k], k});
        groupInto(v, h.bwdPos, h.bwdOff, h.bwdPtr);
    }
    h.nBins = static_cast<int>(fBins.size());
    h.fwdBinOf = wBinOf;
    h.bwdBinOf = bBinOf;
    // the top lists: every level's tasks (positions) outside the bins
    auto topOf = [&](const std::vector<int>& ptr, const std::vector<int>& items, const std::vector<int>& binOfItem,
                     std::vector<int>& outPtr, std::vector<int>& out) {
        outPtr.assign(ptr.size(), 0);
        out.clear();
        for (size_t l = 0; l + 1 < ptr.size(); l++) {
            for (int q = ptr[l]; q < ptr[l + 1]; q++)
                if (binOfItem[items[q]] < 0) out.push_back(items[q]);
            outPtr[l + 1] = static_cast<int>(out.size());
        }
    };
    topOf(p.levelPtr, p.levelTask, h.taskBin, h.topLevelPtr, h.topTask);
    topOf(p.fwdLevelPtr, p.fwdLevelPos, wBinOf, h.topFwdPtr, h.topFwd);
    topOf(p.bwdLevelPtr, p.bwdLevelPos, bBinOf, h.topBwdPtr, h.topBwd);
    return h;
}

// The invariants the bin kernels rely on, checked on the host: every LU block in exactly one of (a bin, a top level),
// every position likewise in each sweep; a bin task's update operands and pivot belong to its bin and sit on an
// earlier level of it; a bin position's forward columns belong to its bin on earlier forward levels; its backward
// columns sit on earlier backward levels of its bin or outside every bin (finished before the bins' backward sweep);
// no bin task on a narrow factorization level, no bin position in the narrow forward tail or backward head.
std::string checkSubtreeBins(const BlockPlan& p, const NarrowBounds& nbd, const SubtreeBinsHost& h) {
    const int nLu = p.nU + p.nL, nb = p.nb;
    if (h.nBins == 0) return "";
    auto phases = [](const std::vector<int>& phasePtr, int nBins) {
        std::vector<int> ph(nBins, 0);
        for (size_t f = 0; f + 1 < phasePtr.size(); f++)
            for (int b = phasePtr[f]; b < phasePtr[f + 1]; b++) ph[b] = static_cast<int>(f);
        return ph;
    };
    const std::vector<int> phaseOf = phases(h.phasePtr, h.nBins);
    std::vector<int> seen(nLu, 0), binLevel(nLu, -1);
    for (int b = 0; b < h.nBins; b++)
        for (int v = h.levPtr[b]; v < h.levPtr[b + 1]; v++)
            for (int q = h.levOff[v]; q < h.levOff[v + 1]; q++) {
                const int t = h.task[q];
                seen[t]++;
                binLevel[t] = v - h.levPtr[b];
                if (p.level[t] >= nbd.factorFrom) return "bin task on a narrow level";
            }
    for (int t : h.topTask) seen[t]++;
    for (int t = 0; t < nLu; t++)
        if (seen[t] != 1) return "LU block " + std::to_string(t) + " scheduled " + std::to_string(seen[t]) + " times";
    for (int t = 0; t < nLu; t++) {
        const int bt = h.taskBin[t];
        if (bt < 0) continue;
        // a block read by a bin task: earlier on the same bin, or in a bin of an earlier phase
        auto before = [&](int src) {
            const int bs = h.taskBin[src];
            return bs >= 0 && (bs == bt ? binLevel[src] < binLevel[t] : phaseOf[bs] < phaseOf[bt]);
        };
        for (int q = p.opPtr[t]; q < p.opPtr[t + 1]; q++)
            for (int src : {p.opL[q], p.opU[q]})
                if (!before(src)) {
                    return "bin task " + std::to_string(t) + " reads block " + std::to_string(src) + " not before it";
                }
        if (t >= p.nU && !before(p.uPtr[h.posOf[t]])) return "L block before its pivot";
    }
    // each sweep: every position once (front positions: not in the backward sweep, the dense front solves them)
    auto place = [&](const std::vector<int>& ptr, const std::vector<int>& off, const std::vector<int>& pos,
                     int nBins, const std::vector<int>& topPos, bool forward, std::vector<int>& lv) -> std::string {
        std::vector<int> cnt(nb, 0);
        lv.assign(nb, -1);
        for (int b = 0; b < nBins; b++)
            for (int v = ptr[b]; v < ptr[b + 1]; v++)
                for (int q = off[v]; q < off[v + 1]; q++) {
                    cnt[pos[q]]++;
                    lv[pos[q]] = v - ptr[b];
                }
        for (int i : topPos) cnt[i]++;
        for (int i = 0; i < nb; i++) {
            const int want = forward || i < p.frontStart ? 1 : 0;
            if (cnt[i] != want) return "position " + std::to_string(i) + " scheduled " + std::to_string(cnt[i]) + " times";
        }
        return "";
    };
    const int nFwdBins = h.fwdPhasePtr.back(), nBwdBins = h.bwdPhasePtr.back();
    const std::vector<int> fph = phases(h.fwdPhasePtr, nFwdBins), bph = phases(h.bwdPhasePtr, nBwdBins);
    std::vector<int> flv, blv;
    std::string e = place(h.fwdPtr, h.fwdOff, h.fwdPos, nFwdBins, h.topFwd, true, flv);
    if (!e.empty()) return "forward: " + e;
    e = place(h.bwdPtr, h.bwdOff, h.bwdPos, nBwdBins, h.topBwd, false, blv);
    if (!e.empty()) return "backward: " + e;
    // forward: row i reads column k for every L(i, k); backward: row i reads column j for every U(i, j), j > i
    for (int k = 0; k < nb; k++)
        for (int t = p.lPtr[k]; t < p.lPtr[k + 1]; t++) {
            const int i = p.lRow[t];
            const int bi = h.fwdBinOf[i], bk = h.fwdBinOf[k];
            if (bi < 0) continue;
            const bool okFwd = bk >= 0 && (bk == bi ? flv[k] < flv[i] : fph[bk] < fph[bi]);
            if (!okFwd) return "forward column not before its row";
        }
    for (int i = 0; i < nb; i++) {
        const int bi = h.bwdBinOf[i];
        if (bi < 0) continue;
        for (int q = p.uPtr[i] + 1; q < p.uPtr[i + 1]; q++) {
            const int j = p.uCol[q], bj = h.bwdBinOf[j];
            // top positions and later phases' bins are solved before this bin's backward sweep
            const bool okBwd = bj < 0 || (bj == bi ? blv[j] < blv[i] : bph[bj] > bph[bi]);
            if (!okBwd) return "backward column not before its row";
        }
    }
    // no bin position in the narrow forward tail or the backward head
    std::vector<int> fl(nb, -1), bl(nb, -1);
    for (size_t l = 0; l + 1 < p.fwdLevelPtr.size(); l++)
        for (int q = p.fwdLevelPtr[l]; q < p.fwdLevelPtr[l + 1]; q++) fl[p.fwdLevelPos[q]] = static_cast<int>(l);
    for (size_t l = 0; l + 1 < p.bwdLevelPtr.size(); l++)
        for (int q = p.bwdLevelPtr[l]; q < p.bwdLevelPtr[l + 1]; q++) bl[p.bwdLevelPos[q]] = static_cast<int>(l);
    for (int i = 0; i < nb; i++) {
        if (h.fwdBinOf[i] >= 0 && fl[i] >= nbd.fwdFrom) return "bin position in the narrow forward tail";
        if (h.bwdBinOf[i] >= 0 && bl[i] < nbd.bwdUntil) return "bin position in the narrow backward head";
    }
    return "";
}

// Uploads the bins and the top lists (with their split factors) of a structure's device copy.
template <typename SplitFn>
void buildSubtreeBins(DeviceNet& d, const BlockPlan& p, const std::vector<int>& lrowLen, SplitFn splitOf) {
    d.sub = SubtreePlan{};
    const NarrowBounds nbd = binBounds(p);
    SubtreeBinsHost h = planSubtreeBins(p, nbd);
    if (h.nBins == 0) return;
    d.topLevelPtr = h.topLevelPtr;
    d.topFwdPtr = h.topFwdPtr;
    d.topBwdPtr = h.topBwdPtr;
    d.topLevelSplit.assign(d.topLevelPtr.size() - 1, 1);
    for (size_t l = 0; l + 1 < d.topLevelPtr.size(); l++) {
        int m = 0;
        for (int q = d.topLevelPtr[l]; q < d.topLevelPtr[l + 1]; q++)
            m = std::max(m, p.opPtr[h.topTask[q] + 1] - p.opPtr[h.topTask[q]]);
        d.topLevelSplit[l] = splitOf(m, 12);
    }
    d.topFwdSplit.assign(d.topFwdPtr.size() - 1, 1);
    for (size_t l = 0; l + 1 < d.topFwdPtr.size(); l++) {
        int m = 0;
        for (int q = d.topFwdPtr[l]; q < d.topFwdPtr[l + 1]; q++) m = std::max(m, lrowLen[h.topFwd[q]]);
        d.topFwdSplit[l] = splitOf(m, 8);
    }
    d.topBwdSplit.assign(d.topBwdPtr.size() - 1, 1);
    for (size_t l = 0; l + 1 < d.topBwdPtr.size(); l++) {
        int m = 0;
        for (int q = d.topBwdPtr[l]; q < d.topBwdPtr[l + 1]; q++) {
            const int i = h.topBwd[q];
            m = std::max(m, p.uPtr[i + 1] - p.uPtr[i] - 1);
        }
        d.topBwdSplit[l] = splitOf(m, 8);
    }
    d.binPhasePtr = h.phasePtr;
    d.binFwdPhasePtr = h.fwdPhasePtr;
    d.binBwdPhasePtr = h.bwdPhasePtr;
    d.binLevPtr.upload(h.levPtr);
    d.binLevOff.upload(h.levOff);
    d.binTask.upload(h.task);
    d.binFwdPtr.upload(h.fwdPtr);
    d.binFwdOff.upload(h.fwdOff);
    d.binFwdPos.upload(h.fwdPos);
    d.binBwdPtr.upload(h.bwdPtr);
    d.binBwdOff.upload(h.bwdOff);
    d.binBwdPos.upload(h.bwdPos);
    d.topLevelTaskD.upload(h.topTask.empty() ? std::vector<int>{0} : h.topTask);
    d.topFwdPosD.upload(h.topFwd.empty() ? std::vector<int>{0} : h.topFwd);
    d.topBwdPosD.upload(h.topBwd.empty() ? std::vector<int>{0} : h.topBwd);
    d.binTasks = static_cast<int>(h.task.size());
    SubtreePlan& sp = d.sub;
    sp.nBins = h.nBins;
    sp.nPhases = static_cast<int>(d.binPhasePtr.size()) - 1;
    sp.phasePtr = d.binPhasePtr.data();
    sp.nFwdPhases = static_cast<int>(d.binFwdPhasePtr.size()) - 1;
    sp.fwdPhasePtr = d.binFwdPhasePtr.data();
    sp.nBwdPhases = static_cast<int>(d.binBwdPhasePtr.size()) - 1;
    sp.bwdPhasePtr = d.binBwdPhasePtr.data();
    sp.levPtr = d.binLevPtr.as<int>();
    sp.levOff = d.binLevOff.as<int>();
    sp.task = d.binTask.as<int>();
    sp.fwdPtr = d.binFwdPtr.as<int>();
    sp.fwdOff = d.binFwdOff.as<int>();
    sp.fwdPos = d.binFwdPos.as<int>();
    sp.bwdPtr = d.binBwdPtr.as<int>();
    sp.bwdOff = d.binBwdOff.as<int>();
    sp.bwdPos = d.binBwdPos.as<int>();
    sp.topLevelTask = d.topLevelTaskD.as<int>();
    sp.topLevelPtr = d.topLevelPtr.data();
    sp.topLevelSplit = d.topLevelSplit.data();
    sp.topFwdPos = d.topFwdPosD.as<int>();
    sp.topFwdPtr = d.topFwdPtr.data();
    sp.topFwdSplit = d.topFwdSplit.data();
    sp.topBwdPos = d.topBwdPosD.as<int>();
    sp.topBwdPtr = d.topBwdPtr.data();
    sp.topBwdSplit = d.topBwdSplit.data();
}

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
    const NarrowBounds nbd = narrowBounds(p);
    d->factorTo = nbd.factorTo;
    d->factorFrom = nbd.factorFrom;
    // the shared-memory region (regionStart): every block its levels produce gets a slot, in level order, and every
    // update its operands' slots in ops.w (slot + 1 of the L block in the low 16 bits, of the U block in the high 16
    // bits, 0 outside)
    d->regionFrom = regionStart(p, nbd);
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
    d->fwdFrom = nbd.fwdFrom;
    d->bwdUntil = nbd.bwdUntil;
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
    // the transposed solve's entries on the same factors: U^T has L's pattern (row i of U^T reads U(k, i) for every
    // L(i, k)) and L^T has U's (row i of L^T reads L(j, i) for every U(i, j), j > i)
    {
        std::vector<int> lrowU(std::max<size_t>(lrow.size(), 1), 0), uRowL(std::max<size_t>(p.nU, 1), 0);
        auto uBlockOf = [&](int k, int j) {
            auto lo = p.uCol.begin() + p.uPtr[k] + 1, hi = p.uCol.begin() + p.uPtr[k + 1];
            auto it = std::lower_bound(lo, hi, j);
            if (it == hi || *it != j) throw std::runtime_error("transposed solve: U block lookup miss");
            return static_cast<int>(it - p.uCol.begin());
        };
        auto lBlockOf = [&](int i, int k) {
            auto lo = p.lRow.begin() + p.lPtr[k], hi = p.lRow.begin() + p.lPtr[k + 1];
            auto it = std::lower_bound(lo, hi, i);
            if (it == hi || *it != i) throw std::runtime_error("transposed solve: L block lookup miss");
            return p.nU + static_cast<int>(it - p.lRow.begin());
        };
        for (int i = 0; i < nb; i++) {
            for (int q = lrowPtr[i]; q < lrowPtr[i + 1]; q++) lrowU[q] = uBlockOf(lrow[q].y, i);
            for (int q = p.uPtr[i] + 1; q < p.uPtr[i + 1]; q++) uRowL[q] = lBlockOf(p.uCol[q], i);
        }
        d->lrowU.upload(lrowU);
        d->uRowL.upload(uRowL);
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
    buildSubtreeBins(*d, p, lrowLen, splitOf);
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
    v.lrowU = d->lrowU.as<int>();
    v.uRowL = d->uRowL.as<int>();
    v.lrow = d->lrow.as<int2>();
    v.uPtr = d->uPtr.as<int>();
    v.uCol = d->uCol.as<int>();
    OLF_CUDA(cudaDeviceSynchronize());
    // the uploads above are pageable cudaMemcpy calls, whose DMA may still be in flight when they return; the
    // contexts' non-blocking streams would not wait for it
    OLF_CUDA(cudaDeviceSynchronize());
    return d;
}

std::shared_ptr<DeviceNet> NetStructure::onDevice(int device) {
    std::lock_guard<std::mutex> lock(mu);
    auto it = devs.find(device);
    if (it != devs.end()) return it->second;
    auto d = uploadNet(host);
    devs[device] = d;
    return d;
}

std::shared_ptr<DeviceNet> NetStructure::find(int device) {
    std::lock_guard<std::mutex> lock(mu);
    auto it = devs.find(device);
    return it == devs.end() ? nullptr : it->second;
}

// ---------------------------------------------------------------------------------------------------------------
// Batch context
// ---------------------------------------------------------------------------------------------------------------
BatchContext::~BatchContext() {
    if (graph) cudaGraphExecDestroy(graph);
    if (graphSolve) cudaGraphExecDestroy(graphSolve);
    for (cudaGraphExec_t gx : {graphFactor, graphResidual, graphCorrect, graph64, graph64All, graphStep,
                               graphSolveScored, graphStepScored})
        if (gx) cudaGraphExecDestroy(gx);
    if (loopGraph) cudaGraphExecDestroy(loopGraph);
    for (cudaStream_t s : loopStreams)
        if (s) cudaStreamDestroy(s);
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
    b.fp64Left = fp64RestartOn ? fp64Left.as<int8_t>() : nullptr;
    // the FP64 restart starts from the base start in fallback mode (the fallback already tried the lane's own start)
    // or when no per-scenario start was given, else from the lane's own start row
    b.restartFull = (b.fallbackOn || !hasX0Full) ? nullptr : fullSrc;
    b.refine = refine.as<int8_t>();
    b.ssqPart = ssqPart.as<double>();
    b.solveRatio = solveRatio.as<double>();
    b.stepMax = stepMax.as<unsigned long long>();
    b.varType = hasVarType ? varType.as<int8_t>() : nullptr;
    b.vCheck = hasVCheck ? vCheck.as<int8_t>() : nullptr;
    b.laneLive = hasLaneLive ? laneLive.as<int8_t>() : nullptr;
    b.dsRestart = dsRestartBuf.as<int8_t>();
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
    ctx->dn = net->onDevice(ctx->device);
    const Structure& s = net->host;
    const DevNet& v = ctx->dn->view;
    ctx->nS = nScenarios;
    ctx->S = (nScenarios + 31) / 32 * 32;
    const size_t S = ctx->S, n = s.n;
    OLF_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    OLF_CUDA(cudaMallocHost(&ctx->hostActive, 8 * sizeof(int)));
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
    ctx->fp64Left.alloc(S);
    ctx->refine.alloc(S);
    ctx->ssqPart.alloc(static_cast<size_t>(SSQ_STRANDS) * S * 8);
    ctx->solveRatio.alloc(S * 8);
    ctx->stepMax.alloc(2 * S * 8);
    ctx->varType.alloc(n);
    ctx->vCheck.alloc(n);
    ctx->laneLive.alloc(S);
    ctx->dsRestartBuf.alloc(S);
    ctx->nActive.alloc(8 * sizeof(int));
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
    ctx->cfg.corrBound = ctx->corrBound;
    ctx->cfg.polishBelow = 0.0;
    ctx->cfg.batchOfOne = nScenarios == 1 ? 1 : 0;
    if (nRl > 0) {
        for (int i = 0; i < nRl; i++) {
            if (voltageRow[i] < 0 || voltageRow[i] >= s.n) throw std::runtime_error("bad reactiveLimitVoltageRow");
            if (pRow && pRow[i] >= s.n) throw std::runtime_error("bad reactiveLimit pRow");
        }
        // the forced-PV election keys may come later (olfgpu_set_reactive_limit_strongest_pv_keys): zeroed until then
        auto up = [&](DeviceBuffer& d, const void* src, size_t bytes) {
            d.alloc(bytes);
            if (src) OLF_CUDA(cudaMemcpy(d.p, src, bytes, cudaMemcpyHostToDevice));
        };
        ctx->rlKeys = nomV && pRow && staticP && idRank;
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

// Lane state at install; nActive[0] (zeroed before) counts the live lanes.
__global__ void laneInitKernel(DevBatch b) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.S) return;
    const bool live = s < b.nS && (!b.laneLive || b.laneLive[s]);
    if (live) atomicAdd(b.nActive, 1);
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
    if (b.fp64Left) b.fp64Left[s] = live ? 1 : 0;
    b.refine[s] = 0;
    b.solveRatio[s] = 0.0;
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
    if (!ctx.lu64.p) ctx.lu64.alloc(static_cast<size_t>(ctx.dn->view.nLu) * 4 * S * 8);
    DevBatch b = ctx.batch();
    b.lu64 = ctx.lu64.as<double>();
    b.laneMask = ctx.precision64.as<int8_t>();
    return b;
}

// Every factorizing lane in FP64 (an FP64 iteration of the MIXED_FP64_NEAR policy).
DevBatch fp64AllView(BatchContext& ctx) {
    DevBatch b = fp64View(ctx);
    b.laneMask = nullptr;
    return b;
}

}  // namespace

void captureIteration(BatchContext& ctx) {
    const int key = ctx.narrowLanes * 100000 + (ctx.regionFactor ? 50000 : 0) + (ctx.regionSolve ? 20000 : 0) +
                    (ctx.subtrees ? 5000000 : 0) +
                    ctx.precision * 1000 +
                    ctx.refinementSteps * 10 +
                    (ctx.rl.nRl > 0 && ctx.cfg.reactiveLimits ? 1 : 0) +
                    (ctx.ds.nDs > 0 && ctx.cfg.distributedSlack ? 2 : 0);
    // the graphs bake the batch view (pointers, per-request flags) and the settings into their kernel parameters
    const DevBatch now = ctx.batch();
    if (ctx.graph && ctx.graphKey == key && std::memcmp(&now, &ctx.graphBatch, sizeof(DevBatch)) == 0 &&
        std::memcmp(&ctx.cfg, &ctx.graphCfg, sizeof(Settings)) == 0) {
        return;
    }
    dropGraph(ctx.graph);
    dropGraph(ctx.graphSolve);
    dropGraph(ctx.graphFactor);
    dropGraph(ctx.graphResidual);
    dropGraph(ctx.graphCorrect);
    dropGraph(ctx.graph64);
    dropGraph(ctx.graph64All);
    dropGraph(ctx.graphStep);
    dropGraph(ctx.graphSolveScored);
    dropGraph(ctx.graphStepScored);
    const DeviceNet& dn = *ctx.dn;
    const DevNet& net = dn.view;
    const size_t S = ctx.S;
    const bool mixed = ctx.precision == 1;
    if (mixed && !ctx.lu32.p) ctx.lu32.alloc(static_cast<size_t>(net.nLu) * 4 * S * 4);
    if (!mixed && !ctx.lu64.p) ctx.lu64.alloc(static_cast<size_t>(net.nLu) * 4 * S * 8);
    const DevBatch b = ctx.batch();
    const Settings cfg = ctx.cfg;
    const bool rl = ctx.rl.nRl > 0 && cfg.reactiveLimits;
    const bool dsOn = ctx.ds.nDs > 0 && cfg.distributedSlack;
    cudaStream_t st = ctx.stream;
    const Hybrid hy = ctx.hybrid();
    const Hybrid* hp = ctx.useHybrid() ? &hy : nullptr;
    const int nLevels = static_cast<int>(dn.levelPtr.size()) - 1;
    // part 1: fill, test, distributed slack, reactive limits, lane counts
    ctx.graph = captureInto(st, [&] {
        launchIterationStart(b, st);
        launchFill(net, b, true, rl || dsOn, st);
        if (cfg.norm2Threshold > 0.0) launchNorm2(net, b, st);
        launchTest(net, b, cfg, rl ? ctx.rl.remainingPv : nullptr, st);
        if (dsOn) launchDistributedSlack(b, ctx.ds, cfg, st);
        if (rl) launchReactiveLimits(net, b, ctx.rl, cfg, st);
        launchCountSolving(b, mixed ? cfg.refineBelow : -1.0, cfg.maxIter, st);
    });
    if (!mixed) {
        // part 2 (FP64): factorization, solves, (the linear-solve scoring,) step
        for (bool scoredVariant : {false, true}) {
            cudaGraphExec_t g = captureInto(st, [&] {
                launchFactor(net, b, dn.levelPtr.data(), dn.levelSplit.data(), nLevels, false, hp, st);
                launchSolve(net, b, dn.fwd(), dn.bwd(), false, false, hp, st);
                if (scoredVariant) launchScoreSolve(net, b, cfg, st);
                launchStep(net, b, cfg, st);
            });
            (scoredVariant ? ctx.graphSolveScored : ctx.graphSolve) = g;
        }
    } else {
        ctx.graphFactor = captureInto(st, [&] {
            launchFactor(net, b, dn.levelPtr.data(), dn.levelSplit.data(), nLevels, true, hp, st);
            launchCountFp64(b, st);
        });
        ctx.graphSolve = captureInto(st, [&] { launchSolve(net, b, dn.fwd(), dn.bwd(), true, false, hp, st); });
        if (ctx.refinementSteps > 0) {
            // one refinement step of the lanes still refining: the FP64 residual, the correction solve (dx += d), and
            // which lanes' correction is still above the bound
            DevBatch br = b;
            br.laneMask = b.refine;
            ctx.graphResidual = captureInto(st, [&] { launchResidual(net, br, st); });
            ctx.graphCorrect = captureInto(st, [&] {
                launchSolve(net, br, dn.fwd(), dn.bwd(), true, true, hp, st);
                launchCorrectionCheck(net, br, cfg.corrBound, st);
            });
        }
        ctx.graphStep = captureInto(st, [&] { launchStep(net, b, cfg, st); });
        ctx.graphStepScored = captureInto(st, [&] {
            launchScoreSolve(net, b, cfg, st);
            launchStep(net, b, cfg, st);
        });
    }
    ctx.graphKey = key;
    ctx.graphBatch = now;
    ctx.graphCfg = ctx.cfg;
}

// Mixed precision: the FP64 refactor and solve of the flagged lanes (captured on first use: it allocates the FP64
// factors).
void launchFp64Redo(BatchContext& ctx) {
    if (!ctx.graph64) {
        const DeviceNet& dn = *ctx.dn;
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

// MIXED_FP64_NEAR: the FP64 factorization and solves of every factorizing lane (captured on first use).
void launchFp64All(BatchContext& ctx) {
    if (!ctx.graph64All) {
        const DeviceNet& dn = *ctx.dn;
        const DevBatch b64 = fp64AllView(ctx);
        const Hybrid hy = ctx.hybrid();
        const Hybrid* hp = ctx.useHybrid() ? &hy : nullptr;
        cudaStream_t st = ctx.stream;
        ctx.graph64All = captureInto(st, [&] {
            launchFactor(dn.view, b64, dn.levelPtr.data(), dn.levelSplit.data(),
                         static_cast<int>(dn.levelPtr.size()) - 1, false, hp, st);
            launchSolve(dn.view, b64, dn.fwd(), dn.bwd(), false, false, hp, st);
        });
    }
    OLF_CUDA(cudaGraphLaunch(ctx.graph64All, ctx.stream));
}

// One Newton iteration launched phase by phase with CUDA events between the phases (the same kernels in the same
// order as the two captured graphs); the phase times and the lanes that factorized accumulate in the context.
// Returns false when no lane is left iterating.
// The factorization / one solve of an iteration under the context's schedule (level launches or cooperative sweeps).
void factorPhase(BatchContext& ctx, const DevBatch& b, bool fp32) {
    const DeviceNet& dn = *ctx.dn;
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
    const DeviceNet& dn = *ctx.dn;
    if (ctx.schedule == SCHEDULE_COOP) {
        OLF_CUDA(launchSolveCoop(dn.view, b, dn.coop, fp32, fromResidual, ctx.stream));
        return;
    }
    const Hybrid hy = ctx.hybrid();
    launchSolve(dn.view, b, dn.fwd(), dn.bwd(), fp32, fromResidual, ctx.useHybrid() ? &hy : nullptr, ctx.stream);
}

// The refinement steps of a mixed-precision iteration, launched directly: for the lanes still refining, the FP64
// residual, the correction solve and the check of its size; until no lane's correction is above the bound.
void refinementSteps(BatchContext& ctx, const DevBatch& b) {
    const DeviceNet& dn = *ctx.dn;
    cudaStream_t st = ctx.stream;
    DevBatch br = b;
    br.laneMask = b.refine;
    for (int r = 0; r < ctx.refinementSteps; r++) {
        launchResidual(dn.view, br, st);
        solvePhase(ctx, br, true, true);
        launchCorrectionCheck(dn.view, br, ctx.cfg.corrBound, st);
        OLF_CUDA(cudaMemcpyAsync(ctx.hostActive + 2, static_cast<int*>(ctx.nActive.p) + 2, 4, cudaMemcpyDeviceToHost,
                                 st));
        OLF_CUDA(cudaStreamSynchronize(st));
        if (ctx.hostActive[2] <= 0) break;
    }
}

// The linear-solve scoring runs in an iteration where some lane is scored (the host read the count after the test).
bool scoreDue(const BatchContext& ctx) { return ctx.hostActive[4] > 0; }

// Mixed precision under MIXED_FP64_NEAR: an iteration in which some factorizing lane's max |F| is below refineBelow
// (the count the host read after the test) runs in FP64 for all its lanes.
bool fp64Iteration(const BatchContext& ctx) {
    return ctx.precision == 1 && ctx.mixedPolicy == MIXED_FP64_NEAR && ctx.hostActive[2] > 0;
}

// One Newton iteration's factorization, solves, refinement, FP64 refactor and step with cooperative sweeps (the
// cooperative launches are not captured in graphs).
void coopIteration(BatchContext& ctx) {
    const DeviceNet& dn = *ctx.dn;
    const bool mixed = ctx.precision == 1;
    cudaStream_t st = ctx.stream;
    const DevBatch b = ctx.batch();
    if (fp64Iteration(ctx)) {
        ctx.fp64Iterations++;
        const DevBatch b64 = fp64AllView(ctx);
        factorPhase(ctx, b64, false);
        solvePhase(ctx, b64, false, false);
        if (scoreDue(ctx)) launchScoreSolve(dn.view, b, ctx.cfg, st);
        launchStep(dn.view, b, ctx.cfg, st);
        return;
    }
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
    if (scoreDue(ctx)) launchScoreSolve(dn.view, b, ctx.cfg, st);
    launchStep(dn.view, b, ctx.cfg, st);
}

bool phaseTimedIteration(BatchContext& ctx) {
    const DeviceNet& dn = *ctx.dn;
    const DevNet& net = dn.view;
    const bool mixed = ctx.precision == 1;
    const bool rl = ctx.rl.nRl > 0 && ctx.cfg.reactiveLimits;
    const bool dsOn = ctx.ds.nDs > 0 && ctx.cfg.distributedSlack;
    const DevBatch b = ctx.batch();
    cudaStream_t st = ctx.stream;
    cudaEvent_t ev[7];
    for (auto& e : ev) OLF_CUDA(cudaEventCreate(&e));
    OLF_CUDA(cudaEventRecord(ev[0], st));
    launchIterationStart(b, st);
    launchFill(net, b, true, rl || dsOn, st);
    OLF_CUDA(cudaEventRecord(ev[1], st));
    if (ctx.cfg.norm2Threshold > 0.0) launchNorm2(net, b, st);
    launchTest(net, b, ctx.cfg, rl ? ctx.rl.remainingPv : nullptr, st);
    if (dsOn) launchDistributedSlack(b, ctx.ds, ctx.cfg, st);
    if (rl) launchReactiveLimits(net, b, ctx.rl, ctx.cfg, st);
    launchCountSolving(b, mixed ? ctx.cfg.refineBelow : -1.0, ctx.cfg.maxIter, st);
    OLF_CUDA(cudaEventRecord(ev[2], st));
    OLF_CUDA(cudaMemcpyAsync(ctx.hostActive, ctx.nActive.p, 5 * sizeof(int), cudaMemcpyDeviceToHost, st));
    OLF_CUDA(cudaStreamSynchronize(st));
    float ms[6] = {0, 0, 0, 0, 0, 0};
    OLF_CUDA(cudaEventElapsedTime(&ms[0], ev[0], ev[1]));
    OLF_CUDA(cudaEventElapsedTime(&ms[1], ev[1], ev[2]));
    const bool live = ctx.hostActive[0] > 0;
    const int solving = ctx.hostActive[1];
    if (live && solving > 0 && fp64Iteration(ctx)) {
        OLF_CUDA(cudaEventRecord(ev[2], st));
        const DevBatch b64 = fp64AllView(ctx);
        factorPhase(ctx, b64, false);
        OLF_CUDA(cudaEventRecord(ev[3], st));
        solvePhase(ctx, b64, false, false);
        OLF_CUDA(cudaEventRecord(ev[4], st));
        if (scoreDue(ctx)) launchScoreSolve(net, b, ctx.cfg, st);
        OLF_CUDA(cudaEventRecord(ev[5], st));
        launchStep(net, b, ctx.cfg, st);
        OLF_CUDA(cudaEventRecord(ev[6], st));
        OLF_CUDA(cudaEventSynchronize(ev[6]));
        for (int i = 2; i < 6; i++) OLF_CUDA(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]));
        ctx.phaseLanes += solving;
        ctx.fp64Iterations++;
    } else if (live && solving > 0) {
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
        if (scoreDue(ctx)) launchScoreSolve(net, b, ctx.cfg, st);
        OLF_CUDA(cudaEventRecord(ev[5], st));
        launchStep(net, b, ctx.cfg, st);
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
    ctx.hasLaneLive = req.laneLive != nullptr;
    if (req.laneLive) {
        // the staging copy outlives the asynchronous upload: it sits in the pinned outage bits' shadow vector
        ctx.liveHost.assign(ctx.S, 0);
        for (int s2 = 0; s2 < ctx.nS; s2++) ctx.liveHost[s2] = req.laneLive[s2] ? 1 : 0;
        OLF_CUDA(cudaMemcpyAsync(ctx.laneLive.p, ctx.liveHost.data(), ctx.S, cudaMemcpyHostToDevice, st));
        OLF_CUDA(cudaStreamSynchronize(st));
    }
}

// Device-side install of the uploaded inputs: every lane gets the base vectors, then the per-scenario overrides; lane
// state and reactive-limit state reset.  Repeatable (the autotuner reinstalls the same batch for every candidate).
void installLanes(BatchContext& ctx) {
    // mixed precision: a failed lane restarts once in FP64 (the persistent tiles: with every solve refined to the
    // correction bound); not with reactive limits, whose restarts carry the outer loop's state
    ctx.fp64RestartOn = ctx.precision == 1 && ctx.fp64Restart && !(ctx.rl.nRl > 0 && ctx.cfg.reactiveLimits) &&
                        !(ctx.ds.nDs > 0 && ctx.cfg.distributedSlack);
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
    OLF_CUDA(cudaMemsetAsync(ctx.nActive.p, 0, sizeof(int), st));
    laneInitKernel<<<(ctx.S + 127) / 128, 128, 0, st>>>(ctx.batch());
    if (ctx.ds.nDs > 0) OLF_CUDA(cudaMemsetAsync(ctx.dsFailed.p, 0, ctx.dsFailed.bytes, st));
    OLF_CUDA(cudaMemsetAsync(ctx.dsRestartBuf.p, 0, ctx.dsRestartBuf.bytes, st));
    if (ctx.rl.nRl > 0) {
        OLF_CUDA(cudaMemsetAsync(ctx.rlLimitType.p, 0, ctx.rlLimitType.bytes, st));
        OLF_CUDA(cudaMemsetAsync(ctx.rlSwitchCount.p, 0, ctx.rlSwitchCount.bytes, st));
        OLF_CUDA(cudaMemsetAsync(ctx.rlPassSwitched.p, 0, ctx.rlPassSwitched.bytes, st));
    }
}

int roundCap(const BatchContext& ctx) {
    // a fallback restart and an FP64 restart each add one solve
    const int solves = 1 + (ctx.fallbackStart && ctx.hasX0Base && ctx.hasX0Full ? 1 : 0) + (ctx.fp64RestartOn ? 1 : 0);
    return ctx.cfg.reactiveLimits || ctx.cfg.distributedSlack ? (ctx.cfg.maxOuter + 1) * (ctx.cfg.maxIter + 1)
                                                                : solves * (ctx.cfg.maxIter + 1);
}

// The Newton iterations under the context's schedule; returns the batched iterations run (level launches) or 0.
// Fallback mode, before the first iteration: each lane starts from whichever of its own start (x0Full) and the base
// start (x0Base) has the smaller max |F| (two mismatch-only fills over all lanes).
void selectStarts(BatchContext& ctx) {
    const DeviceNet& dn = *ctx.dn;
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

// ---------------------------------------------------------------------------------------------------------------
// The Newton loop inside one graph launch: a conditional WHILE node runs one iteration per pass of its body, and the
// decisions the host loop takes between the iteration's graphs (any lane left, any lane factorizing, refinement
// steps, FP64 refactor, scoring) are conditional IF / WHILE nodes whose handles small kernels set from the lane
// counts.  The iteration counter bounds the loop at the same cap as the host loop.  loopState ints: 0 iterations,
// 1 refinement steps of the iteration, 2 this iteration factorizes in FP32 (mixed) or at all (FP64), 3 it factorizes
// in FP64 (MIXED_FP64_NEAR), 4 FP64 iterations so far.
// ---------------------------------------------------------------------------------------------------------------
__global__ void loopResetKernel(int* state) {
    for (int i = 0; i < 8; i++) state[i] = 0;
}

__global__ void loopCondKernel(cudaGraphConditionalHandle hMain, cudaGraphConditionalHandle hWork,
                               cudaGraphConditionalHandle hScore, cudaGraphConditionalHandle hNear, const int* nActive,
                               int* state, int cap, int mixed, int nearPolicy) {
    const int k = ++state[0];
    const bool live = nActive[0] > 0;
    const bool solving = live && nActive[1] > 0;
    const bool near = mixed && nearPolicy && solving && nActive[2] > 0;
    const bool work = solving && !near;
    state[1] = 0;
    state[2] = work ? 1 : 0;
    state[3] = near ? 1 : 0;
    state[4] += near ? 1 : 0;
    cudaGraphSetConditional(hMain, live && k < cap ? 1u : 0u);
    cudaGraphSetConditional(hWork, work ? 1u : 0u);
    cudaGraphSetConditional(hScore, solving && nActive[4] > 0 ? 1u : 0u);
    if (mixed) cudaGraphSetConditional(hNear, near ? 1u : 0u);
}

// Mixed precision, after the FP32 factorization and solves: refinement while some lane is below refineBelow, then
// the FP64 refactor of the lanes the FP32 factorization flagged
__global__ void loopMixedKernel(cudaGraphConditionalHandle hRefine, cudaGraphConditionalHandle hRedo,
                                const int* nActive, const int* state, int refineSteps) {
    const bool far = state[2] != 0;
    cudaGraphSetConditional(hRefine, far && refineSteps > 0 && nActive[2] > 0 ? 1u : 0u);
    cudaGraphSetConditional(hRedo, far && nActive[3] > 0 ? 1u : 0u);
}

__global__ void refineCondKernel(cudaGraphConditionalHandle hRefine, const int* nActive, int* state, int refineSteps) {
    const int r = ++state[1];
    cudaGraphSetConditional(hRefine, nActive[2] > 0 && r < refineSteps ? 1u : 0u);
}

// A conditional node after the capture's current dependencies on st; returns its body graph.
cudaGraph_t addConditional(cudaStream_t st, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type) {
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaGraph_t cg;
    OLF_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &nd));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    OLF_CUDA(cudaGraphAddNode(&node, cg, deps, nd, &p));
    OLF_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    return p.conditional.phGraph_out[0];
}

// Captures the launches fn makes on stream cs into graph g (a conditional node's body).
void captureBody(cudaStream_t cs, cudaGraph_t g, const std::function<void(cudaStream_t)>& fn) {
    OLF_CUDA(cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    fn(cs);
    cudaGraph_t out;
    OLF_CUDA(cudaStreamEndCapture(cs, &out));
}

cudaGraphConditionalHandle newHandle(cudaGraph_t owner) {
    cudaGraphConditionalHandle h;
    OLF_CUDA(cudaGraphConditionalHandleCreate(&h, owner, 0, cudaGraphCondAssignDefault));
    return h;
}

// Appends one context's device-resident Newton loop to graph g as a branch with no dependencies: the loop state reset,
// the WHILE node, the cap of lanes still iterating, and (withResults) the scenario-major result gather.  Three
// capture streams: cs[0] for the branch, cs[1] for the WHILE body, cs[2] for the bodies nested in it.
void appendNewtonLoop(BatchContext& ctx, cudaGraph_t g, const cudaStream_t* cs, bool withResults,
                      cudaEvent_t resultsDone) {
    const DeviceNet& dn = *ctx.dn;
    const DevNet& net = dn.view;
    const bool mixed = ctx.precision == 1;
    const size_t S = ctx.S;
    if (mixed && !ctx.lu32.p) ctx.lu32.alloc(static_cast<size_t>(net.nLu) * 4 * S * 4);
    if (!ctx.lu64.p) ctx.lu64.alloc(static_cast<size_t>(net.nLu) * 4 * S * 8);
    if (!ctx.loopState.p) ctx.loopState.alloc(8 * sizeof(int));
    const DevBatch b = ctx.batch();
    const DevBatch b64 = fp64View(ctx), b64all = fp64AllView(ctx);
    DevBatch br = b;
    br.laneMask = b.refine;
    const Settings cfg = ctx.cfg;
    const bool rl = ctx.rl.nRl > 0 && cfg.reactiveLimits;
    const bool dsOn = ctx.ds.nDs > 0 && cfg.distributedSlack;
    const Hybrid hy = ctx.hybrid();
    const Hybrid* hp = ctx.useHybrid() ? &hy : nullptr;
    const int nLevels = static_cast<int>(dn.levelPtr.size()) - 1;
    int* state = ctx.loopState.as<int>();
    const int* nActive = static_cast<const int*>(ctx.nActive.p);
    const int cap = roundCap(ctx);
    const int steps = ctx.refinementSteps;
    const bool nearPolicy = ctx.mixedPolicy == MIXED_FP64_NEAR;
    OLF_CUDA(cudaStreamBeginCaptureToGraph(cs[0], g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    loopResetKernel<<<1, 1, 0, cs[0]>>>(state);
    cudaGraphConditionalHandle hMain;
    OLF_CUDA(cudaGraphConditionalHandleCreate(&hMain, g, 1, cudaGraphCondAssignDefault));
    cudaGraph_t body = addConditional(cs[0], hMain, cudaGraphCondTypeWhile);
    const cudaGraphConditionalHandle hWork = newHandle(body), hScore = newHandle(body);
    const cudaGraphConditionalHandle hRefine = mixed ? newHandle(body) : 0, hRedo = mixed ? newHandle(body) : 0,
                                     hNear = mixed ? newHandle(body) : 0;
    captureBody(cs[1], body, [&](cudaStream_t st) {
        launchIterationStart(b, st);
        launchFill(net, b, true, rl || dsOn, st);
        if (cfg.norm2Threshold > 0.0) launchNorm2(net, b, st);
        launchTest(net, b, cfg, rl ? ctx.rl.remainingPv : nullptr, st);
        if (dsOn) launchDistributedSlack(b, ctx.ds, cfg, st);
        if (rl) launchReactiveLimits(net, b, ctx.rl, cfg, st);
        launchCountSolving(b, mixed ? cfg.refineBelow : -1.0, cfg.maxIter, st);
        loopCondKernel<<<1, 1, 0, st>>>(hMain, hWork, hScore, hNear, nActive, state, cap, mixed ? 1 : 0,
                                        nearPolicy ? 1 : 0);
        if (!mixed) {
            captureBody(cs[2], addConditional(st, hWork, cudaGraphCondTypeIf), [&](cudaStream_t s2) {
                launchFactor(net, b, dn.levelPtr.data(), dn.levelSplit.data(), nLevels, false, hp, s2);
                launchSolve(net, b, dn.fwd(), dn.bwd(), false, false, hp, s2);
            });
        } else {
            captureBody(cs[2], addConditional(st, hWork, cudaGraphCondTypeIf), [&](cudaStream_t s2) {
                launchFactor(net, b, dn.levelPtr.data(), dn.levelSplit.data(), nLevels, true, hp, s2);
                launchCountFp64(b, s2);
                launchSolve(net, b, dn.fwd(), dn.bwd(), true, false, hp, s2);
            });
            loopMixedKernel<<<1, 1, 0, st>>>(hRefine, hRedo, nActive, state, steps);
            if (steps > 0) {
                captureBody(cs[2], addConditional(st, hRefine, cudaGraphCondTypeWhile), [&](cudaStream_t s2) {
                    launchResidual(net, br, s2);
                    launchSolve(net, br, dn.fwd(), dn.bwd(), true, true, hp, s2);
                    launchCorrectionCheck(net, br, cfg.corrBound, s2);
                    refineCondKernel<<<1, 1, 0, s2>>>(hRefine, nActive, state, steps);
                });
            }
            captureBody(cs[2], addConditional(st, hRedo, cudaGraphCondTypeIf), [&](cudaStream_t s2) {
                launchFactor(net, b64, dn.levelPtr.data(), dn.levelSplit.data(), nLevels, false, hp, s2);
                launchSolve(net, b64, dn.fwd(), dn.bwd(), false, false, hp, s2);
            });
            captureBody(cs[2], addConditional(st, hNear, cudaGraphCondTypeIf), [&](cudaStream_t s2) {
                launchFactor(net, b64all, dn.levelPtr.data(), dn.levelSplit.data(), nLevels, false, hp, s2);
                launchSolve(net, b64all, dn.fwd(), dn.bwd(), false, false, hp, s2);
            });
        }
        captureBody(cs[2], addConditional(st, hScore, cudaGraphCondTypeIf),
                    [&](cudaStream_t s2) { launchScoreSolve(net, b, cfg, s2); });
        launchStep(net, b, cfg, st);
    });
    capKernel<<<(ctx.S + 127) / 128, 128, 0, cs[0]>>>(b);
    if (withResults) {
        const int n = ctx.net->host.n;
        dim3 blk(32, 8), grd((n + 31) / 32, (ctx.nS + 31) / 32);
        resultsKernel<<<grd, blk, 0, cs[0]>>>(ctx.x.as<double>(), ctx.iter.as<int>(), ctx.normOut.as<double>(),
                                              ctx.status.as<int>(), ctx.out.as<double>(), n, ctx.nS, ctx.S);
        // an event node: a stream outside the graph can wait for this branch's results alone
        if (resultsDone) OLF_CUDA(cudaEventRecordWithFlags(resultsDone, cs[0], cudaEventRecordExternal));
    }
    cudaGraph_t top;
    OLF_CUDA(cudaStreamEndCapture(cs[0], &top));
}

// The key of everything a loop graph bakes in besides the batch view and settings.
long long loopKey(const BatchContext& ctx) {
    return ((((static_cast<long long>(ctx.narrowLanes) * 2 + (ctx.regionFactor ? 1 : 0)) * 2 + (ctx.regionSolve ? 1 : 0)) *
                 2 + (ctx.subtrees ? 1 : 0)) * 2 + ctx.precision) * 4096 * 64 +
           static_cast<long long>(ctx.refinementSteps) * 4096 * 2 + ctx.mixedPolicy * 4096 + roundCap(ctx);
}

// One context's Newton loop as one graph launch on its stream; returns the iterations run.
int runDeviceLoop(BatchContext& ctx) {
    cudaStream_t st = ctx.stream;
    const DevBatch now = ctx.batch();
    const long long key = loopKey(ctx);
    if (!ctx.loopGraph || ctx.loopGraphKey != key || std::memcmp(&now, &ctx.loopBatch, sizeof(DevBatch)) != 0 ||
        std::memcmp(&ctx.cfg, &ctx.loopCfg, sizeof(Settings)) != 0) {
        dropGraph(ctx.loopGraph);
        if (!ctx.loopStreams[0]) {
            for (auto& s : ctx.loopStreams) OLF_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        }
        cudaGraph_t g;
        OLF_CUDA(cudaGraphCreate(&g, 0));
        appendNewtonLoop(ctx, g, ctx.loopStreams, false, nullptr);
        OLF_CUDA(cudaGraphInstantiate(&ctx.loopGraph, g, 0));
        cudaGraphDestroy(g);
        ctx.loopGraphKey = key;
        ctx.loopBatch = now;
        ctx.loopCfg = ctx.cfg;
    }
    OLF_CUDA(cudaGraphLaunch(ctx.loopGraph, st));
    OLF_CUDA(cudaMemcpyAsync(ctx.hostActive + 5, ctx.loopState.p, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
    OLF_CUDA(cudaStreamSynchronize(st));
    ctx.fp64Iterations = 0;
    int st4 = 0;
    OLF_CUDA(cudaMemcpy(&st4, static_cast<int*>(ctx.loopState.p) + 4, sizeof(int), cudaMemcpyDeviceToHost));
    ctx.fp64Iterations = st4;
    return ctx.hostActive[5];
}

int runIterations(BatchContext& ctx) {
    cudaStream_t st = ctx.stream;
    const DeviceNet& dn = *ctx.dn;
    const bool mixed = ctx.precision == 1;
    const size_t S = ctx.S;
    if (mixed && !ctx.lu32.p) ctx.lu32.alloc(static_cast<size_t>(dn.view.nLu) * 4 * S * 4);
    if (!mixed && !ctx.lu64.p) ctx.lu64.alloc(static_cast<size_t>(dn.view.nLu) * 4 * S * 8);
    const int cap = roundCap(ctx);
    if (ctx.fallbackStart && ctx.hasX0Base && ctx.hasX0Full) selectStarts(ctx);
    if (ctx.deviceLoop && !ctx.phaseTiming && ctx.schedule != SCHEDULE_PERSISTENT && ctx.schedule != SCHEDULE_COOP) {
        ctx.fp64Iterations = 0;
        return runDeviceLoop(ctx);
    }
    if (ctx.schedule == SCHEDULE_PERSISTENT) {
        if (dn.view.frontF > 0) throw std::runtime_error("the persistent schedule does not run dense-front plans");
        PersistentPlan plan = dn.persistent;
        plan.maxRounds = cap;
        launchPersistent(dn.view, ctx.batch(), ctx.rl, ctx.cfg, plan, ctx.lanesPerTile, ctx.threads, mixed, st);
        OLF_CUDA(cudaGetLastError());
        return 0;
    }
    captureIteration(ctx);
    ctx.fp64Iterations = 0;
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
        OLF_CUDA(cudaMemcpyAsync(ctx.hostActive, ctx.nActive.p, 5 * sizeof(int), cudaMemcpyDeviceToHost, st));
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
            OLF_CUDA(cudaGraphLaunch(scoreDue(ctx) ? ctx.graphSolveScored : ctx.graphSolve, st));
            continue;
        }
        if (fp64Iteration(ctx)) {
            ctx.fp64Iterations++;
            launchFp64All(ctx);
            OLF_CUDA(cudaGraphLaunch(scoreDue(ctx) ? ctx.graphStepScored : ctx.graphStep, st));
            continue;
        }
        // mixed: FP32 factorization, then (while the FP32 solves run) the count of lanes flagged for FP64
        OLF_CUDA(cudaGraphLaunch(ctx.graphFactor, st));
        OLF_CUDA(cudaMemcpyAsync(ctx.hostActive + 3, static_cast<int*>(ctx.nActive.p) + 3, 4, cudaMemcpyDeviceToHost,
                                 st));
        OLF_CUDA(cudaEventRecord(ctx.countReady, st));
        OLF_CUDA(cudaGraphLaunch(ctx.graphSolve, st));
        if (ctx.graphResidual && ctx.hostActive[2] > 0) {
            // the lanes near convergence refine until their correction is below the bound (at most refinementSteps)
            for (int r = 0; r < ctx.refinementSteps; r++) {
                OLF_CUDA(cudaGraphLaunch(ctx.graphResidual, st));
                OLF_CUDA(cudaGraphLaunch(ctx.graphCorrect, st));
                OLF_CUDA(cudaMemcpyAsync(ctx.hostActive + 2, static_cast<int*>(ctx.nActive.p) + 2, 4,
                                         cudaMemcpyDeviceToHost, st));
                OLF_CUDA(cudaStreamSynchronize(st));
                if (ctx.hostActive[2] <= 0) break;
            }
        }
        OLF_CUDA(cudaEventSynchronize(ctx.countReady));
        if (ctx.hostActive[3] > 0) launchFp64Redo(ctx);
        OLF_CUDA(cudaGraphLaunch(scoreDue(ctx) ? ctx.graphStepScored : ctx.graphStep, st));
    }
    capKernel<<<(ctx.S + 127) / 128, 128, 0, st>>>(ctx.batch());
    return k;
}

// Times every candidate schedule on the installed batch and keeps the fastest (the batch is reinstalled before each).
void autotune(BatchContext& ctx) {
    struct Candidate { int schedule, lanes, threads; };
    std::vector<Candidate> cands;
    for (int narrow : {0, 1, 2, 4}) cands.push_back({SCHEDULE_LEVELS, narrow, 256});
    if (ctx.dn->regionSlots > 0) {
        for (int narrow : {0, 2}) cands.push_back({SCHEDULE_LEVELS_SHARED, narrow, 256});
    }
    if (ctx.dn->fwdRegionSlots > 0 || ctx.dn->bwdRegionSlots > 0) {
        cands.push_back({SCHEDULE_LEVELS_SHARED_ALL, 0, 256});
    }
    if (ctx.dn->sub.nBins > 0) cands.push_back({SCHEDULE_SUBTREES, 0, 256});
    cands.push_back({SCHEDULE_COOP, 0, 512});
    // the persistent tiles run neither dense-front plans, nor the distributed-slack loop, the 2-norm test or the
    // MAX_VOLTAGE_CHANGE clamp
    const bool persistentFits = ctx.dn->view.frontF == 0 && !ctx.cfg.distributedSlack && ctx.cfg.norm2Threshold <= 0.0 &&
                                ctx.cfg.svsMode == 0;
    if (persistentFits) {
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
        ctx.regionFactor = c.schedule == SCHEDULE_LEVELS_SHARED || c.schedule == SCHEDULE_LEVELS_SHARED_ALL ||
                           c.schedule == SCHEDULE_SUBTREES;
        ctx.regionSolve = c.schedule == SCHEDULE_LEVELS_SHARED_ALL || c.schedule == SCHEDULE_SUBTREES;
        ctx.subtrees = c.schedule == SCHEDULE_SUBTREES;
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

void setDistributedSlack(BatchContext& ctx, int nDs, const int* row, const double* factor, const double* baseTarget,
                         const double* maxDelta, const double* minDelta, int slackRow, double slackTargetP) {
    OLF_CUDA(cudaSetDevice(ctx.device));
    const int n = ctx.net->host.n;
    if (nDs <= 0) {
        ctx.ds = DevDs{};
        return;
    }
    if (slackRow < 0 || slackRow >= n) throw std::runtime_error("bad slackBusPhiRow");
    double fsum = 0.0;
    for (int i = 0; i < nDs; i++) {
        if (row[i] < 0 || row[i] >= n) throw std::runtime_error("bad distributedSlackBusPhiRow");
        if (!(factor[i] >= 0.0)) throw std::runtime_error("negative distributed-slack factor");
        if (!(minDelta[i] <= 0.0 && maxDelta[i] >= 0.0)) {
            throw std::runtime_error("distributed-slack bounds must contain the base target");
        }
        fsum += factor[i];
    }
    if (!(fsum > 0.0)) throw std::runtime_error("distributed-slack factors sum to zero");
    std::vector<double> f(factor, factor + nDs);
    for (double& v : f) v /= fsum;
    const size_t S = ctx.S;
    auto up = [&](DeviceBuffer& d, const void* src, size_t bytes) {
        d.alloc(bytes);
        OLF_CUDA(cudaMemcpy(d.p, src, bytes, cudaMemcpyHostToDevice));
    };
    up(ctx.dsRow, row, nDs * 4);
    up(ctx.dsFactor, f.data(), nDs * 8);
    up(ctx.dsBase, baseTarget, nDs * 8);
    up(ctx.dsMax, maxDelta, nDs * 8);
    up(ctx.dsMin, minDelta, nDs * 8);
    ctx.dsPrev.alloc(static_cast<size_t>(nDs) * S * 8);
    ctx.dsFailed.alloc(S);
    OLF_CUDA(cudaDeviceSynchronize());   // the pageable uploads have landed before the context's stream reads them
    DevDs& d = ctx.ds;
    d.nDs = nDs;
    d.row = ctx.dsRow.as<int>();
    d.factor = ctx.dsFactor.as<double>();
    d.baseTarget = ctx.dsBase.as<double>();
    d.maxDelta = ctx.dsMax.as<double>();
    d.minDelta = ctx.dsMin.as<double>();
    d.slackRow = slackRow;
    d.slackTargetP = slackTargetP;
    d.prevTarget = ctx.dsPrev.as<double>();
    d.failed = ctx.dsFailed.as<int8_t>();
}

void setStrongestPvKeys(BatchContext& ctx, const double* nomV, const int* pRow, const double* staticP,
                        const int* idRank) {
    OLF_CUDA(cudaSetDevice(ctx.device));
    const int nRl = ctx.rl.nRl;
    const int n = ctx.net->host.n;
    for (int i = 0; i < nRl; i++)
        if (pRow[i] >= n) throw std::runtime_error("bad reactiveLimit pRow");
    auto put = [&](DeviceBuffer& d, const void* src, size_t bytes) {
        OLF_CUDA(cudaMemcpyAsync(d.p, src, bytes, cudaMemcpyHostToDevice, ctx.stream));
    };
    put(ctx.rlNomV, nomV, nRl * 8);
    put(ctx.rlPRow, pRow, nRl * 4);
    put(ctx.rlStaticP, staticP, nRl * 8);
    put(ctx.rlIdRank, idRank, nRl * 4);
    OLF_CUDA(cudaStreamSynchronize(ctx.stream));
    ctx.rlKeys = true;
}

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
    if (ctx.rl.nRl > 0 && !ctx.rlKeys) {
        // batch_solve_jni.cu:103-111: without the keys OLF's strongest-bus-stays-PV rule cannot be reproduced
        throw std::runtime_error("reactive-limit entries installed without the forced-PV election keys "
                                 "(olfgpu_set_reactive_limit_strongest_pv_keys)");
    }
    if (req.stateVectorScalingMode != SVS_NONE && req.stateVectorScalingMode != SVS_MAX_VOLTAGE_CHANGE) {
        throw std::runtime_error("state vector scaling mode " + std::to_string(req.stateVectorScalingMode) +
                                 " is not supported (NONE 0 and MAX_VOLTAGE_CHANGE 2 are)");
    }
    const bool clamp = req.stateVectorScalingMode == SVS_MAX_VOLTAGE_CHANGE;
    if (clamp && !req.varType) throw std::runtime_error("MAX_VOLTAGE_CHANGE needs the variable types (varType)");
    if (clamp && !(req.maxDv > 0.0 && req.maxDphi > 0.0)) {
        throw std::runtime_error("MAX_VOLTAGE_CHANGE needs positive maxDv and maxDphi");
    }
    if ((clamp || req.convEpsPerEq > 0.0) && ctx.schedule == SCHEDULE_PERSISTENT) {
        throw std::runtime_error("the persistent schedule runs the ||F||inf test and the plain step only");
    }
    Settings cfg = ctx.cfg;
    cfg.maxIter = req.maxIter;
    cfg.norm2Threshold = req.convEpsPerEq > 0.0 ? std::sqrt(req.convEpsPerEq * req.convEpsPerEq * n) : 0.0;
    cfg.svsMode = req.stateVectorScalingMode;
    cfg.maxDv = req.maxDv;
    cfg.maxDphi = req.maxDphi;
    cfg.corrBound = ctx.corrBound;
    cfg.polishBelow = ctx.fallbackStart ? ctx.polishRatio * req.tol : 0.0;
    cfg.realistic = ctx.hasVCheck ? 1 : 0;
    cfg.minV = ctx.realisticMinV;
    cfg.maxV = ctx.realisticMaxV;
    if (clamp) {
        std::vector<int8_t> vt(n);
        for (int r = 0; r < n; r++) vt[r] = static_cast<int8_t>(req.varType[r] == VAR_BUS_V || req.varType[r] == VAR_BUS_PHI
                                                                     ? req.varType[r] : -1);
        // stream-ordered (a pageable copy is staged before the call returns, so vt may go)
        OLF_CUDA(cudaMemcpyAsync(ctx.varType.p, vt.data(), n, cudaMemcpyHostToDevice, ctx.stream));
    }
    ctx.hasVarType = clamp;
    cfg.tol = req.tol;
    cfg.rlTol = req.reactiveLimitTol;
    cfg.maxOuter = req.maxOuter;
    cfg.maxSwitch = req.maxPqPvSwitch;
    cfg.reactiveLimits = ctx.rl.nRl > 0 && ctx.reactiveLimitsLoop && !req.skipReactiveLimits ? 1 : 0;
    cfg.distributedSlack = ctx.ds.nDs > 0 && ctx.dsLoop ? 1 : 0;
    cfg.slackDistTol = req.slackDistTol;
    cfg.rejectDsFailure = req.rejectDsFailure ? 1 : 0;
    if (cfg.distributedSlack && ctx.schedule == SCHEDULE_PERSISTENT) {
        throw std::runtime_error("the persistent schedule does not run the distributed-slack outer loop");
    }
    if (cfg.distributedSlack && ctx.fallbackStart) {
        throw std::runtime_error("the fallback start is not available with distributed slack");
    }
    cfg.mixed = ctx.precision;
    cfg.refinementSteps = ctx.refinementSteps;
    cfg.refineBelow = ctx.refineBelow;
    cfg.growthLimit = ctx.growthLimit;
    ctx.cfg = cfg;   // (the iteration graphs are re-captured when the settings they baked in change)
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
    if (loopGraph) cudaGraphExecDestroy(loopGraph);
    for (cudaStream_t s : capStreams)
        if (s) cudaStreamDestroy(s);
    for (cudaEvent_t e : ready) cudaEventDestroy(e);
    for (cudaEvent_t e : done) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
    if (hostItems) cudaFreeHost(hostItems);
}

MultiContext* createMultiContext(const std::vector<BatchContext*>& members) {
    if (members.empty()) throw std::runtime_error("a multi-grid context needs at least one batch context");
    const int device = members[0]->device;
    for (const BatchContext* c : members) {
        if (!c) throw std::runtime_error("null batch context");
        if (c->device != device) throw std::runtime_error("the batch contexts of a multi-grid launch share one device");
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
    m->done.resize(members.size());
    for (auto& e : m->done) OLF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
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

// The members' device-resident Newton loops as the branches of one graph (rebuilt when a member's schedule, batch view
// or settings changed).
void launchMultiLoops(MultiContext& m) {
    const size_t k = m.members.size();
    bool same = m.loopGraph && m.loopKeys.size() == k;
    for (size_t i = 0; same && i < k; i++) {
        const BatchContext& c = *m.members[i];
        const DevBatch now = c.batch();
        same = m.loopKeys[i] == loopKey(c) && std::memcmp(&now, &m.loopBatches[i], sizeof(DevBatch)) == 0 &&
               std::memcmp(&c.cfg, &m.loopCfgs[i], sizeof(Settings)) == 0;
    }
    if (!same) {
        dropGraph(m.loopGraph);
        if (!m.capStreams[0]) {
            for (auto& s : m.capStreams) OLF_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        }
        cudaGraph_t g;
        OLF_CUDA(cudaGraphCreate(&g, 0));
        m.loopKeys.clear();
        m.loopBatches.clear();
        m.loopCfgs.clear();
        for (size_t i = 0; i < k; i++) {
            BatchContext* c = m.members[i];
            appendNewtonLoop(*c, g, m.capStreams, true, m.done[i]);
            m.loopKeys.push_back(loopKey(*c));
            m.loopBatches.push_back(c->batch());
            m.loopCfgs.push_back(c->cfg);
        }
        OLF_CUDA(cudaGraphInstantiate(&m.loopGraph, g, 0));
        cudaGraphDestroy(g);
    }
    OLF_CUDA(cudaGraphLaunch(m.loopGraph, m.stream));
}

// Lanes of every member reset to their staged inputs, then the one launch (and the members' result gathers).
void runMulti(MultiContext& m, bool fp32) {
    cudaStream_t st = m.stream;
    for (size_t i = 0; i < m.members.size(); i++) {
        BatchContext& c = *m.members[i];
        installLanes(c);
        // each member starts from its selected starts (fallback mode), as a solo solve does
        if (c.fallbackStart && c.hasX0Base && c.hasX0Full) selectStarts(c);
        OLF_CUDA(cudaEventRecord(m.ready[i], c.stream));
        OLF_CUDA(cudaStreamWaitEvent(st, m.ready[i], 0));
    }
    if (m.lanesPerTile == 0) {
        launchMultiLoops(m);
        return;
    }
    const std::vector<int> idx = launchOrder(m, m.order);
    int tile = 0;
    for (size_t k = 0; k < idx.size(); k++) {
        BatchContext& c = *m.members[idx[k]];
        MultiItem& it = m.hostItems[k];
        it.net = c.dn->view;
        it.b = c.batch();
        it.rl = c.rl;
        it.cfg = c.cfg;
        it.plan = c.dn->persistent;
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

bool multiTilesFit(const BatchContext& c) {
    return c.dn->view.frontF == 0 && !c.cfg.distributedSlack && c.cfg.norm2Threshold <= 0.0 && c.cfg.svsMode == SVS_NONE &&
           !c.cfg.realistic && !(c.precision == 1 && c.mixedPolicy == MIXED_FP64_NEAR);
}

void autotuneMulti(MultiContext& m, bool fp32) {
    cudaEvent_t e0, e1;
    OLF_CUDA(cudaEventCreate(&e0));
    OLF_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    MultiTuning pick{};
    m.tuning.clear();
    bool tilesFit = true;      // the persistent tiles run neither dense-front plans nor the extra outer loops / tests
    for (const BatchContext* c : m.members) tilesFit = tilesFit && multiTilesFit(*c);
    {
        m.lanesPerTile = 0;
        OLF_CUDA(cudaEventRecord(e0, m.stream));
        runMulti(m, fp32);
        OLF_CUDA(cudaEventRecord(e1, m.stream));
        OLF_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        OLF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        m.tuning.push_back({0, 0, 0, ms});
        best = ms;
        pick = m.tuning.back();
    }
    if (tilesFit)
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
        if (m.lanesPerTile > 0 && !m.autotunePending && !multiTilesFit(*c)) {
            throw std::runtime_error("the persistent tiles of a multi-grid launch run the plain Newton loop with "
                                     "reactive limits only (no dense-front plan, distributed slack, 2-norm test, step "
                                     "clamp, realistic band or FP64-near policy): use lanesPerTile 0");
        }
        if (m.lanesPerTile == 0 && (c->schedule == SCHEDULE_PERSISTENT || c->schedule == SCHEDULE_COOP)) {
            throw std::runtime_error("the device-resident loops of a multi-grid launch run level schedules (0, 3, 4 or 5)");
        }
        if (c->precision != precision) {
            throw std::runtime_error("the batch contexts of a multi-grid launch share one precision");
        }
    }
    const bool fp32 = precision == 1;
    for (BatchContext* c : m.members) {
        const size_t lu = static_cast<size_t>(c->dn->view.nLu) * 4 * c->S;
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
            // device loops: a member's results go to the host on its own stream as soon as its branch of the graph
            // has gathered them, while the other branches still run; persistent tiles: after the launch
            cudaStream_t cs = st;
            if (m.lanesPerTile == 0) {
                cs = c.stream;
                OLF_CUDA(cudaStreamWaitEvent(cs, m.done[i], 0));
            }
            OLF_CUDA(cudaMemcpyAsync(outs[i], c.out.p, static_cast<size_t>(c.nS) * (c.net->host.n + 3) * 8,
                                     cudaMemcpyDeviceToHost, cs));
        }
    }
    OLF_CUDA(cudaStreamSynchronize(st));
    for (BatchContext* c : m.members) OLF_CUDA(cudaStreamSynchronize(c->stream));
    OLF_CUDA(cudaEventElapsedTime(&m.lastMs, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (BatchContext* c : m.members) {
        c->lastIterations = 0;
        if (m.lanesPerTile == 0) {
            int st[5] = {0, 0, 0, 0, 0};
            OLF_CUDA(cudaMemcpy(st, c->loopState.p, sizeof(st), cudaMemcpyDeviceToHost));
            c->lastIterations = st[0];
            c->fp64Iterations = st[4];
        }
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
    const DeviceNet& dn = *ctx.dn;
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
    OLF_CUDA(cudaMemsetAsync(ctx.nActive.p, 0, sizeof(int), st));
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
    const DeviceNet& dn = *ctx.dn;
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
    OLF_CUDA(cudaMemsetAsync(ctx.nActive.p, 0, sizeof(int), st));
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

void linearSolveBoth(BatchContext& ctx, const double* csrVals, const double* rhs, const double* rhsT, int precision,
                     double* x, double* y) {
    OLF_CUDA(cudaSetDevice(ctx.device));
    const Structure& s = ctx.net->host;
    const DeviceNet& dn = *ctx.dn;
    const DevNet& net = dn.view;
    const int n = s.n;
    const size_t S = ctx.S;
    cudaStream_t st = ctx.stream;
    const bool fp32 = precision == 1;
    if (fp32 && !ctx.lu32.p) ctx.lu32.alloc(static_cast<size_t>(net.nLu) * 4 * S * 4);
    if (!fp32 && !ctx.lu64.p) ctx.lu64.alloc(static_cast<size_t>(net.nLu) * 4 * S * 8);
    std::vector<double> J(ctx.J.bytes / 8, 0.0), F(static_cast<size_t>(n) * S, 0.0), C(static_cast<size_t>(n) * S, 0.0);
    for (int sc = 0; sc < ctx.nS; sc++) {
        for (int k = 0; k < s.nnz; k++) {
            J[static_cast<size_t>(dn.csrToA[k]) * S + sc] = csrVals[static_cast<size_t>(sc) * s.nnz + k];
        }
        for (int r = 0; r < n; r++) {
            if (rhs) F[static_cast<size_t>(r) * S + sc] = -rhs[static_cast<size_t>(sc) * n + r];
            if (rhsT) C[static_cast<size_t>(r) * S + sc] = rhsT[static_cast<size_t>(sc) * n + r];
        }
    }
    OLF_CUDA(cudaMemcpyAsync(ctx.J.p, J.data(), ctx.J.bytes, cudaMemcpyHostToDevice, st));
    OLF_CUDA(cudaMemcpyAsync(ctx.F.p, F.data(), F.size() * 8, cudaMemcpyHostToDevice, st));
    OLF_CUDA(cudaMemcpyAsync(ctx.res.p, C.data(), C.size() * 8, cudaMemcpyHostToDevice, st));
    const DevBatch b = ctx.batch();
    OLF_CUDA(cudaMemsetAsync(ctx.nActive.p, 0, sizeof(int), st));
    laneInitKernel<<<(ctx.S + 127) / 128, 128, 0, st>>>(b);
    launchFactor(net, b, dn.levelPtr.data(), dn.levelSplit.data(), static_cast<int>(dn.levelPtr.size()) - 1, fp32,
                 nullptr, st);
    std::vector<double> out(static_cast<size_t>(n) * S);
    auto gather = [&](double* dst) {
        OLF_CUDA(cudaMemcpyAsync(out.data(), ctx.dx.p, out.size() * 8, cudaMemcpyDeviceToHost, st));
        OLF_CUDA(cudaStreamSynchronize(st));
        for (int sc = 0; sc < ctx.nS; sc++)
            for (int r = 0; r < n; r++) dst[static_cast<size_t>(sc) * n + r] = out[static_cast<size_t>(r) * S + sc];
    };
    if (rhs && x) {
        launchSolve(net, b, dn.fwd(), dn.bwd(), fp32, false, nullptr, st);
        gather(x);
    }
    if (rhsT && y) {
        launchSolveTransposed(net, b, dn.fwd(), dn.bwd(), fp32, st);
        gather(y);
    }
    OLF_CUDA(cudaStreamSynchronize(st));
    OLF_CUDA(cudaGetLastError());
}

}  // namespace olfb200
