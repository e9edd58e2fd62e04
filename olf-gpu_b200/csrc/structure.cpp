// Host-side structure build: the reference-compatible equation structure and the bus-block LU plan.
#include "structure.hpp"

#include <algorithm>
#include <cstring>
#include <numeric>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>

namespace olfb200 {

namespace {

// Scatter tables {role, rowEnd, rowEq, colEnd, colVar} of the three families, in output order
// (equations/generated/{closed_branch,open_branch,shunt}_scatter.h: 0 residual, 1 jacobian, 2 skip).
const int CB_SCATTER[CB_OUTPUTS][5] = {
    {0, 0, 0, -1, -1}, {1, 0, 0, 0, 1}, {1, 0, 0, 1, 1}, {1, 0, 0, 0, 0}, {1, 0, 0, 1, 0}, {1, 0, 0, 2, 0},
    {1, 0, 0, 2, 1},   {0, 0, 1, -1, -1}, {1, 0, 1, 0, 1}, {1, 0, 1, 1, 1}, {1, 0, 1, 0, 0}, {1, 0, 1, 1, 0},
    {1, 0, 1, 2, 0},   {1, 0, 1, 2, 1},   {0, 1, 0, -1, -1}, {1, 1, 0, 0, 1}, {1, 1, 0, 1, 1}, {1, 1, 0, 0, 0},
    {1, 1, 0, 1, 0},   {1, 1, 0, 2, 0},   {1, 1, 0, 2, 1},   {0, 1, 1, -1, -1}, {1, 1, 1, 0, 1}, {1, 1, 1, 1, 1},
    {1, 1, 1, 0, 0},   {1, 1, 1, 1, 0},   {1, 1, 1, 2, 0},   {1, 1, 1, 2, 1}};
const int OB_SCATTER[OB_OUTPUTS][5] = {{0, 1, 0, -1, -1}, {1, 1, 0, 1, 1}, {0, 1, 1, -1, -1}, {1, 1, 1, 1, 1},
                                       {0, 0, 0, -1, -1}, {1, 0, 0, 0, 1}, {0, 0, 1, -1, -1}, {1, 0, 1, 0, 1}};
const int SH_SCATTER[SH_OUTPUTS][5] = {{0, 0, 0, -1, -1}, {1, 0, 0, 0, 1}, {0, 0, 1, -1, -1}, {1, 0, 1, 0, 1},
                                       {1, 0, 1, 2, 0}};

// One scatter row of one element -> (row, col); -1 when absent (csr_pattern.cu:38-71).
inline void resolveCb(const int* t, const int* ix, int& row, int& col) {
    row = col = -1;
    if (t[0] == 2) return;
    row = ix[t[1] * 2 + t[2]];
    if (t[0] == 1) col = ix[4 + t[3] * 2 + t[4]];
}
inline void resolveOb(const int* t, const int* ix, int& row, int& col) {
    row = col = -1;
    if (t[0] == 2) return;
    row = ix[t[1] * 2 + t[2]];
    if (t[0] == 1) col = ix[4 + t[3]];
}
inline void resolveSh(const int* t, const int* ix, int& row, int& col) {
    row = col = -1;
    if (t[0] == 2) return;
    row = ix[t[2]];
    if (t[0] == 1) col = (t[3] == 2) ? ix[3] : ix[2];
}

void fail(const std::string& what) { throw std::runtime_error(what); }

void checkRange(const char* what, const int* a, int count, int stride, std::initializer_list<int> slots, int lo,
                int hi) {
    for (int e = 0; e < count; e++) {
        for (int sl : slots) {
            int v = a[static_cast<size_t>(e) * stride + sl];
            if (v < lo || v >= hi) {
                fail(std::string("bad ") + what + " at elem " + std::to_string(e) + " slot " + std::to_string(sl) +
                     ": " + std::to_string(v) + " (allowed [" + std::to_string(lo) + ", " + std::to_string(hi) + "))");
            }
        }
    }
}

// The diagonal pairing of every equation row with its strong variable column (csr_pattern.cu:85-240, restricted to
// the closed-branch, open-branch, shunt and identity-row families).
std::vector<int> rowMapOf(int n, int ncb, const int* cb, int nob, const int* ob, int nsh, const int* sh, int nid,
                          const int* idRows) {
    std::vector<int> rm(n, -1);
    auto pair = [&](int row, int col) {
        if (row < 0 || col < 0) return;
        if (rm[row] == -1) rm[row] = col;
        else if (rm[row] != col) fail("conflicting diagonal pairing for equation row " + std::to_string(row));
    };
    auto pairP = [&](int prow, int phcol) { pair(prow, prow == phcol ? phcol : prow); };
    auto movedV = [&](int qrow, int vcol) {
        if (vcol >= 0 && qrow != vcol) pair(vcol, vcol);
    };
    for (int e = 0; e < ncb; e++) {
        const int* ix = cb + static_cast<size_t>(e) * CB_INDICES;
        pairP(ix[0], ix[4]);
        pairP(ix[2], ix[6]);
        pair(ix[1], ix[1]);
        pair(ix[3], ix[3]);
        movedV(ix[1], ix[5]);
        movedV(ix[3], ix[7]);
        if (ix[9] >= 0) pair(ix[9], ix[9]);
        if (ix[8] >= 0) pair(ix[8], ix[8]);
    }
    for (int e = 0; e < nob; e++) {
        const int* ix = ob + static_cast<size_t>(e) * OB_INDICES;
        pair(ix[1], ix[1]);
        pair(ix[3], ix[3]);
        movedV(ix[1], ix[4]);
        movedV(ix[3], ix[5]);
    }
    for (int e = 0; e < nsh; e++) {
        const int* ix = sh + static_cast<size_t>(e) * SH_INDICES;
        pair(ix[1], ix[1]);
        movedV(ix[1], ix[2]);
        if (ix[3] >= 0) pair(ix[3], ix[3]);
    }
    for (int i = 0; i < nid; i++) pair(idRows[i], idRows[i]);
    std::vector<char> used(n, 0);
    for (int r = 0; r < n; r++) {
        if (rm[r] < 0) fail("equation row " + std::to_string(r) + " of " + std::to_string(n) + " has no diagonal pairing");
        if (used[rm[r]]) fail("diagonal pairing is not a bijection (column " + std::to_string(rm[r]) + " claimed twice)");
        used[rm[r]] = 1;
    }
    return rm;
}

int csrAt(const std::vector<int>& rowPtr, const std::vector<int>& colIdx, int row, int col) {
    auto b = colIdx.begin() + rowPtr[row], e = colIdx.begin() + rowPtr[row + 1];
    auto it = std::lower_bound(b, e, col);
    if (it == e || *it != col) fail("CSR pattern lookup miss");
    return static_cast<int>(it - colIdx.begin());
}

}  // namespace

Structure buildStructure(int n, int ncb, const double* cbPar, const int* cbIx, int nob, const double* obPar,
                         const int* obIx, int nsh, const double* shPar, const int* shIx, int nid, const int* idRows,
                         int ordering) {
    if (n <= 0) fail("empty system (n = " + std::to_string(n) + ")");
    if (ncb < 0 || nob < 0 || nsh < 0 || nid < 0) fail("negative element count");
    // input range checks (structure_jni.cu:71-118)
    checkRange("closedBranchIndices", cbIx, ncb, CB_INDICES, {0, 1, 2, 3, 4, 5, 6, 7, 8, 9}, -1, n);
    checkRange("closedBranchIndices.alternateQRows", cbIx, ncb, CB_INDICES, {10, 11}, -1, n);
    checkRange("openBranchIndices", obIx, nob, OB_INDICES, {0, 1, 2, 3, 4, 5}, -1, n);
    checkRange("shuntIndices", shIx, nsh, SH_INDICES, {0, 1, 2, 3}, -1, n);
    checkRange("shuntIndices.alternateQRows", shIx, nsh, SH_INDICES, {4}, -1, n);
    checkRange("identityRows", idRows, nid, 1, {0}, 0, n);
    for (int e = 0; e < ncb; e++) {
        const int* ix = cbIx + static_cast<size_t>(e) * CB_INDICES;
        if (ix[8] >= 0 || ix[9] >= 0 || ix[10] >= 0 || ix[11] >= 0) {
            fail("closed branch " + std::to_string(e) +
                 ": transformer control columns and reactive relocation are not supported by this engine");
        }
        for (int k = 0; k < 8; k++) {
            if (ix[k] < 0) fail("closed branch " + std::to_string(e) + " has an absent row/column at slot " + std::to_string(k));
        }
    }
    for (int e = 0; e < nsh; e++) {
        if (shIx[static_cast<size_t>(e) * SH_INDICES + 3] >= 0 || shIx[static_cast<size_t>(e) * SH_INDICES + 4] >= 0) {
            fail("shunt " + std::to_string(e) + ": voltage-controlling shunts are not supported by this engine");
        }
    }
    Structure s;
    s.n = n;
    s.ncb = ncb;
    s.nob = nob;
    s.nsh = nsh;
    s.nElements = ncb + nob + nsh;
    s.rowMap = rowMapOf(n, ncb, cbIx, nob, obIx, nsh, shIx, nid, idRows);
    // packs with their rows mapped (shared_structure.cu:85-97)
    s.cbIx.assign(cbIx, cbIx + static_cast<size_t>(ncb) * CB_INDICES);
    s.obIx.assign(obIx, obIx + static_cast<size_t>(nob) * OB_INDICES);
    s.shIx.assign(shIx, shIx + static_cast<size_t>(nsh) * SH_INDICES);
    for (int e = 0; e < ncb; e++)
        for (int k : {0, 1, 2, 3, 10, 11}) {
            int& r = s.cbIx[static_cast<size_t>(e) * CB_INDICES + k];
            if (r >= 0) r = s.rowMap[r];
        }
    for (int e = 0; e < nob; e++)
        for (int k : {0, 1, 2, 3}) {
            int& r = s.obIx[static_cast<size_t>(e) * OB_INDICES + k];
            if (r >= 0) r = s.rowMap[r];
        }
    for (int e = 0; e < nsh; e++)
        for (int k : {0, 1, 4}) {
            int& r = s.shIx[static_cast<size_t>(e) * SH_INDICES + k];
            if (r >= 0) r = s.rowMap[r];
        }
    s.cbPar.assign(cbPar, cbPar + static_cast<size_t>(ncb) * CB_PARAMS);
    s.obPar.assign(obPar, obPar + static_cast<size_t>(nob) * OB_PARAMS);
    s.shPar.assign(shPar, shPar + static_cast<size_t>(nsh) * SH_PARAMS);

    // fixed superset pattern: role-1 entries + guaranteed diagonal, sorted and unique (shared_structure.cu:111-221)
    std::vector<int64_t> pat;
    pat.reserve(static_cast<size_t>(ncb) * 24 + static_cast<size_t>(nob) * 4 + static_cast<size_t>(nsh) * 3 + n);
    int row, col;
    for (int e = 0; e < ncb; e++)
        for (int k = 0; k < CB_OUTPUTS; k++) {
            resolveCb(CB_SCATTER[k], &s.cbIx[static_cast<size_t>(e) * CB_INDICES], row, col);
            if (CB_SCATTER[k][0] == 1 && row >= 0 && col >= 0) pat.push_back(static_cast<int64_t>(row) * n + col);
        }
    for (int e = 0; e < nob; e++)
        for (int k = 0; k < OB_OUTPUTS; k++) {
            resolveOb(OB_SCATTER[k], &s.obIx[static_cast<size_t>(e) * OB_INDICES], row, col);
            if (OB_SCATTER[k][0] == 1 && row >= 0 && col >= 0) pat.push_back(static_cast<int64_t>(row) * n + col);
        }
    for (int e = 0; e < nsh; e++)
        for (int k = 0; k < SH_OUTPUTS; k++) {
            resolveSh(SH_SCATTER[k], &s.shIx[static_cast<size_t>(e) * SH_INDICES], row, col);
            if (SH_SCATTER[k][0] == 1 && row >= 0 && col >= 0) pat.push_back(static_cast<int64_t>(row) * n + col);
        }
    for (int r = 0; r < n; r++) pat.push_back(static_cast<int64_t>(r) * n + r);
    std::sort(pat.begin(), pat.end());
    pat.erase(std::unique(pat.begin(), pat.end()), pat.end());
    s.nnz = static_cast<int>(pat.size());
    s.rowPtr.assign(n + 1, 0);
    s.colIdx.resize(s.nnz);
    for (int i = 0; i < s.nnz; i++) {
        s.colIdx[i] = static_cast<int>(pat[i] % n);
        s.rowPtr[pat[i] / n + 1]++;
    }
    for (int r = 0; r < n; r++) s.rowPtr[r + 1] += s.rowPtr[r];
    // role-folded destinations (structure_build.cuh:51-66): >= 0 J slot, -2-row F row, -1 skip
    auto dest = [&](auto table, int outputs, auto resolve, const std::vector<int>& ix, int stride, int count) {
        std::vector<int> d(static_cast<size_t>(count) * outputs, -1);
        for (int e = 0; e < count; e++)
            for (int k = 0; k < outputs; k++) {
                int r, c;
                resolve(table[k], &ix[static_cast<size_t>(e) * stride], r, c);
                if (table[k][0] == 1 && r >= 0 && c >= 0) d[static_cast<size_t>(e) * outputs + k] = csrAt(s.rowPtr, s.colIdx, r, c);
                else if (table[k][0] == 0 && r >= 0) d[static_cast<size_t>(e) * outputs + k] = -2 - r;
            }
        return d;
    };
    s.cbDest = dest(CB_SCATTER, CB_OUTPUTS, resolveCb, s.cbIx, CB_INDICES, ncb);
    s.obDest = dest(OB_SCATTER, OB_OUTPUTS, resolveOb, s.obIx, OB_INDICES, nob);
    s.shDest = dest(SH_SCATTER, SH_OUTPUTS, resolveSh, s.shIx, SH_INDICES, nsh);
    s.diagPos.resize(n);
    for (int r = 0; r < n; r++) s.diagPos[r] = csrAt(s.rowPtr, s.colIdx, r, r);

    // ---- bus-block view: every column must be one bus's angle or magnitude, and rows are paired to them ----
    s.colNode.assign(n, -1);
    std::vector<int> nodeCol;
    auto addNode = [&](int cphi, int cv) {
        if (cphi < 0 || cv < 0) return;
        int a = s.colNode[cphi], b = s.colNode[cv];
        if (a < 0 && b < 0) {
            int k = static_cast<int>(nodeCol.size() / 2);
            nodeCol.push_back(cphi);
            nodeCol.push_back(cv);
            s.colNode[cphi] = 2 * k;
            s.colNode[cv] = 2 * k + 1;
        } else if (a != (b & ~1) || a < 0 || b < 0 || (a & 1) != 0 || (b & 1) != 1) {
            fail("columns " + std::to_string(cphi) + "/" + std::to_string(cv) +
                 " are not one bus's angle/magnitude pair: unsupported variable layout");
        }
    };
    for (int e = 0; e < ncb; e++) {
        const int* ix = &s.cbIx[static_cast<size_t>(e) * CB_INDICES];
        addNode(ix[4], ix[5]);
        addNode(ix[6], ix[7]);
    }
    for (int e = 0; e < nsh; e++) {
        const int* ix = &s.shIx[static_cast<size_t>(e) * SH_INDICES];
        addNode(ix[0], ix[2]);  // the P row (mapped) is the bus's angle column
    }
    for (int e = 0; e < nob; e++) {
        const int* ix = &s.obIx[static_cast<size_t>(e) * OB_INDICES];
        if (ix[4] >= 0) addNode(ix[0], ix[4]);
        if (ix[5] >= 0) addNode(ix[2], ix[5]);
    }
    for (int c = 0; c < n; c++) {
        if (s.colNode[c] < 0) fail("column " + std::to_string(c) + " belongs to no bus: unsupported variable layout");
    }
    s.nb = static_cast<int>(nodeCol.size() / 2);
    s.nodeCol = nodeCol;
    // every row of a bus must carry that bus's own equations: row index == paired column, so the rows of node k are
    // its two columns; the J rows of branch/shunt outputs must land on their bus's rows
    for (int e = 0; e < ncb; e++) {
        const int* ix = &s.cbIx[static_cast<size_t>(e) * CB_INDICES];
        if (ix[0] != ix[4] || ix[1] != ix[5] || ix[2] != ix[6] || ix[3] != ix[7]) {
            fail("closed branch " + std::to_string(e) + ": its P/Q rows are not its buses' own rows (relocated "
                 "equations are not supported by this engine)");
        }
    }
    for (int e = 0; e < nsh; e++) {
        const int* ix = &s.shIx[static_cast<size_t>(e) * SH_INDICES];
        if (ix[1] != ix[2]) fail("shunt " + std::to_string(e) + ": its Q row is not its bus's own row");
    }
    for (int e = 0; e < nob; e++) {
        const int* ix = &s.obIx[static_cast<size_t>(e) * OB_INDICES];
        if ((ix[4] >= 0 && ix[1] != ix[4]) || (ix[5] >= 0 && ix[3] != ix[5])) {
            fail("open branch " + std::to_string(e) + ": its Q row is not its bus's own row");
        }
    }
    buildBlockPlan(s, ordering);
    return s;
}

// ---------------------------------------------------------------------------------------------------------------
// Block-LU plan
// ---------------------------------------------------------------------------------------------------------------

namespace {

// Minimum-degree order of an undirected graph (adjacency lists, no self loops): the elimination graph is kept
// explicitly; a vertex of least current degree is eliminated next, ties going to the lowest index.
std::vector<int> minimumDegree(int nb, std::vector<std::vector<int>> adj) {
    std::vector<int> deg(nb), order;
    order.reserve(nb);
    std::vector<char> gone(nb, 0);
    std::vector<int> mark(nb, -1);
    // buckets of vertices by degree, kept as sorted sets of indices via vectors rebuilt lazily
    int maxd = 0;
    for (int v = 0; v < nb; v++) {
        deg[v] = static_cast<int>(adj[v].size());
        maxd = std::max(maxd, deg[v]);
    }
    std::vector<std::vector<int>> bucket(nb + 1);
    for (int v = nb - 1; v >= 0; v--) bucket[deg[v]].push_back(v);   // popped from the back: lowest index first
    int stamp = 0;
    int mind = 0;
    for (int step = 0; step < nb; step++) {
        int v = -1;
        while (v < 0) {
            while (bucket[mind].empty()) mind++;
            // lazily discard stale entries
            int cand = bucket[mind].back();
            bucket[mind].pop_back();
            if (!gone[cand] && deg[cand] == mind) {
                // lowest index among the live entries of this bucket
                int best = cand;
                for (int u : bucket[mind]) {
                    if (!gone[u] && deg[u] == mind && u < best) best = u;
                }
                if (best != cand) bucket[mind].push_back(cand);
                v = best;
            }
        }
        gone[v] = 1;
        order.push_back(v);
        std::vector<int> nbr;
        for (int u : adj[v])
            if (!gone[u]) nbr.push_back(u);
        for (int u : nbr) {
            ++stamp;
            std::vector<int> nu;
            nu.reserve(adj[u].size() + nbr.size());
            for (int w : adj[u])
                if (!gone[w] && mark[w] != stamp) { mark[w] = stamp; nu.push_back(w); }
            for (int w : nbr)
                if (w != u && mark[w] != stamp) { mark[w] = stamp; nu.push_back(w); }
            adj[u].swap(nu);
            deg[u] = static_cast<int>(adj[u].size());
            bucket[deg[u]].push_back(u);
            if (deg[u] < mind) mind = deg[u];
        }
        std::vector<int>().swap(adj[v]);
    }
    return order;
}

// Minimum degree relaxed toward a shallow elimination tree: each step considers the live vertices whose current degree
// is at most SHALLOW_SLACK above the least one and eliminates the one of least weight * degree + height (ties: lowest
// index), where a vertex's height is one more than that of the highest eliminated vertex it has absorbed, i.e. the
// height its elimination-tree node will have.  The dependency levels of the block LU follow the tree's height (two
// per tree level in the scaled plan), and plain minimum degree, which breaks its many ties by index, grows long
// chains.  A larger weight stays closer to minimum degree (fewer block updates), a smaller one trades updates for
// height.
constexpr int SHALLOW_SLACK = 4;

std::vector<int> minimumDegreeShallow(int nb, std::vector<std::vector<int>> adj, long long weight) {
    std::vector<int> deg(nb), hgt(nb, 0), order;
    order.reserve(nb);
    std::vector<char> gone(nb, 0);
    std::vector<int> mark(nb, -1);
    // per degree: the live vertices keyed by (height, index)
    std::vector<std::set<std::pair<int, int>>> byDeg(nb + 1);
    for (int v = 0; v < nb; v++) {
        deg[v] = static_cast<int>(adj[v].size());
        byDeg[deg[v]].insert({0, v});
    }
    int stamp = 0, mind = 0;
    for (int step = 0; step < nb; step++) {
        while (byDeg[mind].empty()) mind++;
        int v = -1;
        long long best = 0;
        for (int d = mind; d <= std::min(nb, mind + SHALLOW_SLACK); d++) {
            if (byDeg[d].empty()) continue;
            const auto& e = *byDeg[d].begin();
            const long long key = (weight * d + e.first) * (nb + 1) + e.second;
            if (v < 0 || key < best) {
                best = key;
                v = e.second;
            }
        }
        byDeg[deg[v]].erase({hgt[v], v});
        gone[v] = 1;
        order.push_back(v);
        std::vector<int> nbr;
        for (int u : adj[v])
            if (!gone[u]) nbr.push_back(u);
        for (int u : nbr) {
            byDeg[deg[u]].erase({hgt[u], u});
            ++stamp;
            std::vector<int> nu;
            nu.reserve(adj[u].size() + nbr.size());
            for (int w : adj[u])
                if (!gone[w] && mark[w] != stamp) { mark[w] = stamp; nu.push_back(w); }
            for (int w : nbr)
                if (w != u && mark[w] != stamp) { mark[w] = stamp; nu.push_back(w); }
            adj[u].swap(nu);
            deg[u] = static_cast<int>(adj[u].size());
            hgt[u] = std::max(hgt[u], hgt[v] + 1);
            byDeg[deg[u]].insert({hgt[u], u});
            if (deg[u] < mind) mind = deg[u];
        }
        std::vector<int>().swap(adj[v]);
    }
    return order;
}

// Nested dissection by recursive bisection on breadth-first level structures: the middle level of a BFS from a
// pseudo-peripheral vertex is the separator; parts below a threshold are ordered by minimum degree.
void dissect(const std::vector<std::vector<int>>& adj, std::vector<int>& verts, std::vector<int>& out,
             std::vector<int>& where, int tag, int& nextTag) {
    const int m = static_cast<int>(verts.size());
    if (m <= 64) {
        // local minimum degree on the induced subgraph
        std::vector<int> local(m);
        for (int i = 0; i < m; i++) where[verts[i]] = tag, local[i] = verts[i];
        std::vector<int> idx(adj.size() > 0 ? 0 : 0);
        std::vector<std::vector<int>> sub(m);
        std::vector<int> pos;
        // map vertex -> local index through a sorted copy
        std::vector<std::pair<int, int>> key(m);
        for (int i = 0; i < m; i++) key[i] = {verts[i], i};
        std::sort(key.begin(), key.end());
        auto find = [&](int v) {
            auto it = std::lower_bound(key.begin(), key.end(), std::make_pair(v, -1));
            return (it != key.end() && it->first == v) ? it->second : -1;
        };
        for (int i = 0; i < m; i++)
            for (int w : adj[verts[i]]) {
                if (where[w] != tag) continue;
                int j = find(w);
                if (j >= 0) sub[i].push_back(j);
            }
        std::vector<int> o = minimumDegree(m, sub);
        for (int i : o) out.push_back(verts[i]);
        return;
    }
    for (int v : verts) where[v] = tag;
    // BFS twice to find a pseudo-peripheral start, then level structure
    std::vector<int> lvl;
    auto bfs = [&](int s, std::vector<int>& level, int& last) {
        level.assign(0, 0);
        std::vector<int> q{s};
        std::vector<int> dist;
        // use where[] as membership; a temporary visited tag
        int vis = nextTag++;
        std::vector<int> seen;
        where[s] = vis;
        seen.push_back(s);
        size_t h = 0;
        std::vector<int> d{0};
        while (h < q.size()) {
            int u = q[h];
            int du = d[h];
            h++;
            for (int w : adj[u]) {
                if (where[w] == tag) {
                    where[w] = vis;
                    seen.push_back(w);
                    q.push_back(w);
                    d.push_back(du + 1);
                }
            }
        }
        last = q.back();
        level = d;
        // restore membership tag
        for (int w : seen) where[w] = tag;
        return q;
    };
    int last;
    std::vector<int> q0 = bfs(verts[0], lvl, last);
    if (static_cast<int>(q0.size()) < m) {
        // disconnected subgraph: order the component reached, then the rest, separately
        std::vector<int> a(q0.begin(), q0.end());
        std::vector<char> in(0);
        std::vector<int> b;
        int t = nextTag++;
        for (int v : a) where[v] = t;
        for (int v : verts)
            if (where[v] != t) b.push_back(v);
        int ta = nextTag++, tb = nextTag++;
        dissect(adj, a, out, where, ta, nextTag);
        for (int v : b) where[v] = tb;
        dissect(adj, b, out, where, tb, nextTag);
        return;
    }
    int last2;
    std::vector<int> q = bfs(last, lvl, last2);
    q = bfs(last2, lvl, last);
    int maxLevel = lvl.back();
    if (maxLevel < 2) {
        std::vector<std::vector<int>> dummy;
        // tiny diameter: fall back to minimum degree on the whole part
        int t = nextTag++;
        for (int v : verts) where[v] = t;
        std::vector<int> copy = verts;
        where[copy[0]] = t;
        // reuse the small-part path by forcing the threshold
        std::vector<std::pair<int, int>> key(m);
        for (int i = 0; i < m; i++) key[i] = {verts[i], i};
        std::sort(key.begin(), key.end());
        std::vector<std::vector<int>> sub(m);
        for (int i = 0; i < m; i++)
            for (int w : adj[verts[i]]) {
                if (where[w] != t) continue;
                auto it = std::lower_bound(key.begin(), key.end(), std::make_pair(w, -1));
                sub[i].push_back(it->second);
            }
        std::vector<int> o = minimumDegree(m, sub);
        for (int i : o) out.push_back(verts[i]);
        return;
    }
    // separator: the level that splits the vertex count in half
    std::vector<int> cnt(maxLevel + 1, 0);
    for (int d : lvl) cnt[d]++;
    int half = m / 2, acc = 0, sepLevel = 1;
    for (int l = 0; l <= maxLevel; l++) {
        acc += cnt[l];
        if (acc >= half) { sepLevel = std::max(1, std::min(l, maxLevel - 1)); break; }
    }
    std::vector<int> A, B, S;
    for (size_t i = 0; i < q.size(); i++) {
        if (lvl[i] < sepLevel) A.push_back(q[i]);
        else if (lvl[i] == sepLevel) S.push_back(q[i]);
        else B.push_back(q[i]);
    }
    // thin the separator: a separator vertex with no neighbour in B moves to A
    std::vector<int> S2;
    int tB = nextTag++;
    for (int v : B) where[v] = tB;
    for (int v : S) {
        bool touchesB = false;
        for (int w : adj[v]) touchesB |= (where[w] == tB);
        if (touchesB) S2.push_back(v);
        else A.push_back(v);
    }
    int tA = nextTag++;
    for (int v : A) where[v] = tA;
    dissect(adj, A, out, where, tA, nextTag);
    for (int v : B) where[v] = tB;
    dissect(adj, B, out, where, tB, nextTag);
    for (int v : S2) out.push_back(v);
    for (int v : S2) where[v] = -1;
}

std::vector<int> nestedDissection(int nb, const std::vector<std::vector<int>>& adj) {
    std::vector<int> verts(nb), out, where(nb, 0);
    std::iota(verts.begin(), verts.end(), 0);
    int nextTag = 1;
    out.reserve(nb);
    dissect(adj, verts, out, where, 0, nextTag);
    return out;
}

void buildPlan(Structure& s, int ordering, long long shallowWeight);

// The shallow-tree order is built for several degree weights and the plan of least cost is kept: 1.5 per dependency
// level (factorization, forward and backward solve) plus 1 per thousand block updates per lane.  On the 9,241-bus
// grid's 500-outage FP64 step (weight 8: 10.90 ms, 4: 11.15 ms, 2 with a slack of 6: 11.66 ms, 2: 11.76 ms) this
// cost ranks the four plans as the measured step times do.
constexpr long long SHALLOW_WEIGHTS[] = {2, 4, 6, 8};

double planCost(const BlockPlan& p) {
    const size_t levels = (p.levelPtr.size() - 1) + (p.fwdLevelPtr.size() - 1) + (p.bwdLevelPtr.size() - 1);
    return 1.5 * static_cast<double>(levels) + static_cast<double>(p.blockOps) / 1000.0;
}

}  // namespace

void buildBlockPlan(Structure& s, int ordering) {
    if ((ordering & ~(PLAN_DEFERRED_L | PLAN_DENSE_FRONT)) != ORDER_MIN_DEGREE_SHALLOW) {
        buildPlan(s, ordering, 0);
        return;
    }
    BlockPlan best;
    double bestCost = 0.0;
    bool have = false;
    for (long long w : SHALLOW_WEIGHTS) {
        s.plan = BlockPlan{};
        buildPlan(s, ordering, w);
        const double cost = planCost(s.plan);
        if (!have || cost < bestCost) {
            best = std::move(s.plan);
            bestCost = cost;
            have = true;
        }
    }
    s.plan = std::move(best);
}

namespace {

void buildPlan(Structure& s, int ordering, long long shallowWeight) {
    BlockPlan& p = s.plan;
    const int nb = s.nb;
    p.nb = nb;
    // node graph from the CSR pattern (structurally symmetric for these families; symmetrised anyway)
    std::vector<std::vector<int>> adj(nb);
    for (int r = 0; r < s.n; r++) {
        int a = s.colNode[r] >> 1;
        for (int k = s.rowPtr[r]; k < s.rowPtr[r + 1]; k++) {
            int b = s.colNode[s.colIdx[k]] >> 1;
            if (a != b) {
                adj[a].push_back(b);
                adj[b].push_back(a);
            }
        }
    }
    for (auto& l : adj) {
        std::sort(l.begin(), l.end());
        l.erase(std::unique(l.begin(), l.end()), l.end());
    }
    // A block pattern by node row (diagonal included)
    p.aPtr.assign(nb + 1, 0);
    p.aCol.clear();
    p.aDiag.assign(nb, -1);
    for (int a = 0; a < nb; a++) {
        std::vector<int> cols = adj[a];
        cols.push_back(a);
        std::sort(cols.begin(), cols.end());
        for (int c : cols) {
            if (c == a) p.aDiag[a] = static_cast<int>(p.aCol.size());
            p.aCol.push_back(c);
        }
        p.aPtr[a + 1] = static_cast<int>(p.aCol.size());
    }
    p.deferredL = (ordering & PLAN_DEFERRED_L) != 0;
    const bool denseFront = (ordering & PLAN_DENSE_FRONT) != 0;
    if (p.deferredL && denseFront) fail("the deferred-L and dense-front plans cannot be combined");
    ordering &= ~(PLAN_DEFERRED_L | PLAN_DENSE_FRONT);
    // ordering
    if (ordering == ORDER_NATURAL) {
        p.perm.resize(nb);
        std::iota(p.perm.begin(), p.perm.end(), 0);
    } else if (ordering == ORDER_NESTED_DISSECTION) {
        p.perm = nestedDissection(nb, adj);
    } else if (ordering == ORDER_MIN_DEGREE_SHALLOW) {
        p.perm = minimumDegreeShallow(nb, adj, shallowWeight);
    } else {
        p.perm = minimumDegree(nb, adj);
    }
    if (static_cast<int>(p.perm.size()) != nb) fail("ordering is not a permutation");
    p.iperm.assign(nb, -1);
    for (int k = 0; k < nb; k++) p.iperm[p.perm[k]] = k;
    // symbolic elimination in the chosen order: struct(k) = positions > k adjacent to k in the filled graph
    std::vector<std::vector<int>> st(nb);
    {
        std::vector<std::vector<int>> g(nb);
        for (int a = 0; a < nb; a++)
            for (int b : adj[a]) g[p.iperm[a]].push_back(p.iperm[b]);
        // elimination via the elimination tree: struct(k) = (adj(k) > k) U (struct(c) \ {k}) over children c
        std::vector<int> parent(nb, -1);
        std::vector<int> mark(nb, -1);
        std::vector<std::vector<int>> children(nb);
        for (int k = 0; k < nb; k++) {
            std::vector<int> sk;
            mark[k] = k;
            for (int j : g[k])
                if (j > k && mark[j] != k) { mark[j] = k; sk.push_back(j); }
            for (int c : children[k])
                for (int j : st[c])
                    if (j > k && mark[j] != k) { mark[j] = k; sk.push_back(j); }
            std::sort(sk.begin(), sk.end());
            st[k] = sk;
            if (!sk.empty()) {
                parent[k] = sk[0];
                children[sk[0]].push_back(k);
            }
        }
    }
    // U rows and L columns
    p.uPtr.assign(nb + 1, 0);
    p.lPtr.assign(nb + 1, 0);
    p.uCol.clear();
    p.lRow.clear();
    for (int k = 0; k < nb; k++) {
        p.uCol.push_back(k);
        for (int j : st[k]) p.uCol.push_back(j);
        p.uPtr[k + 1] = static_cast<int>(p.uCol.size());
        for (int i : st[k]) p.lRow.push_back(i);
        p.lPtr[k + 1] = static_cast<int>(p.lRow.size());
    }
    p.nU = static_cast<int>(p.uCol.size());
    p.nL = static_cast<int>(p.lRow.size());
    const int nLu = p.nU + p.nL;
    auto uBlock = [&](int k, int j) {  // block id of U(k, j), j >= k
        auto b = p.uCol.begin() + p.uPtr[k], e = p.uCol.begin() + p.uPtr[k + 1];
        auto it = std::lower_bound(b + 1, e, j);
        if (j == k) return p.uPtr[k];
        if (it == e || *it != j) fail("U block lookup miss");
        return static_cast<int>(it - p.uCol.begin());
    };
    auto lBlock = [&](int i, int k) {  // block id of L(i, k), i > k
        auto b = p.lRow.begin() + p.lPtr[k], e = p.lRow.begin() + p.lPtr[k + 1];
        auto it = std::lower_bound(b, e, i);
        if (it == e || *it != i) fail("L block lookup miss");
        return p.nU + static_cast<int>(it - p.lRow.begin());
    };
    // A -> LU block map
    p.aToLu.assign(p.aCol.size(), -1);
    p.luToA.assign(nLu, -1);
    for (int a = 0; a < nb; a++) {
        for (int t = p.aPtr[a]; t < p.aPtr[a + 1]; t++) {
            int i = p.iperm[a], j = p.iperm[p.aCol[t]];
            int id = i <= j ? uBlock(i, j) : lBlock(i, j);
            p.aToLu[t] = id;
            p.luToA[id] = t;
        }
    }
    // update pairs: pivot m contributes L(a,m) * U(m,b) to entry (a,b) for every a, b in struct(m)
    std::vector<int> cnt(nLu, 0);
    int64_t ops = 0;
    for (int m = 0; m < nb; m++) {
        const auto& sm = st[m];
        for (int a : sm)
            for (int b : sm) {
                int id = a <= b ? uBlock(a, b) : lBlock(a, b);
                cnt[id]++;
                ops++;
            }
    }
    p.blockOps = ops;
    p.opPtr.assign(nLu + 1, 0);
    for (int id = 0; id < nLu; id++) p.opPtr[id + 1] = p.opPtr[id] + cnt[id];
    p.opL.assign(ops, 0);
    p.opU.assign(ops, 0);
    p.opD.assign(ops, 0);
    std::vector<int> fillPos(p.opPtr.begin(), p.opPtr.end() - 1);
    for (int m = 0; m < nb; m++) {
        const auto& sm = st[m];
        for (int a : sm) {
            int la = lBlock(a, m);
            for (int b : sm) {
                int id = a <= b ? uBlock(a, b) : lBlock(a, b);
                int q = fillPos[id]++;
                p.opL[q] = la;
                p.opU[q] = uBlock(m, b);
                p.opD[q] = p.deferredL ? p.uPtr[m] : -1;
            }
        }
    }
    // dense front: the trailing F positions; an absent block would be a structural zero (an exact zero through the
    // dense elimination)
    p.opOuterEnd.assign(nLu, 0);
    for (int id = 0; id < nLu; id++) p.opOuterEnd[id] = p.opPtr[id + 1];
    p.frontStart = nb;
    p.frontF = 0;
    p.frontBlocks.clear();
    std::vector<int> uRow(p.nU);
    for (int k = 0; k < nb; k++)
        for (int t = p.uPtr[k]; t < p.uPtr[k + 1]; t++) uRow[t] = k;
    auto findBlock = [&](int a, int b) {   // LU block of positions (a, b), or -1 when structurally zero
        if (a <= b) {
            if (a == b) return p.uPtr[a];
            auto lo = p.uCol.begin() + p.uPtr[a] + 1, hi = p.uCol.begin() + p.uPtr[a + 1];
            auto it = std::lower_bound(lo, hi, b);
            return it != hi && *it == b ? static_cast<int>(it - p.uCol.begin()) : -1;
        }
        auto lo = p.lRow.begin() + p.lPtr[b], hi = p.lRow.begin() + p.lPtr[b + 1];
        auto it = std::lower_bound(lo, hi, a);
        return it != hi && *it == a ? p.nU + static_cast<int>(it - p.lRow.begin()) : -1;
    };
    // levels of the plan with the front starting at position k0 (k0 = nb: no front); returns the level count
    std::vector<int> lvl(nLu, 0);
    auto levelsWith = [&](int k0, std::vector<int>& level) {
        int mx = -1;
        auto one = [&](int id, int lv, bool front) {
            const int end = front ? p.opPtr[id] : p.opPtr[id + 1];
            int q = p.opPtr[id];
            for (; q < p.opPtr[id + 1]; q++) {
                if (front && uRow[p.opU[q]] >= k0) break;   // a front block stops at the first pivot of the front
                int dep = std::max(level[p.opL[q]], level[p.opU[q]]);
                if (p.opD[q] >= 0) dep = std::max(dep, level[p.opD[q]]);
                lv = std::max(lv, dep + 1);
            }
            (void)end;
            level[id] = lv;
            mx = std::max(mx, lv);
        };
        for (int k = 0; k < nb; k++) {
            for (int t = p.uPtr[k]; t < p.uPtr[k + 1]; t++) one(t, 0, k >= k0 && p.uCol[t] >= k0);
            for (int t = p.lPtr[k]; t < p.lPtr[k + 1]; t++) {
                const bool front = k >= k0 && p.lRow[t] >= k0;
                one(p.nU + t, front || p.deferredL ? 0 : level[p.uPtr[k]] + 1, front);
            }
        }
        return mx + 1;
    };
    if (denseFront) {
        // the largest trailing block (<= MAX_FRONT pivots) with every block present: a front padded with structural
        // zeros measured slower (more dense work, fewer resident CTAs) than the levels it removed
        int bestF = 0;
        for (int f = std::min(MAX_FRONT, nb); f >= 4 && bestF == 0; f--) {
            bool dense = true;
            for (int k = nb - f; k < nb && dense; k++) {
                dense = p.uPtr[k + 1] - p.uPtr[k] == nb - k && p.lPtr[k + 1] - p.lPtr[k] == nb - 1 - k;
            }
            if (dense) bestF = f;
        }
        if (bestF > 0) {
            const int F = bestF;
            p.frontF = F;
            p.frontStart = nb - F;
            p.frontBlocks.assign(static_cast<size_t>(F) * F, -1);
            for (int i = 0; i < F; i++)
                for (int j = 0; j < F; j++)
                    p.frontBlocks[static_cast<size_t>(i) * F + j] = findBlock(p.frontStart + i, p.frontStart + j);
            // a front block's task keeps the prefix of its updates whose pivot precedes the front (pivots ascend)
            for (int id : p.frontBlocks) {
                if (id < 0) continue;
                int q = p.opPtr[id];
                while (q < p.opPtr[id + 1] && uRow[p.opU[q]] < p.frontStart) q++;
                p.opOuterEnd[id] = q;
            }
        }
    }
    // levels: a task runs one level after every block its updates read (L, U and, deferred-L, the pivot's inverse); a
    // scaled L block waits for its column's pivot; a front block's partial sum waits for nothing in the front
    p.level.assign(nLu, 0);
    const int maxLevel = levelsWith(p.frontStart, p.level) - 1;
    p.levelPtr.assign(maxLevel + 2, 0);
    for (int id = 0; id < nLu; id++) p.levelPtr[p.level[id] + 1]++;
    for (int l = 0; l <= maxLevel; l++) p.levelPtr[l + 1] += p.levelPtr[l];
    p.levelTask.assign(nLu, 0);
    {
        std::vector<int> w(p.levelPtr.begin(), p.levelPtr.end() - 1);
        for (int id = 0; id < nLu; id++) p.levelTask[w[p.level[id]]++] = id;
    }
    // solve levels: forward f(i) = 1 + max f(k) over k with i in struct(k); backward b(i) = 1 + max b(j), j in struct(i).
    // With a dense front, a front position's forward level task only applies the columns before the front (the dense
    // front solve does the rest), and the front positions are solved backward by the dense front before any level.
    const int k0 = p.frontStart;
    std::vector<int> fl(nb, 0), bl(nb, 0);
    for (int k = 0; k < nb; k++) {
        if (k >= k0) continue;
        for (int i : st[k]) fl[i] = std::max(fl[i], fl[k] + 1);
    }
    for (int i = nb - 1; i >= 0; i--) {
        if (i >= k0) {
            bl[i] = -1;
            continue;
        }
        for (int j : st[i])
            if (j < k0) bl[i] = std::max(bl[i], bl[j] + 1);
    }
    auto group = [&](const std::vector<int>& lv, std::vector<int>& ptr, std::vector<int>& pos) {
        int mx = 0, cnt = 0;
        for (int v : lv) {
            mx = std::max(mx, v);
            cnt += v >= 0;
        }
        ptr.assign(mx + 2, 0);
        for (int v : lv)
            if (v >= 0) ptr[v + 1]++;
        for (int l = 0; l <= mx; l++) ptr[l + 1] += ptr[l];
        pos.assign(cnt, 0);
        std::vector<int> w(ptr.begin(), ptr.end() - 1);
        for (int i = 0; i < static_cast<int>(lv.size()); i++)
            if (lv[i] >= 0) pos[w[lv[i]]++] = i;
    };
    group(fl, p.fwdLevelPtr, p.fwdLevelPos);
    group(bl, p.bwdLevelPtr, p.bwdLevelPos);
}

}  // namespace

int64_t checkBlockPlan(const BlockPlan& plan, int plantedFault, std::string& first) {
    BlockPlan p = plan;   // a planted fault changes this copy only
    const int nb = p.nb, nLu = p.nU + p.nL;
    // where every LU block sits: U block t is (uRow[t], uCol[t]); L block nU + t is (lRow[t], lCol[t])
    std::vector<int> rowOf(nLu), colOf(nLu);
    for (int k = 0; k < nb; k++) {
        for (int t = p.uPtr[k]; t < p.uPtr[k + 1]; t++) rowOf[t] = k, colOf[t] = p.uCol[t];
        for (int t = p.lPtr[k]; t < p.lPtr[k + 1]; t++) rowOf[p.nU + t] = p.lRow[t], colOf[p.nU + t] = k;
    }
    if (plantedFault == 1) {
        // a task moved one level up, beside a block it reads: the deepest task with an update
        int victim = -1;
        for (int id = 0; id < nLu; id++)
            if (p.opPtr[id + 1] > p.opPtr[id] && (victim < 0 || p.level[id] > p.level[victim])) victim = id;
        if (victim >= 0) {
            p.level[victim]--;
            p.levelPtr.assign(p.levelPtr.size(), 0);
            for (int id = 0; id < nLu; id++) p.levelPtr[p.level[id] + 1]++;
            for (size_t l = 0; l + 1 < p.levelPtr.size(); l++) p.levelPtr[l + 1] += p.levelPtr[l];
            std::vector<int> w(p.levelPtr.begin(), p.levelPtr.end() - 1);
            for (int id = 0; id < nLu; id++) p.levelTask[w[p.level[id]]++] = id;
        }
    } else if (plantedFault == 2) {
        // one update dropped from the longest update list
        int victim = 0;
        for (int id = 1; id < nLu; id++)
            if (p.opPtr[id + 1] - p.opPtr[id] > p.opPtr[victim + 1] - p.opPtr[victim]) victim = id;
        const int q = p.opPtr[victim];
        if (p.opPtr[victim + 1] > q) {
            p.opL.erase(p.opL.begin() + q);
            p.opU.erase(p.opU.begin() + q);
            p.opD.erase(p.opD.begin() + q);
            for (int id = victim + 1; id <= nLu; id++) p.opPtr[id]--;
            for (int id = victim + 1; id < nLu; id++) p.opOuterEnd[id]--;
            if (p.opOuterEnd[victim] > q) p.opOuterEnd[victim]--;
        }
    } else if (plantedFault == 3) {
        // a forward-solve position of the last level swapped with one of the first
        if (!p.fwdLevelPos.empty()) std::swap(p.fwdLevelPos[0], p.fwdLevelPos.back());
    }
    int64_t bad = 0;
    auto fail = [&](const std::string& what) {
        if (bad++ == 0) first = what;
    };
    auto blockAt = [&](int a, int b) -> int {
        if (a <= b) {
            if (a == b) return p.uPtr[a];
            auto lo = p.uCol.begin() + p.uPtr[a] + 1, hi = p.uCol.begin() + p.uPtr[a + 1];
            auto it = std::lower_bound(lo, hi, b);
            return it != hi && *it == b ? static_cast<int>(it - p.uCol.begin()) : -1;
        }
        auto lo = p.lRow.begin() + p.lPtr[b], hi = p.lRow.begin() + p.lPtr[b + 1];
        auto it = std::lower_bound(lo, hi, a);
        return it != hi && *it == a ? p.nU + static_cast<int>(it - p.lRow.begin()) : -1;
    };
    auto where = [&](int id) {
        return " (block " + std::to_string(rowOf[id]) + "," + std::to_string(colOf[id]) + ")";
    };

    // (1) closure of the symbolic factorization and the update lists: L(a, m) by rows, U(m, b) by columns, m ascending
    std::vector<std::vector<int>> lByRow(nb), uByCol(nb);
    for (int m = 0; m < nb; m++) {
        for (int t = p.lPtr[m]; t < p.lPtr[m + 1]; t++) lByRow[p.lRow[t]].push_back(p.nU + t);
        for (int t = p.uPtr[m] + 1; t < p.uPtr[m + 1]; t++) uByCol[p.uCol[t]].push_back(t);
    }
    for (int m = 0; m < nb; m++)
        for (int t = p.lPtr[m]; t < p.lPtr[m + 1]; t++)
            for (int u = p.uPtr[m] + 1; u < p.uPtr[m + 1]; u++)
                if (blockAt(p.lRow[t], p.uCol[u]) < 0)
                    fail("fill not closed: the update L(" + std::to_string(p.lRow[t]) + "," + std::to_string(m) +
                         ") U(" + std::to_string(m) + "," + std::to_string(p.uCol[u]) + ") has no block");
    for (int id = 0; id < nLu; id++) {
        const int a = rowOf[id], b = colOf[id], top = std::min(a, b);
        const std::vector<int>& L = lByRow[a];
        const std::vector<int>& U = uByCol[b];
        int q = p.opPtr[id];
        size_t i = 0, j = 0;
        bool ok = true;
        while (i < L.size() && j < U.size()) {
            const int mi = colOf[L[i]], mj = rowOf[U[j]];
            if (mi >= top || mj >= top) break;
            if (mi < mj) {
                i++;
                continue;
            }
            if (mj < mi) {
                j++;
                continue;
            }
            const int d = p.deferredL ? p.uPtr[mi] : -1;
            if (q >= p.opPtr[id + 1] || p.opL[q] != L[i] || p.opU[q] != U[j] || p.opD[q] != d) ok = false;
            q++, i++, j++;
        }
        if (!ok || q != p.opPtr[id + 1]) fail("update list differs from the symbolic factorization" + where(id));
    }

    // (2) factorization levels: every block once; every block a task reads lies on a strictly earlier level
    const int nLevels = static_cast<int>(p.levelPtr.size()) - 1;
    std::vector<int> lev(nLu, -1);
    for (int l = 0; l < nLevels; l++)
        for (int k = p.levelPtr[l]; k < p.levelPtr[l + 1]; k++) {
            const int id = p.levelTask[k];
            if (id < 0 || id >= nLu || lev[id] >= 0) fail("a block is not exactly one level task");
            else lev[id] = l;
        }
    for (int id = 0; id < nLu; id++)
        if (lev[id] < 0) fail("a block has no level task" + where(id));
    const int fs = p.frontStart;
    auto inFront = [&](int id) { return rowOf[id] >= fs && colOf[id] >= fs; };
    for (int id = 0; id < nLu; id++) {
        if (lev[id] < 0) continue;
        const int lv = lev[id];
        for (int q = p.opPtr[id]; q < p.opOuterEnd[id]; q++) {
            const bool early = lev[p.opL[q]] < lv && lev[p.opU[q]] < lv && (p.opD[q] < 0 || lev[p.opD[q]] < lv);
            if (!early) fail("a task reads a block of its own or a later level" + where(id));
        }
        if (inFront(id)) {
            // the level task applies exactly the updates whose pivot precedes the front; the dense front the rest
            const int e = p.opOuterEnd[id];
            for (int q = p.opPtr[id]; q < p.opPtr[id + 1]; q++)
                if ((rowOf[p.opU[q]] < fs) != (q < e))
                    fail("a front block's level task splits its updates wrongly" + where(id));
        } else if (p.opOuterEnd[id] != p.opPtr[id + 1]) {
            fail("a block outside the front leaves updates to the front" + where(id));
        }
        if (rowOf[id] > colOf[id] && !p.deferredL && !inFront(id) && !(lev[p.uPtr[colOf[id]]] < lv))
            fail("an L block is scaled before its pivot is inverted" + where(id));
    }
    if (p.frontF > 0) {
        const int F = p.frontF;
        for (int i = 0; i < F; i++)
            for (int j = 0; j < F; j++) {
                const int id = p.frontBlocks[static_cast<size_t>(i) * F + j];
                if (id < 0 || id != blockAt(fs + i, fs + j)) fail("the dense front's block table is incomplete");
            }
    }

    // (3) solve levels: the forward sweep reads y(k) for L(i, k), k before the front; the backward sweep x(j) for
    // U(i, j), the front's positions solved first by the dense front
    auto levelsOf = [&](const std::vector<int>& ptr, const std::vector<int>& pos, std::vector<int>& lv,
                        const char* what) {
        for (size_t l = 0; l + 1 < ptr.size(); l++)
            for (int k = ptr[l]; k < ptr[l + 1]; k++) {
                const int i = pos[k];
                if (i < 0 || i >= nb || lv[i] != -2) fail(std::string(what) + ": a position is not exactly once");
                else lv[i] = static_cast<int>(l);
            }
    };
    std::vector<int> fl(nb, -2), bl(nb, -2);
    levelsOf(p.fwdLevelPtr, p.fwdLevelPos, fl, "forward levels");
    levelsOf(p.bwdLevelPtr, p.bwdLevelPos, bl, "backward levels");
    for (int i = 0; i < nb; i++) {
        if (fl[i] < 0) fail("forward levels: position " + std::to_string(i) + " missing");
        if (i >= fs) {
            if (bl[i] != -2) fail("backward levels: a front position on a level");
            bl[i] = -1;
        } else if (bl[i] < 0) {
            fail("backward levels: position " + std::to_string(i) + " missing");
        }
    }
    for (int k = 0; k < std::min(fs, nb); k++)
        for (int t = p.lPtr[k]; t < p.lPtr[k + 1]; t++)
            if (!(fl[k] < fl[p.lRow[t]])) fail("forward sweep: a position reads an entry of its own or a later level");
    for (int i = 0; i < std::min(fs, nb); i++)
        for (int t = p.uPtr[i] + 1; t < p.uPtr[i + 1]; t++)
            if (!(bl[p.uCol[t]] < bl[i])) fail("backward sweep: a position reads an entry of its own or a later level");
    return bad;
}

}  // namespace olfb200
