// ORACLE -- test infrastructure only.  Glue that exposes, through a C ABI, the reference's OWN host code for the
// structure (row map, pattern entries, role-folded destinations) and its OWN generated formula headers, compiled
// from the reference's sources where they lie (see Makefile).  Used only by the tests, to pin the oracle and the
// engine against the reference bit for bit.  The pattern assembly below restates shared_structure.cu:73-221 for the
// closed-branch, open-branch, shunt and identity-row families (the other families are empty in these inputs).
#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "structure/structure_build.cuh"

#define CLOSED_BRANCH_FN
#define OPEN_BRANCH_FN
#define SHUNT_FN
#include "equations/generated/closed_branch.cuh"
#include "equations/generated/open_branch.cuh"
#include "equations/generated/shunt.cuh"

using namespace olfgpu;

extern "C" int olfref_structure(int n, int ncb, const int* cbIdx, int nob, const int* obIdx, int nsh, const int* shIdx,
                                int nid, const int* idRows, int* rowMapOut, int* nnzOut, int* rowPtrOut, int* colIdxOut,
                                int colCap, int* cbDest, int* obDest, int* shDest, int* diagPos, char* err) {
    try {
        std::vector<int> rowMap = buildRowMap(n, ncb, cbIdx, nob, obIdx, nsh, shIdx, 0, nullptr, 0, nullptr, 0, nullptr,
                                              nid, idRows);
        auto mapRows = [&](const int* idx, int count, int stride, std::initializer_list<int> slots) {
            std::vector<int> out(idx, idx + static_cast<size_t>(count) * stride);
            for (int e = 0; e < count; e++) {
                for (int s : slots) {
                    int& r = out[static_cast<size_t>(e) * stride + s];
                    if (r >= 0) r = rowMap[r];
                }
            }
            return out;
        };
        std::vector<int> cb = mapRows(cbIdx, ncb, 12, {0, 1, 2, 3, 10, 11});
        std::vector<int> ob = mapRows(obIdx, nob, 6, {0, 1, 2, 3});
        std::vector<int> sh = mapRows(shIdx, nsh, 5, {0, 1, 4});
        std::vector<std::pair<int, int>> pat;
        collectPattern(ncb, cb.data(), 12, CLOSED_BRANCH_SCATTER, CLOSED_BRANCH_OUTPUT_COUNT, resolveClosedBranch, pat);
        collectPattern(nob, ob.data(), 6, OPEN_BRANCH_SCATTER, OPEN_BRANCH_OUTPUT_COUNT, resolveOpenBranch, pat);
        collectPattern(nsh, sh.data(), 5, SHUNT_SCATTER, SHUNT_OUTPUT_COUNT, resolveShunt, pat);
        for (int r = 0; r < n; r++) pat.emplace_back(r, r);
        std::sort(pat.begin(), pat.end());
        pat.erase(std::unique(pat.begin(), pat.end()), pat.end());
        const int nnz = static_cast<int>(pat.size());
        *nnzOut = nnz;
        std::memcpy(rowMapOut, rowMap.data(), sizeof(int) * n);
        if (nnz > colCap) throw std::runtime_error("colIdx capacity too small");
        std::vector<int> rowPtr(n + 1, 0), colIdx(nnz);
        for (int i = 0; i < nnz; i++) {
            colIdx[i] = pat[i].second;
            rowPtr[pat[i].first + 1]++;
        }
        for (int r = 0; r < n; r++) rowPtr[r + 1] += rowPtr[r];
        CsrPattern pos{rowPtr.data(), colIdx.data()};
        std::vector<int> d1 = buildDest(ncb, cb.data(), 12, CLOSED_BRANCH_SCATTER, CLOSED_BRANCH_OUTPUT_COUNT,
                                        resolveClosedBranch, pos);
        std::vector<int> d2 = buildDest(nob, ob.data(), 6, OPEN_BRANCH_SCATTER, OPEN_BRANCH_OUTPUT_COUNT,
                                        resolveOpenBranch, pos);
        std::vector<int> d3 = buildDest(nsh, sh.data(), 5, SHUNT_SCATTER, SHUNT_OUTPUT_COUNT, resolveShunt, pos);
        std::memcpy(rowPtrOut, rowPtr.data(), sizeof(int) * (n + 1));
        std::memcpy(colIdxOut, colIdx.data(), sizeof(int) * nnz);
        std::memcpy(cbDest, d1.data(), sizeof(int) * d1.size());
        std::memcpy(obDest, d2.data(), sizeof(int) * d2.size());
        std::memcpy(shDest, d3.data(), sizeof(int) * d3.size());
        for (int r = 0; r < n; r++) diagPos[r] = pos.at(r, r);
        return 0;
    } catch (const std::exception& e) {
        std::strncpy(err, e.what(), 255);
        err[255] = 0;
        return -1;
    }
}

extern "C" void olfref_closed_branch(const double* p, double v1, double r1, double v2, double a1, double ph1,
                                     double ph2, double* o) {
    powsybl::openloadflow::updateClosedBranch(p[0], p[1], p[2], p[3], p[4], v1, r1, v2, p[5], a1, ph1, ph2, 0,
            o + 0, o + 1, o + 2, o + 3, o + 4, o + 5, o + 6, o + 7, o + 8, o + 9, o + 10, o + 11, o + 12, o + 13,
            o + 14, o + 15, o + 16, o + 17, o + 18, o + 19, o + 20, o + 21, o + 22, o + 23, o + 24, o + 25, o + 26,
            o + 27);
}

extern "C" void olfref_open_branch(const double* p, double v1, double v2, double* o) {
    powsybl::openloadflow::updateOpenBranch(p[0], p[1], p[2], p[3], p[4], p[5], v1, p[6], v2, 0, o + 0, o + 1, o + 2,
                                            o + 3, o + 4, o + 5, o + 6, o + 7);
}

extern "C" void olfref_shunt(const double* p, double v, double* o) {
    powsybl::openloadflow::updateShunt(v, p[0], p[1], 0, o + 0, o + 1, o + 2, o + 3, o + 4);
}
