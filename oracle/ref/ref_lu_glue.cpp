// ORACLE -- test infrastructure only.  Exposes, through a C ABI, the reference's OWN host LU, compiled from its
// sources where they lie (see Makefile): the fast engine's symbolic plan (native/cuda/lu/scalar_lu_plan.cu,
// buildScalarLuPlan) on the reference's minimum-degree order (native/cuda/lu/minimum_degree.cu, minimumDegreeOrder),
// and the one-lane host ports of that engine's numeric factorization and solve (native/host/lu_transposed_check.cpp:
// 74-145, factorFast / solveFast: left-looking, static pivots, the reference's pivot clamp and multiplier limit).
// The reference's check program is compiled here as part of this translation unit with its main() renamed, so its
// file-local functions can be called.  Used only by the tests and the fixture script, to pin the oracle's linear
// solve and Newton trajectory against the reference's own LU.
#define main olfref_lu_host_check_main
#include "lu_transposed_check.cpp"
#undef main

#include <cstring>
#include <exception>

namespace {

struct RefLu {
    int n = 0;
    ScalarLuPlan plan;
    ScalarLuColumns columns;   // the factors' columns the transposed solve reads (buildScalarLuColumns)
};

void setError(char* err, const char* what) {
    if (err) {
        std::strncpy(err, what, 255);
        err[255] = 0;
    }
}

}  // namespace

// The reference's fast-engine plan of the CSR pattern (rowPtr[n + 1], colIdx[nnz]) on its minimum-degree order,
// the same order for rows and columns (the structure pairs every equation row with its diagonal variable).  Returns
// an opaque handle, or null with the reason in err (256 bytes).
extern "C" void* olfref_lu_plan(int n, const int* rowPtr, const int* colIdx, int* nnzLuOut, int* levelsOut, char* err) {
    try {
        auto* h = new RefLu();
        h->n = n;
        const std::vector<int> md = minimumDegreeOrder(n, rowPtr, colIdx);
        h->plan = buildScalarLuPlan(n, rowPtr, colIdx, md.data(), md.data());
        h->columns = buildScalarLuColumns(h->plan);
        if (nnzLuOut) *nnzLuOut = h->plan.nnzLu;
        if (levelsOut) *levelsOut = h->plan.factorSteps();
        return h;
    } catch (const std::exception& e) {
        setError(err, e.what());
        return nullptr;
    }
}

extern "C" void olfref_lu_free(void* h) { delete static_cast<RefLu*>(h); }

// x with A x = b, A given by its CSR values in the planned pattern's order: the reference's one-lane factorization
// then its level-ordered forward and backward solves.  Returns the factorization's trouble count (clamped pivots and
// multipliers beyond the limit; 0 when the engine trusts the lane), or -1 on an error.
extern "C" int olfref_lu_solve(void* handle, const double* vals, const double* b, double* x) {
    try {
        const RefLu& h = *static_cast<const RefLu*>(handle);
        const std::vector<double> a(vals, vals + h.plan.nnzA);
        int trouble = 0;
        const std::vector<double> lu = factorFast(h.plan, a, trouble);
        const std::vector<double> rhs(b, b + h.n);
        const std::vector<double> z = solveFast(h.plan, lu, rhs);
        std::memcpy(x, z.data(), sizeof(double) * static_cast<size_t>(h.n));
        return trouble;
    } catch (const std::exception&) {
        return -1;
    }
}

// x with A^T x = b on the same one-lane factors: the reference's transposed solve (solveFastTransposed,
// native/host/lu_transposed_check.cpp:145-173, over the row bodies of lu/transposed_solve.cuh).  Returns the
// factorization's trouble count, or -1 on an error.
extern "C" int olfref_lu_solve_transposed(void* handle, const double* vals, const double* b, double* x) {
    try {
        const RefLu& h = *static_cast<const RefLu*>(handle);
        const std::vector<double> a(vals, vals + h.plan.nnzA);
        int trouble = 0;
        const std::vector<double> lu = factorFast(h.plan, a, trouble);
        const std::vector<double> rhs(b, b + h.n);
        const std::vector<double> z = solveFastTransposed(h.plan, h.columns, lu, rhs);
        std::memcpy(x, z.data(), sizeof(double) * static_cast<size_t>(h.n));
        return trouble;
    } catch (const std::exception&) {
        return -1;
    }
}
