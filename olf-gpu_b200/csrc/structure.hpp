// Host-side structure of one network: the reference-compatible equation structure (row map, fixed superset CSR
// pattern, role-folded scatter map, diagonal slots) and the engine's bus-block view of it with the block-LU plan.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace olfb200 {

constexpr int CB_OUTPUTS = 28;   // closed_branch_scatter.h: CLOSED_BRANCH_OUTPUT_COUNT
constexpr int OB_OUTPUTS = 8;    // open_branch_scatter.h
constexpr int SH_OUTPUTS = 5;    // shunt_scatter.h
constexpr int CB_PARAMS = 8, CB_INDICES = 12;
constexpr int OB_PARAMS = 7, OB_INDICES = 6;
constexpr int SH_PARAMS = 2, SH_INDICES = 5;

// Block-LU plan on the bus graph (2x2 blocks).  Positions are elimination positions 0..nb-1.
//   U rows:  for pivot k, blocks (k, j) j in {k} U struct(k), diagonal first, then ascending j.
//   L cols:  for pivot k, blocks (i, k) i in struct(k), ascending i.
// Every LU block has an id in [0, nLuBlocks): U blocks first (uPtr), then L blocks (lPtr offset by nU).
struct BlockPlan {
    int nb = 0;
    std::vector<int> perm;        // elimination position -> node
    std::vector<int> iperm;       // node -> elimination position
    std::vector<int> uPtr, uCol;  // U rows (CSR over positions), uCol[pos] = column position j
    std::vector<int> lPtr, lRow;  // L cols (CSC over positions), lRow[pos] = row position i
    int nU = 0, nL = 0;
    // A blocks (the Jacobian's block pattern in node order, block-CSR by node row, diagonal included) and where
    // each A block sits in the LU storage (-1 never happens: the fill is a superset of A).
    std::vector<int> aPtr, aCol;  // by node
    std::vector<int> aDiag;       // node -> A block id of its diagonal
    std::vector<int> aToLu;       // A block id -> LU block id
    std::vector<int> luToA;       // LU block id -> A block id or -1 (pure fill-in)
    // Factorization: one task per LU block; its updates (L block, U block, the pivot's diagonal block) in ascending
    // pivot order; its level.  Default plan: L(i,k) = (A(i,k) - sum L(i,m) U(m,k)) inv(D_k) when its task runs, one
    // level after the pivot D_k.  Deferred-L plan: L blocks are computed unscaled (A(i,k) - sum L~(i,m) inv(D_m)
    // U(m,k)), so an update applies the pivot's inverted diagonal itself and an L block does not wait for its own
    // column's pivot; one last pass scales every L block by its pivot's inverse.
    std::vector<int> opPtr, opL, opU, opD;   // per LU block (opD -1: the L block is already scaled)
    bool deferredL = false;
    // Dense-front plan: positions frontStart .. nb-1 (frontF pivots); frontBlocks[i * F + j] is the LU block of front
    // positions (i, j), -1 for a structural zero; a front block's level task applies only its updates from pivots
    // before the front (opOuterEnd) and stores the partial sum, the dense front kernel does the rest.
    int frontStart = 0, frontF = 0;
    std::vector<int> frontBlocks, opOuterEnd;
    std::vector<int> level;             // per LU block
    std::vector<int> levelPtr, levelTask;  // tasks grouped by level (CSR); tasks are LU block ids
    // Triangular solves: forward over positions in L, backward in U; level sets of positions.
    std::vector<int> fwdLevelPtr, fwdLevelPos, bwdLevelPtr, bwdLevelPos;
    int64_t blockOps = 0;               // total 2x2 block multiply-subtracts per factorization
};

struct Structure {
    int n = 0, nnz = 0, ncb = 0, nob = 0, nsh = 0, nElements = 0;
    std::vector<int> rowMap, rowPtr, colIdx, diagPos;
    std::vector<int> cbDest, obDest, shDest;
    std::vector<double> cbPar, obPar, shPar;
    std::vector<int> cbIx, obIx, shIx;  // packs with rows mapped through rowMap
    // bus-block view
    int nb = 0;
    std::vector<int> nodeCol;           // [nb*2]: the node's angle (P row) and magnitude (Q row) columns
    std::vector<int> colNode;           // [n]: column -> node*2 + slot
    BlockPlan plan;
};

// Builds the structure; throws std::runtime_error on bad or unsupported input.
Structure buildStructure(int n, int ncb, const double* cbPar, const int* cbIx, int nob, const double* obPar,
                         const int* obIx, int nsh, const double* shPar, const int* shIx, int nid, const int* idRows,
                         int ordering);

// Orderings of the bus graph for the block LU (low bits), and the plan variant flag: PLAN_DEFERRED_L keeps the L
// factor unscaled during the factorization (half the dependency levels, one more block read per update).
enum Ordering { ORDER_MIN_DEGREE = 0, ORDER_NESTED_DISSECTION = 1, ORDER_NATURAL = 2, ORDER_MIN_DEGREE_SHALLOW = 3 };
constexpr int PLAN_DEFERRED_L = 8;
// Plan flag: the trailing positions of the elimination order whose blocks are all present (at most MAX_FRONT pivots,
// the root separators of the elimination tree) are factorized as one dense front in shared memory instead of one
// dependency level per step.
constexpr int PLAN_DENSE_FRONT = 16;
constexpr int MAX_FRONT = 32;

void buildBlockPlan(Structure& s, int ordering);

// Verifies a block-LU plan on the host from its dependency data alone, independently of how its levels were assigned
// (a level launch must share no data between its tasks; the reference checks its own LU schedules the same way,
// native/host/lu_transposed_check.cpp:175-216):
//  (1) the symbolic factorization is closed (every update L(a, m) U(m, b), m < min(a, b), lands on a block of the
//      pattern) and every block's update list is exactly those pivots m, ascending, with their operands (and, in the
//      deferred-L plan, the pivot inverse of m);
//  (2) the factorization levels hold every LU block once, and every block a task reads (the operands of the updates it
//      applies, the pivot inverse it scales by) lies on a strictly earlier level; a dense-front block's task applies
//      exactly its updates whose pivot precedes the front, and the front's block table is complete;
//  (3) the forward levels hold every position once, the backward levels every position outside the dense front once,
//      and every solution entry a position reads comes from a strictly earlier level (the front first, backward).
// plantedFault 1..3 checks a copy with one planted error instead (a task moved one level up; an update dropped; two
// forward positions swapped between the first and the last level), for tests of the check itself.  Returns the number
// of violations; first describes the first one.
int64_t checkBlockPlan(const BlockPlan& plan, int plantedFault, std::string& first);

}  // namespace olfb200
