/*
 * ORACLE -- test infrastructure only.
 *
 * A plain-C CPU restatement of the reference's batched AC Newton-Raphson N-1 path, used as the parity checker of the
 * CUDA engine and as the timed CPU baseline.  Only the tests, the smoke check and the benchmark's CPU-baseline leg
 * load this library; the product path never calls it.
 *
 * What it restates (reference files, paths relative to the reference project):
 *   - the OLF closed-branch / open-branch / shunt flow terms and their derivatives:
 *       native/cuda/equations/generated/closed_branch.cuh:30-229, open_branch.cuh:24-87, shunt.cuh:20-60
 *   - the scatter tables: native/cuda/equations/generated/{closed_branch,open_branch,shunt}_scatter.h
 *   - the diagonal-pairing row map: native/cuda/structure/csr_pattern.cu:75-240 (closed/open/shunt/identity parts)
 *   - the fixed superset CSR pattern: native/cuda/structure/shared_structure.cu:111-221 and
 *     structure_build.cuh:32-42 (collectPattern), the role-folded scatter map structure_build.cuh:51-66 (buildDest)
 *     and the diagonal slots shared_structure.cu:322-324
 *   - F = sum of element outputs - target (fill_launch.cu:117-126) and the FIXED_VARIABLE row mode
 *     (fill_launch.cu:82-115)
 *   - the Newton loop's test and status rules: native/cuda/solver/newton_iteration.cu:276-397 (>= 1 iteration,
 *     a test passing at the budget is MAX_ITERATION_REACHED, non-finite mismatch is DIVERGED)
 *   - the reactive-limit outer loop, local controllers: native/cuda/outerloop/reactive_limits.cu:321-359 and the
 *     forced-PV election reactive_limits.cu:417-448
 * The linear solves use a Gilbert-Peierls left-looking sparse LU with partial pivoting (Gilbert & Peierls, 1988) on
 * a minimum-degree column order of A + A^T -- an exact FP64 solver, independent of the engine's static-pivot
 * block LU.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define CB_OUT 28
#define OB_OUT 8
#define SH_OUT 5

/* ---------------------------------------------------------------------------------------------------------------
 * Flow terms (OLF formulas; R2 = 1, A2 = 0).
 * ------------------------------------------------------------------------------------------------------------- */

/* closed_branch.cuh:161-229: outputs in the scatter-table order p1, dp1dv1, dp1dv2, dp1dph1, dp1dph2, dp1da1,
 * dp1dr1, q1, ..., q2, ..., dq2dr1. params: y g1 g2 b1 b2 ksi r1 a1. */
void oracle_closed_branch(const double *p, double v1, double r1, double v2, double a1, double ph1, double ph2,
                          double *o)
{
    const double y = p[0], g1 = p[1], g2 = p[2], b1 = p[3], b2 = p[4], ksi = p[5];
    const double th1 = ksi - a1 - ph1 + ph2;
    const double th2 = ksi + a1 + ph1 - ph2;
    const double sk = sin(ksi), ck = cos(ksi);
    const double s1 = sin(th1), c1 = cos(th1), s2 = sin(th2), c2 = cos(th2);
    const double w1c = y * r1 * v1 * v2 * c1, w1s = y * r1 * v1 * v2 * s1;
    const double w2c = y * r1 * v1 * v2 * c2, w2s = y * r1 * v1 * v2 * s2;
    o[0] = r1 * v1 * (g1 * r1 * v1 + y * r1 * v1 * sk - y * v2 * s1);
    o[1] = r1 * (2 * g1 * r1 * v1 + 2 * y * r1 * v1 * sk - y * v2 * s1);
    o[2] = -y * r1 * v1 * s1;
    o[3] = w1c;
    o[4] = -w1c;
    o[5] = w1c;
    o[6] = v1 * (2 * r1 * v1 * (g1 + y * sk) - y * v2 * s1);
    o[7] = r1 * v1 * (-b1 * r1 * v1 + y * r1 * v1 * ck - y * v2 * c1);
    o[8] = r1 * (-2 * b1 * r1 * v1 + 2 * y * r1 * v1 * ck - y * v2 * c1);
    o[9] = -y * r1 * v1 * c1;
    o[10] = -w1s;
    o[11] = w1s;
    o[12] = -w1s;
    o[13] = v1 * (2 * r1 * v1 * (-b1 + y * ck) - y * v2 * c1);
    o[14] = v2 * (g2 * v2 - y * r1 * v1 * s2 + y * v2 * sk);
    o[15] = -y * r1 * v2 * s2;
    o[16] = 2 * g2 * v2 - y * r1 * v1 * s2 + 2 * y * v2 * sk;
    o[17] = -w2c;
    o[18] = w2c;
    o[19] = -w2c;
    o[20] = -y * v1 * v2 * s2;
    o[21] = v2 * (-b2 * v2 - y * r1 * v1 * c2 + y * v2 * ck);
    o[22] = -y * r1 * v2 * c2;
    o[23] = -2 * b2 * v2 - y * r1 * v1 * c2 + 2 * y * v2 * ck;
    o[24] = w2s;
    o[25] = -w2s;
    o[26] = w2s;
    o[27] = -y * v1 * v2 * c2;
}

/* open_branch.cuh:65-87: outputs p2, dp2dv2, q2, dq2dv2, p1, dp1dv1, q1, dq1dv1. params: y ksi g1 b1 g2 b2 r1. */
void oracle_open_branch(const double *p, double v1, double v2, double *o)
{
    const double y = p[0], ksi = p[1], g1 = p[2], b1 = p[3], g2 = p[4], b2 = p[5], r1 = p[6];
    const double sk = sin(ksi), ck = cos(ksi);
    const double d1 = (g1 + y * sk) * (g1 + y * sk) + (-b1 + y * ck) * (-b1 + y * ck);
    const double d2 = (g2 + y * sk) * (g2 + y * sk) + (-b2 + y * ck) * (-b2 + y * ck);
    const double gp2 = g2 + y * y * g1 / d1 + (b1 * b1 + g1 * g1) * y * sk / d1;
    const double bq2 = b2 + y * y * b1 / d1 - (b1 * b1 + g1 * g1) * y * ck / d1;
    const double gp1 = g1 + y * y * g2 / d2 + (b2 * b2 + g2 * g2) * y * sk / d2;
    const double bq1 = b1 + y * y * b2 / d2 - (b2 * b2 + g2 * g2) * y * ck / d2;
    o[0] = v2 * v2 * gp2;
    o[1] = 2 * v2 * gp2;
    o[2] = -v2 * v2 * bq2;
    o[3] = -2 * v2 * bq2;
    o[4] = r1 * r1 * v1 * v1 * gp1;
    o[5] = 2 * r1 * r1 * v1 * gp1;
    o[6] = -r1 * r1 * v1 * v1 * bq1;
    o[7] = -2 * v1 * r1 * r1 * bq1;
}

/* shunt.cuh:47-60: outputs p, dpdv, q, dqdv, dqdb. params: g b. */
void oracle_shunt(const double *p, double v, double *o)
{
    const double g = p[0], b = p[1];
    o[0] = g * v * v;
    o[1] = 2 * g * v;
    o[2] = -b * v * v;
    o[3] = -2 * b * v;
    o[4] = -v * v;
}

/* Scatter tables {role, rowEnd, rowEq, colEnd, colVar}: role 0 residual, 1 jacobian, 2 skip. */
static const int CB_SCATTER[CB_OUT][5] = {
    {0, 0, 0, -1, -1}, {1, 0, 0, 0, 1}, {1, 0, 0, 1, 1}, {1, 0, 0, 0, 0}, {1, 0, 0, 1, 0}, {1, 0, 0, 2, 0},
    {1, 0, 0, 2, 1},   {0, 0, 1, -1, -1}, {1, 0, 1, 0, 1}, {1, 0, 1, 1, 1}, {1, 0, 1, 0, 0}, {1, 0, 1, 1, 0},
    {1, 0, 1, 2, 0},   {1, 0, 1, 2, 1},   {0, 1, 0, -1, -1}, {1, 1, 0, 0, 1}, {1, 1, 0, 1, 1}, {1, 1, 0, 0, 0},
    {1, 1, 0, 1, 0},   {1, 1, 0, 2, 0},   {1, 1, 0, 2, 1},   {0, 1, 1, -1, -1}, {1, 1, 1, 0, 1}, {1, 1, 1, 1, 1},
    {1, 1, 1, 0, 0},   {1, 1, 1, 1, 0},   {1, 1, 1, 2, 0},   {1, 1, 1, 2, 1}};
static const int OB_SCATTER[OB_OUT][5] = {{0, 1, 0, -1, -1}, {1, 1, 0, 1, 1}, {0, 1, 1, -1, -1}, {1, 1, 1, 1, 1},
                                          {0, 0, 0, -1, -1}, {1, 0, 0, 0, 1}, {0, 0, 1, -1, -1}, {1, 0, 1, 0, 1}};
static const int SH_SCATTER[SH_OUT][5] = {{0, 0, 0, -1, -1}, {1, 0, 0, 0, 1}, {0, 0, 1, -1, -1}, {1, 0, 1, 0, 1},
                                          {1, 0, 1, 2, 0}};

/* csr_pattern.cu:38-71 (resolve*): a scatter row of one element -> (row, col), -1 when absent. */
static void resolve_cb(const int *s, const int *ix, int *row, int *col)
{
    *row = *col = -1;
    if (s[0] == 2) return;
    *row = ix[s[1] * 2 + s[2]];
    if (s[0] == 1) *col = ix[4 + s[3] * 2 + s[4]];
}
static void resolve_ob(const int *s, const int *ix, int *row, int *col)
{
    *row = *col = -1;
    if (s[0] == 2) return;
    *row = ix[s[1] * 2 + s[2]];
    if (s[0] == 1) *col = ix[4 + s[3]];
}
static void resolve_sh(const int *s, const int *ix, int *row, int *col)
{
    *row = *col = -1;
    if (s[0] == 2) return;
    *row = ix[s[2]];
    if (s[0] == 1) *col = (s[3] == 2) ? ix[3] : ix[2];
}

/* ---------------------------------------------------------------------------------------------------------------
 * Structure: row map, pattern, destinations.
 * ------------------------------------------------------------------------------------------------------------- */

typedef struct {
    int n, nnz, ncb, nob, nsh;
    int *row_map;               /* [n] equation row -> paired variable column */
    int *row_ptr, *col_idx;     /* CSR pattern (rows = mapped equations, cols = variables) */
    int *diag_pos;              /* [n] */
    int *cb_dest, *ob_dest, *sh_dest; /* role-folded destinations */
    double *cb_par, *ob_par, *sh_par;
    int *cb_ix, *ob_ix, *sh_ix; /* packed indices, rows mapped */
    char error[256];
} oracle_structure;

/* csr_pattern.cu:85-160 (buildRowMap's pairing): equation row `row` takes variable column `col` as its diagonal,
 * each column claimed once. */
static int pair_rc(int *rm, int row, int col, char *err)
{
    if (row < 0 || col < 0) return 0;
    if (rm[row] == -1) {
        rm[row] = col;
    } else if (rm[row] != col) {
        if (err) strcpy(err, "conflicting diagonal pairing");
        return -1;
    }
    return 0;
}

/* csr_pattern.cu:85-240 restricted to the closed-branch, open-branch, shunt and identity-row families. */
static int build_row_map(int n, int ncb, const int *cb_ix, int nob, const int *ob_ix, int nsh, const int *sh_ix,
                         int nid, const int *id_rows, int *rm, char *err)
{
    for (int i = 0; i < n; i++) rm[i] = -1;
    int rc = 0;
#define PAIR_P(prow, phcol) rc |= pair_rc(rm, (prow), (prow) == (phcol) ? (phcol) : (prow), err)
#define MOVED_V(qrow, vcol)                                                                                           \
    do {                                                                                                              \
        if ((vcol) >= 0 && (qrow) != (vcol)) rc |= pair_rc(rm, (vcol), (vcol), err);                                  \
    } while (0)
    for (int e = 0; e < ncb; e++) {
        const int *ix = cb_ix + (size_t)e * 12;
        PAIR_P(ix[0], ix[4]);
        PAIR_P(ix[2], ix[6]);
        rc |= pair_rc(rm, ix[1], ix[1], err);
        rc |= pair_rc(rm, ix[3], ix[3], err);
        MOVED_V(ix[1], ix[5]);
        MOVED_V(ix[3], ix[7]);
        if (ix[9] >= 0) rc |= pair_rc(rm, ix[9], ix[9], err);
        if (ix[8] >= 0) rc |= pair_rc(rm, ix[8], ix[8], err);
    }
    for (int e = 0; e < nob; e++) {
        const int *ix = ob_ix + (size_t)e * 6;
        rc |= pair_rc(rm, ix[1], ix[1], err);
        rc |= pair_rc(rm, ix[3], ix[3], err);
        MOVED_V(ix[1], ix[4]);
        MOVED_V(ix[3], ix[5]);
    }
    for (int e = 0; e < nsh; e++) {
        const int *ix = sh_ix + (size_t)e * 5;
        rc |= pair_rc(rm, ix[1], ix[1], err);
        MOVED_V(ix[1], ix[2]);
        if (ix[3] >= 0) rc |= pair_rc(rm, ix[3], ix[3], err);
    }
    for (int i = 0; i < nid; i++) rc |= pair_rc(rm, id_rows[i], id_rows[i], err);
#undef PAIR_P
#undef MOVED_V
    if (rc) return -1;
    char *used = (char *)calloc((size_t)n, 1);
    for (int r = 0; r < n; r++) {
        if (rm[r] < 0) {
            if (err) strcpy(err, "an equation row has no diagonal pairing");
            free(used);
            return -1;
        }
        if (used[rm[r]]) {
            if (err) strcpy(err, "diagonal pairing is not a bijection");
            free(used);
            return -1;
        }
        used[rm[r]] = 1;
    }
    free(used);
    return 0;
}

static int cmp_pair(const void *a, const void *b)
{
    const int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* The CSR slot of (row, col), -1 when absent: the lookup behind buildDest and diagPos (structure_build.cuh:51-66,
 * shared_structure.cu:322-324). */
static int csr_at(const oracle_structure *s, int row, int col)
{
    int lo = s->row_ptr[row], hi = s->row_ptr[row + 1];
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (s->col_idx[mid] < col) lo = mid + 1;
        else hi = mid;
    }
    if (lo >= s->row_ptr[row + 1] || s->col_idx[lo] != col) return -1;
    return lo;
}

void oracle_structure_free(oracle_structure *s)
{
    if (!s) return;
    free(s->row_map); free(s->row_ptr); free(s->col_idx); free(s->diag_pos);
    free(s->cb_dest); free(s->ob_dest); free(s->sh_dest);
    free(s->cb_par); free(s->ob_par); free(s->sh_par);
    free(s->cb_ix); free(s->ob_ix); free(s->sh_ix);
    free(s);
}

/* Builds the structure; returns NULL and writes err (>= 256 bytes) on failure. */
/* Builds the structure (row map csr_pattern.cu:75-240, superset pattern shared_structure.cu:111-221 with
 * collectPattern structure_build.cuh:32-42, destinations buildDest structure_build.cuh:51-66); returns NULL and writes
 * err (>= 256 bytes) on failure. */
oracle_structure *oracle_structure_build(int n, int ncb, const double *cb_par, const int *cb_ix, int nob,
                                         const double *ob_par, const int *ob_ix, int nsh, const double *sh_par,
                                         const int *sh_ix, int nid, const int *id_rows, char *err)
{
    oracle_structure *s = (oracle_structure *)calloc(1, sizeof(oracle_structure));
    s->n = n; s->ncb = ncb; s->nob = nob; s->nsh = nsh;
    s->row_map = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (build_row_map(n, ncb, cb_ix, nob, ob_ix, nsh, sh_ix, nid, id_rows, s->row_map, err) != 0) {
        oracle_structure_free(s);
        return NULL;
    }
    /* index packs rewritten through the row map (shared_structure.cu:85-97: cb slots 0-3,10,11; ob 0-3; sh 0,1,4) */
    s->cb_ix = (int *)malloc(sizeof(int) * (size_t)ncb * 12 + 4);
    s->ob_ix = (int *)malloc(sizeof(int) * (size_t)nob * 6 + 4);
    s->sh_ix = (int *)malloc(sizeof(int) * (size_t)nsh * 5 + 4);
    memcpy(s->cb_ix, cb_ix, sizeof(int) * (size_t)ncb * 12);
    memcpy(s->ob_ix, ob_ix, sizeof(int) * (size_t)nob * 6);
    memcpy(s->sh_ix, sh_ix, sizeof(int) * (size_t)nsh * 5);
    static const int CB_ROWS[6] = {0, 1, 2, 3, 10, 11}, OB_ROWS[4] = {0, 1, 2, 3}, SH_ROWS[3] = {0, 1, 4};
    for (int e = 0; e < ncb; e++)
        for (int k = 0; k < 6; k++) { int *r = &s->cb_ix[(size_t)e * 12 + CB_ROWS[k]]; if (*r >= 0) *r = s->row_map[*r]; }
    for (int e = 0; e < nob; e++)
        for (int k = 0; k < 4; k++) { int *r = &s->ob_ix[(size_t)e * 6 + OB_ROWS[k]]; if (*r >= 0) *r = s->row_map[*r]; }
    for (int e = 0; e < nsh; e++)
        for (int k = 0; k < 3; k++) { int *r = &s->sh_ix[(size_t)e * 5 + SH_ROWS[k]]; if (*r >= 0) *r = s->row_map[*r]; }
    s->cb_par = (double *)malloc(sizeof(double) * (size_t)ncb * 8 + 8);
    s->ob_par = (double *)malloc(sizeof(double) * (size_t)nob * 7 + 8);
    s->sh_par = (double *)malloc(sizeof(double) * (size_t)nsh * 2 + 8);
    memcpy(s->cb_par, cb_par, sizeof(double) * (size_t)ncb * 8);
    memcpy(s->ob_par, ob_par, sizeof(double) * (size_t)nob * 7);
    memcpy(s->sh_par, sh_par, sizeof(double) * (size_t)nsh * 2);

    /* pattern: role-1 entries of every family + the guaranteed diagonal, sorted and unique */
    size_t cap = (size_t)ncb * CB_OUT + (size_t)nob * OB_OUT + (size_t)nsh * SH_OUT + (size_t)n + 1;
    int64_t *pat = (int64_t *)malloc(sizeof(int64_t) * cap);
    size_t np = 0;
    int row, col;
    for (int e = 0; e < ncb; e++)
        for (int k = 0; k < CB_OUT; k++) {
            resolve_cb(CB_SCATTER[k], s->cb_ix + (size_t)e * 12, &row, &col);
            if (CB_SCATTER[k][0] == 1 && row >= 0 && col >= 0) pat[np++] = (int64_t)row * n + col;
        }
    for (int e = 0; e < nob; e++)
        for (int k = 0; k < OB_OUT; k++) {
            resolve_ob(OB_SCATTER[k], s->ob_ix + (size_t)e * 6, &row, &col);
            if (OB_SCATTER[k][0] == 1 && row >= 0 && col >= 0) pat[np++] = (int64_t)row * n + col;
        }
    for (int e = 0; e < nsh; e++)
        for (int k = 0; k < SH_OUT; k++) {
            resolve_sh(SH_SCATTER[k], s->sh_ix + (size_t)e * 5, &row, &col);
            if (SH_SCATTER[k][0] == 1 && row >= 0 && col >= 0) pat[np++] = (int64_t)row * n + col;
        }
    for (int r = 0; r < n; r++) pat[np++] = (int64_t)r * n + r;
    qsort(pat, np, sizeof(int64_t), cmp_pair);
    size_t u = 0;
    for (size_t i = 0; i < np; i++)
        if (u == 0 || pat[i] != pat[u - 1]) pat[u++] = pat[i];
    s->nnz = (int)u;
    s->row_ptr = (int *)calloc((size_t)n + 1, sizeof(int));
    s->col_idx = (int *)malloc(sizeof(int) * u);
    for (size_t i = 0; i < u; i++) {
        s->col_idx[i] = (int)(pat[i] % n);
        s->row_ptr[pat[i] / n + 1]++;
    }
    for (int r = 0; r < n; r++) s->row_ptr[r + 1] += s->row_ptr[r];
    free(pat);
    /* role-folded destinations (structure_build.cuh:51-66) */
    s->cb_dest = (int *)malloc(sizeof(int) * (size_t)ncb * CB_OUT + 4);
    s->ob_dest = (int *)malloc(sizeof(int) * (size_t)nob * OB_OUT + 4);
    s->sh_dest = (int *)malloc(sizeof(int) * (size_t)nsh * SH_OUT + 4);
#define DEST(TABLE, OUT, RES, IX, STRIDE, CNT, DST)                                                                  \
    for (int e = 0; e < (CNT); e++)                                                                                   \
        for (int k = 0; k < (OUT); k++) {                                                                             \
            RES(TABLE[k], (IX) + (size_t)e * (STRIDE), &row, &col);                                                   \
            int d = -1;                                                                                               \
            if (TABLE[k][0] == 1 && row >= 0 && col >= 0) d = csr_at(s, row, col);                                    \
            else if (TABLE[k][0] == 0 && row >= 0) d = -2 - row;                                                      \
            (DST)[(size_t)e * (OUT) + k] = d;                                                                         \
        }
    DEST(CB_SCATTER, CB_OUT, resolve_cb, s->cb_ix, 12, ncb, s->cb_dest)
    DEST(OB_SCATTER, OB_OUT, resolve_ob, s->ob_ix, 6, nob, s->ob_dest)
    DEST(SH_SCATTER, SH_OUT, resolve_sh, s->sh_ix, 5, nsh, s->sh_dest)
#undef DEST
    s->diag_pos = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int r = 0; r < n; r++) s->diag_pos[r] = csr_at(s, r, r);
    return s;
}

int oracle_structure_nnz(const oracle_structure *s) { return s->nnz; }

/* Copies out row map [n], rowPtr [n+1], colIdx [nnz], diagPos [n] and the three destination arrays. */
void oracle_structure_export(const oracle_structure *s, int *row_map, int *row_ptr, int *col_idx, int *diag_pos,
                             int *cb_dest, int *ob_dest, int *sh_dest)
{
    memcpy(row_map, s->row_map, sizeof(int) * (size_t)s->n);
    memcpy(row_ptr, s->row_ptr, sizeof(int) * ((size_t)s->n + 1));
    memcpy(col_idx, s->col_idx, sizeof(int) * (size_t)s->nnz);
    memcpy(diag_pos, s->diag_pos, sizeof(int) * (size_t)s->n);
    memcpy(cb_dest, s->cb_dest, sizeof(int) * (size_t)s->ncb * CB_OUT);
    memcpy(ob_dest, s->ob_dest, sizeof(int) * (size_t)s->nob * OB_OUT);
    memcpy(sh_dest, s->sh_dest, sizeof(int) * (size_t)s->nsh * SH_OUT);
}

/* ---------------------------------------------------------------------------------------------------------------
 * Fill (fill_launch.cu:82-126, the family fills branch_fill.cu:121-191): J values (CSR) and F for one scenario, element
 * order then output order (deterministic).
 * qbuf (optional, [n]): the closed-branch residual outputs on their rows, raw (fill_launch.cu qbuf channel).
 * ------------------------------------------------------------------------------------------------------------- */
static void fill(const oracle_structure *s, const double *x, const double *target, const int *mode,
                 const unsigned char *disabled, double *vals, double *F, double *qbuf)
{
    const int n = s->n;
    for (int r = 0; r < n; r++) F[r] = -target[r];
    if (vals) memset(vals, 0, sizeof(double) * (size_t)s->nnz);
    if (qbuf) memset(qbuf, 0, sizeof(double) * (size_t)n);
    double o[CB_OUT];
    for (int e = 0; e < s->ncb; e++) {
        if (disabled && disabled[e]) continue;
        const double *p = s->cb_par + (size_t)e * 8;
        const int *q = s->cb_ix + (size_t)e * 12;
        const double r1 = q[9] >= 0 ? x[q[9]] : p[6];
        const double a1 = q[8] >= 0 ? x[q[8]] : p[7];
        oracle_closed_branch(p, x[q[5]], r1, x[q[7]], a1, x[q[4]], x[q[6]], o);
        const int *d = s->cb_dest + (size_t)e * CB_OUT;
        for (int k = 0; k < CB_OUT; k++) {
            if (d[k] >= 0) { if (vals) vals[d[k]] += o[k]; }
            else if (d[k] <= -2) {
                F[-2 - d[k]] += o[k];
                if (qbuf) qbuf[-2 - d[k]] += o[k];
            }
        }
    }
    for (int e = 0; e < s->nob; e++) {
        if (disabled && disabled[s->ncb + e]) continue;
        const double *p = s->ob_par + (size_t)e * 7;
        const int *q = s->ob_ix + (size_t)e * 6;
        const double v1 = q[4] >= 0 ? x[q[4]] : 1.0, v2 = q[5] >= 0 ? x[q[5]] : 1.0;
        oracle_open_branch(p, v1, v2, o);
        const int *d = s->ob_dest + (size_t)e * OB_OUT;
        for (int k = 0; k < OB_OUT; k++) {
            if (d[k] >= 0) { if (vals) vals[d[k]] += o[k]; }
            else if (d[k] <= -2) F[-2 - d[k]] += o[k];
        }
    }
    for (int e = 0; e < s->nsh; e++) {
        if (disabled && disabled[s->ncb + s->nob + e]) continue;
        const double *p = s->sh_par + (size_t)e * 2;
        const int *q = s->sh_ix + (size_t)e * 5;
        oracle_shunt(p, x[q[2]], o);
        const int *d = s->sh_dest + (size_t)e * SH_OUT;
        for (int k = 0; k < SH_OUT; k++) {
            if (d[k] >= 0) { if (vals) vals[d[k]] += o[k]; }
            else if (d[k] <= -2) F[-2 - d[k]] += o[k];
        }
    }
    /* FIXED_VARIABLE rows (mode 0): row zeroed, diagonal 1, F = x - target (fill_launch.cu:96-103) */
    for (int r = 0; r < n; r++) {
        if (mode[r] != 0) continue;
        if (vals) {
            for (int k = s->row_ptr[r]; k < s->row_ptr[r + 1]; k++) vals[k] = 0.0;
            vals[s->diag_pos[r]] = 1.0;
        }
        F[r] = x[r] - target[r];
    }
}

/* One scenario's J values and F (parity checks of the engine's fill). */
/* One scenario's J values and F (parity checks of the engine's fill): fill_launch.cu:82-126 with the outaged
 * elements skipped (branch_fill.cu:133). */
void oracle_fill(const oracle_structure *s, const double *x, const double *target, const int *mode,
                 const unsigned char *disabled, double *vals, double *F)
{
    fill(s, x, target, mode, disabled, vals, F, NULL);
}

/* ---------------------------------------------------------------------------------------------------------------
 * Minimum-degree ordering of A + A^T (explicit elimination graph; ties to the lowest index).
 * ------------------------------------------------------------------------------------------------------------- */
typedef struct { int *v; int len, cap; } ivec;

static void iv_push(ivec *a, int x)
{
    if (a->len == a->cap) { a->cap = a->cap ? 2 * a->cap : 8; a->v = (int *)realloc(a->v, sizeof(int) * (size_t)a->cap); }
    a->v[a->len++] = x;
}

/* The oracle's own fill-reducing order for its own LU (not a restatement: the reference orders with
 * minimum_degree.cu, which the tests reach through oracle/ref), so its solves are independent of the engine's plan. */
static void min_degree(int n, const int *rp, const int *ci, int *perm)
{
    ivec *adj = (ivec *)calloc((size_t)n, sizeof(ivec));
    for (int r = 0; r < n; r++)
        for (int k = rp[r]; k < rp[r + 1]; k++) {
            int c = ci[k];
            if (c == r) continue;
            iv_push(&adj[r], c);
            iv_push(&adj[c], r);
        }
    int *mark = (int *)malloc(sizeof(int) * (size_t)n);
    for (int i = 0; i < n; i++) mark[i] = -1;
    /* dedupe adjacency */
    for (int i = 0; i < n; i++) {
        int w = 0;
        for (int k = 0; k < adj[i].len; k++) {
            int c = adj[i].v[k];
            if (mark[c] != i) { mark[c] = i; adj[i].v[w++] = c; }
        }
        adj[i].len = w;
    }
    char *done = (char *)calloc((size_t)n, 1);
    /* degree buckets as doubly linked lists */
    int *head = (int *)malloc(sizeof(int) * (size_t)(n + 1)), *next = (int *)malloc(sizeof(int) * (size_t)n),
        *prev = (int *)malloc(sizeof(int) * (size_t)n), *deg = (int *)malloc(sizeof(int) * (size_t)n);
    for (int d = 0; d <= n; d++) head[d] = -1;
    for (int i = n - 1; i >= 0; i--) {
        deg[i] = adj[i].len;
        next[i] = head[deg[i]]; prev[i] = -1;
        if (head[deg[i]] >= 0) prev[head[deg[i]]] = i;
        head[deg[i]] = i;
    }
    int mind = 0, stamp = n;
    for (int step = 0; step < n; step++) {
        while (head[mind] < 0) mind++;
        /* lowest index among the minimum-degree bucket */
        int v = head[mind], best = v;
        for (int u = v; u >= 0; u = next[u]) if (u < best) best = u;
        v = best;
        if (prev[v] >= 0) next[prev[v]] = next[v]; else head[deg[v]] = next[v];
        if (next[v] >= 0) prev[next[v]] = prev[v];
        done[v] = 1;
        perm[step] = v;
        /* neighbours of v still alive form a clique */
        ivec nb = {0, 0, 0};
        for (int k = 0; k < adj[v].len; k++) if (!done[adj[v].v[k]]) iv_push(&nb, adj[v].v[k]);
        for (int a = 0; a < nb.len; a++) {
            int u = nb.v[a];
            stamp++;
            ivec nu = {0, 0, 0};
            for (int k = 0; k < adj[u].len; k++) {
                int c = adj[u].v[k];
                if (!done[c] && mark[c] != stamp) { mark[c] = stamp; iv_push(&nu, c); }
            }
            for (int b = 0; b < nb.len; b++) {
                int c = nb.v[b];
                if (c != u && mark[c] != stamp) { mark[c] = stamp; iv_push(&nu, c); }
            }
            free(adj[u].v);
            adj[u] = nu;
            /* re-bucket u */
            if (prev[u] >= 0) next[prev[u]] = next[u]; else head[deg[u]] = next[u];
            if (next[u] >= 0) prev[next[u]] = prev[u];
            deg[u] = nu.len;
            next[u] = head[deg[u]]; prev[u] = -1;
            if (head[deg[u]] >= 0) prev[head[deg[u]]] = u;
            head[deg[u]] = u;
            if (deg[u] < mind) mind = deg[u];
        }
        free(nb.v);
        free(adj[v].v);
        adj[v].v = NULL; adj[v].len = adj[v].cap = 0;
    }
    for (int i = 0; i < n; i++) free(adj[i].v);
    free(adj); free(mark); free(done); free(head); free(next); free(prev); free(deg);
}

/* ---------------------------------------------------------------------------------------------------------------
 * Gilbert-Peierls left-looking LU with partial pivoting (columns in a given order): the oracle's own exact solver, not
 * a restatement (the reference's LU is reached through oracle/ref and pins this one in the tests).
 * A is given by rows (CSR); it is transposed to columns first.
 * ------------------------------------------------------------------------------------------------------------- */
typedef struct {
    int n;
    int *cp, *ri;     /* A by columns */
    int *map;         /* CSR position -> CSC position */
    int *q;           /* column order */
    /* factors */
    int *Lp, *Li, *Up, *Ui, *pinv;
    double *Lx, *Ux;
    size_t lcap, ucap;
    /* work */
    double *x;
    int *xi, *stack, *pstack, *flag;
} glu;

static glu *glu_new(int n, const int *rp, const int *ci, const int *q)
{
    glu *g = (glu *)calloc(1, sizeof(glu));
    g->n = n;
    int nnz = rp[n];
    g->cp = (int *)calloc((size_t)n + 1, sizeof(int));
    g->ri = (int *)malloc(sizeof(int) * (size_t)(nnz + 1));
    g->map = (int *)malloc(sizeof(int) * (size_t)(nnz + 1));
    for (int k = 0; k < nnz; k++) g->cp[ci[k] + 1]++;
    for (int c = 0; c < n; c++) g->cp[c + 1] += g->cp[c];
    int *w = (int *)malloc(sizeof(int) * (size_t)n);
    memcpy(w, g->cp, sizeof(int) * (size_t)n);
    for (int r = 0; r < n; r++)
        for (int k = rp[r]; k < rp[r + 1]; k++) {
            int pos = w[ci[k]]++;
            g->ri[pos] = r;
            g->map[k] = pos;
        }
    free(w);
    g->q = (int *)malloc(sizeof(int) * (size_t)n);
    memcpy(g->q, q, sizeof(int) * (size_t)n);
    g->Lp = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    g->Up = (int *)malloc(sizeof(int) * ((size_t)n + 1));
    g->pinv = (int *)malloc(sizeof(int) * (size_t)n);
    g->lcap = g->ucap = (size_t)4 * nnz + (size_t)n;
    g->Li = (int *)malloc(sizeof(int) * g->lcap);
    g->Lx = (double *)malloc(sizeof(double) * g->lcap);
    g->Ui = (int *)malloc(sizeof(int) * g->ucap);
    g->Ux = (double *)malloc(sizeof(double) * g->ucap);
    g->x = (double *)calloc((size_t)n, sizeof(double));
    g->xi = (int *)malloc(sizeof(int) * (size_t)n);
    g->stack = (int *)malloc(sizeof(int) * (size_t)n);
    g->pstack = (int *)malloc(sizeof(int) * (size_t)n);
    g->flag = (int *)malloc(sizeof(int) * (size_t)n);
    return g;
}

static void glu_free(glu *g)
{
    if (!g) return;
    free(g->cp); free(g->ri); free(g->map); free(g->q);
    free(g->Lp); free(g->Up); free(g->pinv); free(g->Li); free(g->Lx); free(g->Ui); free(g->Ux);
    free(g->x); free(g->xi); free(g->stack); free(g->pstack); free(g->flag);
    free(g);
}

/* Factor the CSC values ax (in g's column layout). Returns 0, or -1 when a column has no usable pivot. */
static int glu_factor(glu *g, const double *ax)
{
    const int n = g->n;
    size_t lnz = 0, unz = 0;
    for (int i = 0; i < n; i++) { g->pinv[i] = -1; g->flag[i] = -1; }
    for (int k = 0; k < n; k++) {
        g->Lp[k] = (int)lnz;
        g->Up[k] = (int)unz;
        if (lnz + (size_t)n > g->lcap) {
            g->lcap = 2 * g->lcap + (size_t)n;
            g->Li = (int *)realloc(g->Li, sizeof(int) * g->lcap);
            g->Lx = (double *)realloc(g->Lx, sizeof(double) * g->lcap);
        }
        if (unz + (size_t)n > g->ucap) {
            g->ucap = 2 * g->ucap + (size_t)n;
            g->Ui = (int *)realloc(g->Ui, sizeof(int) * g->ucap);
            g->Ux = (double *)realloc(g->Ux, sizeof(double) * g->ucap);
        }
        const int col = g->q[k];
        /* symbolic reach of A(:,col) in the graph of L (DFS, topological order into xi[top..n)) */
        int top = n;
        for (int p = g->cp[col]; p < g->cp[col + 1]; p++) {
            int j = g->ri[p];
            if (g->flag[j] == k) continue;
            int head = 0;
            g->stack[0] = j;
            while (head >= 0) {
                int jj = g->stack[head];
                int jcol = g->pinv[jj];
                if (g->flag[jj] != k) {
                    g->flag[jj] = k;
                    g->pstack[head] = jcol < 0 ? 0 : g->Lp[jcol];
                }
                int done = 1;
                int pend = jcol < 0 ? 0 : g->Lp[jcol + 1];
                for (int pp = g->pstack[head]; pp < pend; pp++) {
                    int i = g->Li[pp];
                    if (g->flag[i] == k) continue;
                    g->pstack[head] = pp + 1;
                    g->stack[++head] = i;
                    done = 0;
                    break;
                }
                if (done) {
                    head--;
                    g->xi[--top] = jj;
                }
            }
        }
        /* numeric: x = L \ A(:,col) on the reach */
        for (int p = top; p < n; p++) g->x[g->xi[p]] = 0.0;
        for (int p = g->cp[col]; p < g->cp[col + 1]; p++) g->x[g->ri[p]] = ax[p];
        for (int px = top; px < n; px++) {
            int j = g->xi[px];
            int J = g->pinv[j];
            if (J < 0) continue;
            double xj = g->x[j];
            for (int p = g->Lp[J] + 1; p < g->Lp[J + 1]; p++) g->x[g->Li[p]] -= g->Lx[p] * xj;
        }
        /* pivot: the largest non-pivotal entry; keep the structural diagonal when within a factor 10 */
        int ipiv = -1;
        double amax = -1.0;
        for (int px = top; px < n; px++) {
            int i = g->xi[px];
            if (g->pinv[i] < 0) {
                double t = fabs(g->x[i]);
                if (t > amax) { amax = t; ipiv = i; }
            } else {
                g->Ui[unz] = g->pinv[i];
                g->Ux[unz++] = g->x[i];
            }
        }
        if (ipiv < 0 || amax <= 0.0 || !isfinite(amax)) return -1;
        if (g->pinv[col] < 0 && g->flag[col] == k && fabs(g->x[col]) >= 0.1 * amax) ipiv = col;
        double piv = g->x[ipiv];
        g->Ui[unz] = k;
        g->Ux[unz++] = piv;
        g->pinv[ipiv] = k;
        g->Li[lnz] = ipiv;
        g->Lx[lnz++] = 1.0;
        for (int px = top; px < n; px++) {
            int i = g->xi[px];
            if (g->pinv[i] < 0) {
                g->Li[lnz] = i;
                g->Lx[lnz++] = g->x[i] / piv;
            }
            g->x[i] = 0.0;
        }
    }
    g->Lp[n] = (int)lnz;
    g->Up[n] = (int)unz;
    /* L's row indices to pivot order */
    for (size_t p = 0; p < lnz; p++) g->Li[p] = g->pinv[g->Li[p]];
    return 0;
}

/* Solve A z = b; z may alias b. */
static void glu_solve(glu *g, const double *b, double *z)
{
    const int n = g->n;
    double *w = g->x;
    for (int i = 0; i < n; i++) w[g->pinv[i]] = b[i];
    for (int j = 0; j < n; j++) {
        double wj = w[j];
        for (int p = g->Lp[j] + 1; p < g->Lp[j + 1]; p++) w[g->Li[p]] -= g->Lx[p] * wj;
    }
    for (int j = n - 1; j >= 0; j--) {
        w[j] /= g->Ux[g->Up[j + 1] - 1];
        double wj = w[j];
        for (int p = g->Up[j]; p < g->Up[j + 1] - 1; p++) w[g->Ui[p]] -= g->Ux[p] * wj;
    }
    for (int k = 0; k < n; k++) z[g->q[k]] = w[k];
    for (int i = 0; i < n; i++) w[i] = 0.0;
}

/* ---------------------------------------------------------------------------------------------------------------
 * Newton-Raphson with the reference's status rules, plus the reactive-limit outer loop.
 * ------------------------------------------------------------------------------------------------------------- */
enum { ST_CONVERGED = 0, ST_MAX_ITER = 1, ST_UNREALISTIC = 2, ST_DIVERGED = -1, ST_REJECTED = -2,
       ST_LINEAR_SOLVE_FAILED = -3 };

/* iterative_refinement.cuh:21-23: a linear solve whose residual ratio ||J dx + F||inf / ||F||inf exceeds this did not
 * solve its system. */
#define LIN_SOLVE_FAIL_RATIO 1e-2

/* Options of the batched solve beyond the plain Newton loop (NULL: none). */
typedef struct {
    double conv_eps_per_eq;       /* > 0: OLF's ||F||2 < sqrt(eps^2 n) test (newton_iteration.cu:105,241-250) */
    int svs_mode;                 /* 0 NONE, 2 MAX_VOLTAGE_CHANGE (state_vector_scaling.cu:53-97) */
    double max_dv, max_dphi;
    const int *var_type;          /* [n] 0 BUS_V, 1 BUS_PHI */
    const unsigned char *v_check; /* [n] realistic-voltage rows, or NULL (realistic_voltage_check.cu:23-44) */
    double min_v, max_v;
} oracle_opts;

typedef struct {
    int n_rl;
    const int *voltage_row;
    const double *min_q, *max_q, *load_q, *target_v, *nom_v, *static_p;
    const int *p_row, *id_rank;
} oracle_rl;

typedef struct {
    oracle_structure *s;
    int *perm;
} oracle_solver;

oracle_solver *oracle_solver_new(oracle_structure *s)
{
    oracle_solver *o = (oracle_solver *)calloc(1, sizeof(oracle_solver));
    o->s = s;
    o->perm = (int *)malloc(sizeof(int) * (size_t)(s->n > 0 ? s->n : 1));
    min_degree(s->n, s->row_ptr, s->col_idx, o->perm);
    return o;
}

void oracle_solver_free(oracle_solver *o)
{
    if (!o) return;
    free(o->perm);
    free(o);
}

/* The linear-solve residual ratio of a solve J dx = -F (linResidScoreBatch, iterative_refinement.cu:42-65):
 * max |J dx + F| / max |F|, 1e300 when F is zero or the residual is not finite. */
static double solve_ratio(const oracle_structure *s, const double *vals, const double *dx, const double *F)
{
    double mr = 0.0, mf = 0.0;
    int finite = 1;
    for (int r = 0; r < s->n; r++) {
        double acc = F[r];
        for (int k = s->row_ptr[r]; k < s->row_ptr[r + 1]; k++) acc += vals[k] * dx[s->col_idx[k]];
        if (!isfinite(acc)) finite = 0;
        if (fabs(acc) > mr) mr = fabs(acc);
        if (fabs(F[r]) > mf) mf = fabs(F[r]);
    }
    return (mf > 0.0 && finite) ? mr / mf : 1e300;
}

/* One Newton solve in place on x (mode/target may be changed only by the caller). Returns the status.
 * newton_iteration.cu:276-397 with the linear-solve guard of :615-647: at least one iteration; the test at the budget is
 * MAX_ITERATION_REACHED, or, when the solve before it did not solve its system (ratio above LIN_SOLVE_FAIL_RATIO),
 * REJECTED in a batch and LINEAR_SOLVE_FAILED for a batch of one; the second iteration of a scenario's first solve
 * (first_solve: no reactive-limit restart yet) ends LINEAR_SOLVE_FAILED when its solve fails the ratio; a singular
 * factorization ends LINEAR_SOLVE_FAILED at the iteration that met it. */
static int newton(const oracle_structure *s, glu *g, double *x, const double *target, const int *mode,
                  const unsigned char *dis, int max_iter, double tol, int *iters, double *norm_out, double *vals,
                  double *ax, double *F, double *dx, double *qbuf, int first_solve, int batch_of_one,
                  const oracle_opts *op)
{
    const int n = s->n;
    const double thr2 = (op && op->conv_eps_per_eq > 0.0) ? sqrt(op->conv_eps_per_eq * op->conv_eps_per_eq * n) : 0.0;
    double last_ratio = 0.0;
    for (int it = 0;; it++) {
        fill(s, x, target, mode, dis, vals, F, qbuf);
        double nrm = 0.0, ssq = 0.0;
        int finite = 1;
        for (int r = 0; r < n; r++) {
            if (!isfinite(F[r])) { finite = 0; break; }
            double a = fabs(F[r]);
            if (a > nrm) nrm = a;
            ssq += F[r] * F[r];
        }
        *iters = it;
        *norm_out = finite ? nrm : NAN;
        if (!finite) return ST_DIVERGED;
        int converged = thr2 > 0.0 ? sqrt(ssq) < thr2 : nrm < tol;
        if (it > 0 && converged && it < max_iter) return ST_CONVERGED;
        if (it == max_iter) {
            if (!(last_ratio <= LIN_SOLVE_FAIL_RATIO)) return batch_of_one ? ST_LINEAR_SOLVE_FAILED : ST_REJECTED;
            return ST_MAX_ITER;
        }
        for (int k = 0; k < s->nnz; k++) ax[g->map[k]] = vals[k];
        if (glu_factor(g, ax) != 0) return ST_LINEAR_SOLVE_FAILED;
        for (int r = 0; r < n; r++) dx[r] = -F[r];
        glu_solve(g, dx, dx);
        const int guard = first_solve && it == 1, budget = it == max_iter - 1;
        if (guard || budget) {
            double ratio = solve_ratio(s, vals, dx, F);
            if (budget) last_ratio = ratio;
            if (guard && !(ratio <= LIN_SOLVE_FAIL_RATIO)) return ST_LINEAR_SOLVE_FAILED;
        }
        double f = 1.0;
        if (op && op->svs_mode == 2) {
            /* MAX_VOLTAGE_CHANGE: the whole step scaled so max |dV| <= max_dv and max |dphi| <= max_dphi */
            double mdv = 0.0, mdphi = 0.0;
            for (int r = 0; r < n; r++) {
                double a = fabs(dx[r]);
                if (op->var_type[r] == 0) mdv = fmax(mdv, a);
                else if (op->var_type[r] == 1) mdphi = fmax(mdphi, a);
            }
            if (mdv > op->max_dv) f = fmin(f, op->max_dv / mdv);
            if (mdphi > op->max_dphi) f = fmin(f, op->max_dphi / mdphi);
            for (int r = 0; r < n; r++) x[r] += f * dx[r];
        } else {
            for (int r = 0; r < n; r++) x[r] += dx[r];
        }
    }
}

/* realistic_voltage_check.cu:23-44: a checked voltage outside [min_v, max_v] */
static int unrealistic(const oracle_opts *op, int n, const double *x)
{
    if (!op || !op->v_check) return 0;
    for (int r = 0; r < n; r++)
        if (op->v_check[r] && (x[r] < op->min_v || x[r] > op->max_v)) return 1;
    return 0;
}

/* reactive_limits.cu:321-359 (local controllers) + reactive_limits.cu:417-448 (forced-PV election).
 * Returns 1 when a row changed (the scenario restarts its Newton). */
static int reactive_limits_check(const oracle_rl *rl, int n, const double *x, const double *qbuf, int *mode,
                                 double *target, signed char *limit_type, signed char *switch_count,
                                 signed char *pass_switched, signed char *saved_mode, double *saved_target,
                                 double tol, int max_switch)
{
    int remaining_pv = 0;
    for (int i = 0; i < rl->n_rl; i++) pass_switched[i] = 0;
    for (int i = 0; i < rl->n_rl; i++) {
        const int r = rl->voltage_row[i];
        if (mode[r] == 0 && limit_type[i] == 0) {
            double q = qbuf[r] + rl->load_q[i];
            if (q < rl->min_q[i] - tol) {
                saved_target[i] = target[r]; saved_mode[i] = (signed char)mode[r];
                mode[r] = 1; target[r] = rl->min_q[i] - rl->load_q[i];
                limit_type[i] = 1; switch_count[i]++; pass_switched[i] = 1;
            } else if (q > rl->max_q[i] + tol) {
                saved_target[i] = target[r]; saved_mode[i] = (signed char)mode[r];
                mode[r] = 1; target[r] = rl->max_q[i] - rl->load_q[i];
                limit_type[i] = 2; switch_count[i]++; pass_switched[i] = 1;
            } else {
                remaining_pv++;
            }
        } else if (limit_type[i] != 0) {
            double v = x[r];
            double tv = rl->target_v[i];
            int wants = (limit_type[i] == 2 && v > tv) || (limit_type[i] == 1 && v < tv);
            if (wants && switch_count[i] < max_switch) {
                mode[r] = 0; target[r] = tv; limit_type[i] = 0; pass_switched[i] = 2;
            }
        }
    }
    if (remaining_pv == 0) {
        int best = -1, best_id = 0x7fffffff;
        double best_v = -1.0, best_p = -1e300;
        for (int i = 0; i < rl->n_rl; i++) {
            if (pass_switched[i] != 1) continue;
            double v = rl->nom_v[i];
            double p = rl->p_row[i] >= 0 ? target[rl->p_row[i]] : rl->static_p[i];
            int better = best < 0 || v > best_v || (v == best_v && (p > best_p || (p == best_p && rl->id_rank[i] < best_id)));
            if (better) { best = i; best_v = v; best_p = p; best_id = rl->id_rank[i]; }
        }
        if (best >= 0) {
            int r = rl->voltage_row[best];
            mode[r] = saved_mode[best]; target[r] = saved_target[best];
            limit_type[best] = 0; switch_count[best]--; pass_switched[best] = 0;
        }
    }
    for (int i = 0; i < rl->n_rl; i++) if (pass_switched[i]) return 1;
    (void)n;
    return 0;
}

/* Distributed-slack participants (bus level) of the batched solve (NULL: none). */
typedef struct {
    int n_ds;
    const int *row;              /* participants' P rows */
    const double *factor;        /* participation factors (normalised to sum 1 by the solve) */
    const double *base, *max_delta, *min_delta;
    int slack_row;               /* the slack bus's angle row: its closed-branch P is in qbuf there */
    double slack_target_p;
    double dist_tol;             /* slackBusPMaxMismatch (pu) */
    int reject;                  /* a failed distribution ends the scenario REJECTED */
} oracle_ds;

#define P_RESIDUE_EPS 1e-5

/* distributed_slack.cu:211-616 (bus level), after a converged solve: the slack's closed-branch P minus its target
 * is the mismatch; above dist_tol every participant resets to its base target and the whole amount is water-filled
 * over them in proportion to their factors within their bounds.  Returns 1 when the targets moved by more than
 * 0.9 P_RESIDUE_EPS (the scenario re-solves); *failed when more than P_RESIDUE_EPS stayed unplaced. */
static int distributed_slack_check(const oracle_ds *ds, const double *factor, const double *qbuf, double *target,
                                   double *prev, int *failed)
{
    *failed = 0;
    double mis = qbuf[ds->slack_row] - ds->slack_target_p;
    if (!(fabs(mis) > ds->dist_tol && fabs(mis) > P_RESIDUE_EPS)) return 0;
    double absorbed = 0.0;
    for (int i = 0; i < ds->n_ds; i++) {
        absorbed += target[ds->row[i]] - ds->base[i];
        prev[i] = target[ds->row[i]];
        target[ds->row[i]] = ds->base[i];
    }
    double rem = mis + absorbed;
    for (int it = 0; it < ds->n_ds && fabs(rem) > P_RESIDUE_EPS; it++) {
        double fsum = 0.0;
        for (int i = 0; i < ds->n_ds; i++) {
            double cum = target[ds->row[i]] - ds->base[i];
            int sat = rem > 0 ? cum >= ds->max_delta[i] : cum <= ds->min_delta[i];
            if (!sat) fsum += factor[i];
        }
        if (fsum <= 0.0) break;
        double done = 0.0;
        for (int i = 0; i < ds->n_ds; i++) {
            double cum = target[ds->row[i]] - ds->base[i];
            int sat = rem > 0 ? cum >= ds->max_delta[i] : cum <= ds->min_delta[i];
            if (sat) continue;
            double next = fmin(fmax(cum + rem * (factor[i] / fsum), ds->min_delta[i]), ds->max_delta[i]);
            if (next != cum) {
                target[ds->row[i]] = ds->base[i] + next;
                done += next - cum;
            }
        }
        rem -= done;
    }
    double shift = 0.0;
    for (int i = 0; i < ds->n_ds; i++) shift += fabs(target[ds->row[i]] - prev[i]);
    *failed = fabs(rem) > P_RESIDUE_EPS;
    return shift > 0.9 * P_RESIDUE_EPS;
}

/*
 * Batched N-1 solve: scenario s starts from x0 (x0_stride 0: one shared start; n: one per scenario), the base
 * targets and row modes, and disables the elements flagged in disabled[s * n_elements ...].
 * out: per scenario [x(n), iterations, ||F||inf, status] (batch_solve_jni.cu:308-337).
 * Reactive limits: rl may be NULL; max_outer bounds the Newton restarts.  Returns 0.
 */
/* The batched solve with the outer loops; final_target / final_mode ([ns][n], each may be NULL) receive every
 * scenario's targets and row modes as its solve ended with them (the outer loops rewrite both: reactive_limits.cu
 * switches PV rows to PQ at a Q limit, the distributed slack moves its participants' P targets), the per-scenario
 * readbacks of batch_readback_jni.cu:13-45. */
int oracle_solve_batch_final(oracle_solver *o, int ns, const double *x0, int x0_stride, const double *target_base,
                             const int *mode_base, const unsigned char *disabled, int n_elements, int max_iter,
                             double tol, const oracle_rl *rl, double rl_tol, int max_outer, int max_switch, int threads,
                             const oracle_opts *opts, const oracle_ds *ds, double *out, double *final_target,
                             int *final_mode)
{
    const oracle_structure *s = o->s;
    const int n = s->n;
    /* the factors normalised as the engine does: a plain sum in order, then each divided by it */
    const int nds = ds ? ds->n_ds : 0;
    double *dsf = (double *)malloc(sizeof(double) * ((size_t)nds + 1));
    {
        double fsum = 0.0;
        for (int i = 0; i < nds; i++) fsum += ds->factor[i];
        for (int i = 0; i < nds; i++) dsf[i] = ds->factor[i] / fsum;
    }
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
#pragma omp parallel
    {
        glu *g = glu_new(n, s->row_ptr, s->col_idx, o->perm);
        double *vals = (double *)malloc(sizeof(double) * (size_t)s->nnz);
        double *ax = (double *)malloc(sizeof(double) * (size_t)s->nnz);
        double *F = (double *)malloc(sizeof(double) * (size_t)n);
        double *dx = (double *)malloc(sizeof(double) * (size_t)n);
        double *qbuf = (double *)malloc(sizeof(double) * (size_t)n);
        double *target = (double *)malloc(sizeof(double) * (size_t)n);
        int *mode = (int *)malloc(sizeof(int) * (size_t)n);
        int nrl = rl ? rl->n_rl : 0;
        signed char *lt = (signed char *)malloc((size_t)nrl + 1), *sc = (signed char *)malloc((size_t)nrl + 1),
                    *ps = (signed char *)malloc((size_t)nrl + 1), *sm = (signed char *)malloc((size_t)nrl + 1);
        double *st = (double *)malloc(sizeof(double) * ((size_t)nrl + 1));
        double *dsprev = (double *)malloc(sizeof(double) * ((size_t)nds + 1));
#pragma omp for schedule(dynamic, 1)
        for (int sc_i = 0; sc_i < ns; sc_i++) {
            double *x = out + (size_t)sc_i * (n + 3);
            memcpy(x, x0 + (size_t)sc_i * x0_stride, sizeof(double) * (size_t)n);
            memcpy(target, target_base, sizeof(double) * (size_t)n);
            memcpy(mode, mode_base, sizeof(int) * (size_t)n);
            memset(lt, 0, (size_t)nrl + 1); memset(sc, 0, (size_t)nrl + 1);
            const unsigned char *dis = disabled ? disabled + (size_t)sc_i * n_elements : NULL;
            int iters = 0, status = ST_CONVERGED;
            double nrm = 0.0;
            for (int outer = 0;; outer++) {
                status = newton(s, g, x, target, mode, dis, max_iter, tol, &iters, &nrm, vals, ax, F, dx, qbuf,
                                outer == 0, ns == 1, opts);
                if (status != ST_CONVERGED || (nrl == 0 && nds == 0) || outer >= max_outer) break;
                if (nds > 0) {   /* distributed slack first, then reactive limits (the outer-loop order) */
                    int failed = 0;
                    int moved = distributed_slack_check(ds, dsf, qbuf, target, dsprev, &failed);
                    if (failed && ds->reject) {
                        status = ST_REJECTED;
                        break;
                    }
                    if (moved) continue;
                }
                if (nrl == 0) break;
                if (!reactive_limits_check(rl, n, x, qbuf, mode, target, lt, sc, ps, sm, st, rl_tol, max_switch)) break;
            }
            if (status == ST_CONVERGED && unrealistic(opts, n, x)) status = ST_UNREALISTIC;
            x[n] = (double)iters;   /* the last inner solve's iterations (res.iters, newton_iteration.cu:338) */
            x[n + 1] = nrm;
            x[n + 2] = (double)status;
            if (final_target) memcpy(final_target + (size_t)sc_i * n, target, sizeof(double) * (size_t)n);
            if (final_mode) memcpy(final_mode + (size_t)sc_i * n, mode, sizeof(int) * (size_t)n);
        }
        glu_free(g);
        free(vals); free(ax); free(F); free(dx); free(qbuf); free(target); free(mode);
        free(lt); free(sc); free(ps); free(sm); free(st); free(dsprev);
    }
    free(dsf);
    return 0;
}

/* The batched solve with the distributed-slack loop and no final-equation outputs (oracle_solve_batch_final). */
int oracle_solve_batch_ds(oracle_solver *o, int ns, const double *x0, int x0_stride, const double *target_base,
                          const int *mode_base, const unsigned char *disabled, int n_elements, int max_iter, double tol,
                          const oracle_rl *rl, double rl_tol, int max_outer, int max_switch, int threads,
                          const oracle_opts *opts, const oracle_ds *ds, double *out)
{
    return oracle_solve_batch_final(o, ns, x0, x0_stride, target_base, mode_base, disabled, n_elements, max_iter, tol,
                                    rl, rl_tol, max_outer, max_switch, threads, opts, ds, out, NULL, NULL);
}

/* The batched solve without distributed slack: outer_loop_driver.cu:80-460 over newton_iteration.cu:276-397. */
int oracle_solve_batch_ex(oracle_solver *o, int ns, const double *x0, int x0_stride, const double *target_base,
                          const int *mode_base, const unsigned char *disabled, int n_elements, int max_iter, double tol,
                          const oracle_rl *rl, double rl_tol, int max_outer, int max_switch, int threads,
                          const oracle_opts *opts, double *out)
{
    return oracle_solve_batch_ds(o, ns, x0, x0_stride, target_base, mode_base, disabled, n_elements, max_iter, tol,
                                 rl, rl_tol, max_outer, max_switch, threads, opts, NULL, out);
}

/* The batched solve with the default options (no 2-norm test, no step scaling, no realistic check). */
int oracle_solve_batch(oracle_solver *o, int ns, const double *x0, int x0_stride, const double *target_base,
                       const int *mode_base, const unsigned char *disabled, int n_elements, int max_iter, double tol,
                       const oracle_rl *rl, double rl_tol, int max_outer, int max_switch, int threads, double *out)
{
    return oracle_solve_batch_ex(o, ns, x0, x0_stride, target_base, mode_base, disabled, n_elements, max_iter, tol, rl,
                                 rl_tol, max_outer, max_switch, threads, NULL, out);
}

/* Solve one linear system J z = b with the oracle LU (tests of the engine's batched LU; the reference's counterpart is
 * its batched LU, lu/batched_lu.cu:66-149 and scalar_lu.cu:318-334). Returns 0 or -1. */
int oracle_linear_solve(oracle_solver *o, const double *vals, const double *b, double *z)
{
    const oracle_structure *s = o->s;
    glu *g = glu_new(s->n, s->row_ptr, s->col_idx, o->perm);
    double *ax = (double *)calloc((size_t)(s->nnz > 0 ? s->nnz : 1), sizeof(double));
    for (int k = 0; k < s->nnz; k++) ax[g->map[k]] = vals[k];
    int rc = glu_factor(g, ax);
    if (rc == 0) glu_solve(g, b, z);
    free(ax);
    glu_free(g);
    return rc;
}

/* Solve the transposed system J^T z = b with the oracle LU on the explicit transpose (tests of the engine's transposed
 * solve on its own factors, the reference's lu/transposed_solve.cuh:39-159).  Returns 0 or -1 (singular). */
int oracle_linear_solve_transposed(oracle_solver *o, const double *vals, const double *b, double *z)
{
    const oracle_structure *s = o->s;
    const int n = s->n, nnz = s->nnz;
    int *tp = (int *)calloc((size_t)n + 1, sizeof(int));
    int *ti = (int *)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    double *tv = (double *)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
    int *fill = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int *perm = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int k = 0; k < nnz; k++) tp[s->col_idx[k] + 1]++;
    for (int r = 0; r < n; r++) tp[r + 1] += tp[r];
    for (int r = 0; r < n; r++) fill[r] = tp[r];
    for (int r = 0; r < n; r++)                       /* rows ascending: each transposed row's columns ascend */
        for (int k = s->row_ptr[r]; k < s->row_ptr[r + 1]; k++) {
            int q = fill[s->col_idx[k]]++;
            ti[q] = r;
            tv[q] = vals[k];
        }
    min_degree(n, tp, ti, perm);
    glu *g = glu_new(n, tp, ti, perm);
    double *ax = (double *)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
    for (int k = 0; k < nnz; k++) ax[g->map[k]] = tv[k];
    int rc = glu_factor(g, ax);
    if (rc == 0) glu_solve(g, b, z);
    free(ax);
    glu_free(g);
    free(tp); free(ti); free(tv); free(fill); free(perm);
    return rc;
}
