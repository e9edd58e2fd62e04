// Persistent Newton-Raphson kernel: one CTA per tile of L lanes runs the whole Newton loop of its lanes -- fill,
// convergence test, reactive-limit outer loop, block-LU factorization, forward/backward solves, FP64 refinement
// (mixed precision) and the step -- with block barriers between dependency levels.  Lanes never depend on another
// tile, so no CTA ever waits for another one: the only synchronisation is __syncthreads.
//
// Thread t of the CTA serves lane (t % L) of the tile and work slot (t / L); a warp covers 32 / L slots, each reading
// L consecutive lanes (L * sizeof(T) contiguous bytes: one 32-byte sector for L = 4 in FP64, L = 8 in FP32).
#include "persistent.cuh"

#include <cmath>

namespace olfb200 {

namespace {

constexpr int MAX_SLOTS = 512;

template <typename T>
__device__ __forceinline__ void ld4(const T* base, size_t blk, size_t S, int s, T& a, T& b_, T& c, T& d) {
    const T* p = base + blk * 4 * S + s;
    a = p[0];
    b_ = p[S];
    c = p[2 * S];
    d = p[3 * S];
}

template <typename T>
__device__ __forceinline__ void st4(T* base, size_t blk, size_t S, int s, T a, T b_, T c, T d) {
    T* p = base + blk * 4 * S + s;
    p[0] = a;
    p[S] = b_;
    p[2 * S] = c;
    p[3 * S] = d;
}

__device__ __forceinline__ double absMaxP(double m, double v) {
    const double a = fabs(v);
    return (a > m || a != a) ? a : m;   // a NaN in either argument stays
}

// Per-tile state kept in shared memory for the duration of the kernel.
template <int L>
struct TileState {
    int active[L];       // lane iterates
    int pending[L];      // converged this iteration; reactive limits to check
    int solving[L];      // factorizes and steps this iteration
    int iter[L];
    int outer[L];
    int status[L];
    int trouble[L];
    int remainingPv[L];
    int any[L];
    int restart[L];      // failed this iteration and restarts (1: from the fallback start, 2: its FP64-grade restart)
    int refine;          // some lane of the tile is still refining
    int refining[L];     // mixed precision: this lane refines (near convergence or flagged) and its last correction
                         // was above the bound; a lane's refinement never depends on its tile-mates'
    unsigned long long norm[L];
    int live;            // any lane of the tile still active
};

// The split factor of a level with `count` tasks whose longest update list is `longest`: how many slots share a task
// (a power of two up to 32).
__device__ __forceinline__ int splitFor(int count, int longest, int slots) {
    int P = 1;
    while (P < 32 && count * (P * 2) <= slots && (longest + P - 1) / P > 2) P *= 2;
    return P;
}

// Factorization levels [l0, l1) of one tile, l1 being the last level: tasks of a level shared by P slots each
// (splitFor), partial sums added in a fixed order through shared memory; with the deferred-L plan, then the pass that
// scales every unscaled L block by its pivot's inverse.  `trouble` receives 1 for a lane that meets a near-singular 2x2 pivot.
template <typename T, int L>
__device__ void factorLevels(const DevNet& net, const DevBatch& b, T* lu, const int* levelPtr, const int* longest,
                             int l0, int l1, bool solve, int lane, int slot, int slots, int s, T (*red)[4][L],
                             int* trouble) {
    const size_t S = b.S;
    for (int l = l0; l < l1; l++) {
        const int first = levelPtr[l], count = levelPtr[l + 1] - first;
        const int P = splitFor(count, longest[l], slots);
        const int groups = slots / P;
        const int part = slot % P;
        for (int base = 0; base < count; base += groups) {
            const int kk = base + slot / P;
            const bool ok = solve && kk < count;
            T a00 = 0, a01 = 0, a10 = 0, a11 = 0, amax = 0;
            int t = 0;
            Task tk{};
            if (ok) {
                t = net.levelTask[first + kk];
                tk = net.task[t];
                if (part == 0 && tk.aBlock >= 0) {
                    const double* p = b.J + (size_t)tk.aBlock * 4 * S + s;
                    a00 = (T)p[0];
                    a01 = (T)p[S];
                    a10 = (T)p[2 * S];
                    a11 = (T)p[3 * S];
                    amax = fmax(fmax(fabs(a00), fabs(a01)), fmax(fabs(a10), fabs(a11)));
                }
#pragma unroll 2
                for (int q = tk.opBegin + part; q < tk.opEnd; q += P) {
                    const int4 op = net.ops[q];
                    T m00, m01, m10, m11, u00, u01, u10, u11;
                    ld4(lu, (size_t)op.x, S, s, m00, m01, m10, m11);
                    ld4(lu, (size_t)op.y, S, s, u00, u01, u10, u11);
                    if (op.z >= 0) {   // deferred-L plan: L~(a,m) inv(D_m)
                        T d00, d01, d10, d11;
                        ld4(lu, (size_t)op.z, S, s, d00, d01, d10, d11);
                        const T l00 = m00, l01 = m01, l10 = m10, l11 = m11;
                        m00 = l00 * d00 + l01 * d10;
                        m01 = l00 * d01 + l01 * d11;
                        m10 = l10 * d00 + l11 * d10;
                        m11 = l10 * d01 + l11 * d11;
                    }
                    a00 -= m00 * u00 + m01 * u10;
                    a01 -= m00 * u01 + m01 * u11;
                    a10 -= m10 * u00 + m11 * u10;
                    a11 -= m10 * u01 + m11 * u11;
                }
            }
            if (P > 1) {
                // the P partial sums of a task, added pairwise in a fixed tree order
                red[slot][0][lane] = a00;
                red[slot][1][lane] = a01;
                red[slot][2][lane] = a10;
                red[slot][3][lane] = a11;
                __syncthreads();
                for (int wd = P >> 1; wd > 0; wd >>= 1) {
                    if (part < wd) {
                        red[slot][0][lane] += red[slot + wd][0][lane];
                        red[slot][1][lane] += red[slot + wd][1][lane];
                        red[slot][2][lane] += red[slot + wd][2][lane];
                        red[slot][3][lane] += red[slot + wd][3][lane];
                    }
                    __syncthreads();
                }
                if (part == 0) {
                    a00 = red[slot][0][lane];
                    a01 = red[slot][1][lane];
                    a10 = red[slot][2][lane];
                    a11 = red[slot][3][lane];
                }
            }
            if (ok && part == 0) {
                if (tk.diag == -2) {
                    const T det = a00 * a11 - a01 * a10;
                    const T scale = fabs(a00 * a11) + fabs(a01 * a10);
                    if (!(fabs(det) > (T)1e-13 * scale) || !isfinite(det)) *trouble = 1;
                    const T inv = (T)1 / det;
                    if (sizeof(T) == 4 && b.precision64) {
                        // the pivot-growth flag of the mixed precision (tile schedules answer it with refinement)
                        const float dmax = fmaxf(fmaxf(fabsf((float)a00), fabsf((float)a01)),
                                                 fmaxf(fabsf((float)a10), fabsf((float)a11)));
                        const float kappa = dmax * dmax * fabsf((float)inv);
                        const float grow = amax > 0 ? dmax / (float)amax : 1.0f;
                        if (!(kappa <= (float)b.growthLimit) || !(grow <= (float)b.growthLimit)) b.precision64[s] = 1;
                    }
                    st4(lu, (size_t)t, S, s, a11 * inv, -a01 * inv, -a10 * inv, a00 * inv);
                } else if (tk.diag >= 0 && !net.deferredL) {
                    T i00, i01, i10, i11;
                    ld4(lu, (size_t)tk.diag, S, s, i00, i01, i10, i11);
                    st4(lu, (size_t)t, S, s, a00 * i00 + a01 * i10, a00 * i01 + a01 * i11, a10 * i00 + a11 * i10,
                        a10 * i01 + a11 * i11);
                } else {
                    st4(lu, (size_t)t, S, s, a00, a01, a10, a11);
                }
            }
            if (P > 1) __syncthreads();
        }
        __syncthreads();
    }
    if (solve && net.deferredL) {
        for (int id = net.nU + slot; id < net.nLu; id += slots) {
            T a00, a01, a10, a11, i00, i01, i10, i11;
            ld4(lu, (size_t)id, S, s, a00, a01, a10, a11);
            ld4(lu, (size_t)net.task[id].diag, S, s, i00, i01, i10, i11);
            st4(lu, (size_t)id, S, s, a00 * i00 + a01 * i10, a00 * i01 + a01 * i11, a10 * i00 + a11 * i10,
                a10 * i01 + a11 * i11);
        }
    }
    __syncthreads();
}

// Triangular-solve levels [l0, l1) of one tile: dir 0 forward (L rows), dir 1 backward (U rows, times the inverse
// diagonal block), in place on w.
template <typename T, int L>
__device__ void solveLevels(const DevNet& net, const DevBatch& b, const T* lu, T* w, const int* lp, const int* lpos,
                            const int* longest, int dir, int l0, int l1, bool solve, int lane, int slot, int slots,
                            int s, T (*red)[4][L]) {
    const size_t S = b.S;
    for (int l = l0; l < l1; l++) {
        const int first = lp[l], count = lp[l + 1] - first;
        const int P = splitFor(count, longest[l], slots);
        const int groups = slots / P;
        const int part = slot % P;
        for (int base = 0; base < count; base += groups) {
            const int kk = base + slot / P;
            const bool ok = solve && kk < count;
            T w0 = 0, w1 = 0;
            int i = 0;
            if (ok) {
                i = lpos[first + kk];
                if (part == 0) {
                    w0 = w[(2 * (size_t)i) * S + s];
                    w1 = w[(2 * (size_t)i + 1) * S + s];
                }
                if (dir == 0) {
                    for (int q = net.lrowPtr[i] + part; q < net.lrowEnd[i]; q += P) {
                        const int2 e = net.lrow[q];
                        T l00, l01, l10, l11;
                        ld4(lu, (size_t)e.x, S, s, l00, l01, l10, l11);
                        const T y0 = w[(2 * (size_t)e.y) * S + s], y1 = w[(2 * (size_t)e.y + 1) * S + s];
                        w0 -= l00 * y0 + l01 * y1;
                        w1 -= l10 * y0 + l11 * y1;
                    }
                } else {
                    for (int q = net.uPtr[i] + 1 + part; q < net.uPtr[i + 1]; q += P) {
                        const int j = net.uCol[q];
                        T u00, u01, u10, u11;
                        ld4(lu, (size_t)q, S, s, u00, u01, u10, u11);
                        const T x0 = w[(2 * (size_t)j) * S + s], x1 = w[(2 * (size_t)j + 1) * S + s];
                        w0 -= u00 * x0 + u01 * x1;
                        w1 -= u10 * x0 + u11 * x1;
                    }
                }
            }
            if (P > 1) {
                red[slot][0][lane] = w0;
                red[slot][1][lane] = w1;
                __syncthreads();
                for (int wd = P >> 1; wd > 0; wd >>= 1) {
                    if (part < wd) {
                        red[slot][0][lane] += red[slot + wd][0][lane];
                        red[slot][1][lane] += red[slot + wd][1][lane];
                    }
                    __syncthreads();
                }
                if (part == 0) {
                    w0 = red[slot][0][lane];
                    w1 = red[slot][1][lane];
                }
            }
            if (ok && part == 0) {
                if (dir == 0) {
                    w[(2 * (size_t)i) * S + s] = w0;
                    w[(2 * (size_t)i + 1) * S + s] = w1;
                } else {
                    T i00, i01, i10, i11;
                    ld4(lu, (size_t)net.uPtr[i], S, s, i00, i01, i10, i11);
                    w[(2 * (size_t)i) * S + s] = i00 * w0 + i01 * w1;
                    w[(2 * (size_t)i + 1) * S + s] = i10 * w0 + i11 * w1;
                }
            }
            if (P > 1) __syncthreads();
        }
        __syncthreads();
    }
}

}  // namespace

// The whole Newton loop of one tile of L lanes (the tile index picks the lanes); the body of both persistent kernels.
template <typename T, int L>
__device__ void newtonTile(const DevNet& net, const DevBatch& b, const DevRl& rl, const Settings& cfg,
                           const PersistentPlan& plan, int tile) {
    const int tid = threadIdx.x;
    const int lane = tid % L;
    const int slot = tid / L;
    const int slots = blockDim.x / L;
    const int s0 = tile * L;
    const int s = s0 + lane;
    const size_t S = b.S;
    T* lu = sizeof(T) == 8 ? reinterpret_cast<T*>(b.lu64) : reinterpret_cast<T*>(b.lu32);
    T* w = sizeof(T) == 8 ? reinterpret_cast<T*>(b.w64) : reinterpret_cast<T*>(b.w32);
    __shared__ TileState<L> ts;
    __shared__ T red[MAX_SLOTS / L][4][L];
    __shared__ double fred[MAX_SLOTS / L][L];
    const bool rlOn = cfg.reactiveLimits && rl.nRl > 0;

    if (tid < L) {
        ts.active[tid] = b.active[s0 + tid];
        ts.pending[tid] = 0;
        ts.iter[tid] = b.iter[s0 + tid];
        ts.outer[tid] = b.outer[s0 + tid];
        ts.status[tid] = b.status[s0 + tid];
        ts.trouble[tid] = 0;
        ts.norm[tid] = 0ull;
    }
    __syncthreads();

    for (int round = 0; round < plan.maxRounds; round++) {
        if (tid == 0) {
            int any = 0;
            for (int k = 0; k < L; k++) any |= ts.active[k];
            ts.live = any;
        }
        __syncthreads();
        if (!ts.live) break;
        const bool act = ts.active[lane];
        // ---------------- fill (fillKernel's terms; one (bus, lane) per thread) ----------------
        double fmax = 0.0;
        if (act) {
            const int words = b.S >> 5;
            for (int node = slot; node < net.nb; node += slots) {
                const int cP = net.nodeCol[2 * node], cV = net.nodeCol[2 * node + 1];
                const double thi = b.x[cP * S + s], vi = b.x[cV * S + s];
                const bool idP = b.mode[cP * S + s] == MODE_FIXED_VARIABLE;
                const bool idQ = b.mode[cV * S + s] == MODE_FIXED_VARIABLE;
                double fp = 0.0, fq = 0.0, qcl = 0.0;
                double d00 = 0.0, d01 = 0.0, d10 = 0.0, d11 = 0.0;
                double o00 = 0.0, o01 = 0.0, o10 = 0.0, o11 = 0.0;
                int curNb = -1, curBlk = -1;
                for (int t = net.sidePtr[node]; t <= net.sidePtr[node + 1]; t++) {
                    const bool end = t == net.sidePtr[node + 1];
                    Side sd{};
                    if (!end) sd = net.side[t];
                    if (end || sd.neighbour != curNb) {
                        if (curBlk >= 0) {
                            double* J = b.J + (size_t)curBlk * 4 * S + s;
                            J[0] = idP ? 0.0 : o00;
                            J[S] = idP ? 0.0 : o01;
                            J[2 * S] = idQ ? 0.0 : o10;
                            J[3 * S] = idQ ? 0.0 : o11;
                        }
                        if (end) break;
                        curNb = sd.neighbour;
                        curBlk = sd.aBlock;
                        o00 = o01 = o10 = o11 = 0.0;
                    }
                    const uint32_t word = b.disabled[(size_t)sd.element * words + (s >> 5)];
                    if ((word >> (s & 31)) & 1u) continue;
                    const double* p = net.cbPar + (size_t)sd.element * 8;
                    const double y = p[0], g1 = p[1], g2 = p[2], b1 = p[3], b2 = p[4], ksi = p[5], r1 = p[6], a1 = p[7];
                    const double2 tr = net.cbTrig[sd.element];
                    const double sk = tr.x, ck = tr.y;
                    const int jP = net.nodeCol[2 * sd.neighbour], jV = net.nodeCol[2 * sd.neighbour + 1];
                    const double thj = b.x[jP * S + s], vj = b.x[jV * S + s];
                    if (sd.side == 0) {
                        const double v1 = vi, v2 = vj;
                        double s1, c1;
                        sincos(ksi - a1 - thi + thj, &s1, &c1);
                        const double wc = y * r1 * v1 * v2 * c1, ws = y * r1 * v1 * v2 * s1;
                        const double q1 = r1 * v1 * (-b1 * r1 * v1 + y * r1 * v1 * ck - y * v2 * c1);
                        fp += r1 * v1 * (g1 * r1 * v1 + y * r1 * v1 * sk - y * v2 * s1);
                        fq += q1;
                        qcl += q1;
                        d00 += wc;
                        d01 += r1 * (2 * g1 * r1 * v1 + 2 * y * r1 * v1 * sk - y * v2 * s1);
                        d10 += -ws;
                        d11 += r1 * (-2 * b1 * r1 * v1 + 2 * y * r1 * v1 * ck - y * v2 * c1);
                        o00 += -wc;
                        o01 += -y * r1 * v1 * s1;
                        o10 += ws;
                        o11 += -y * r1 * v1 * c1;
                    } else {
                        const double v1 = vj, v2 = vi;
                        double s2, c2;
                        sincos(ksi + a1 + thj - thi, &s2, &c2);
                        const double wc = y * r1 * v1 * v2 * c2, ws = y * r1 * v1 * v2 * s2;
                        const double q2 = v2 * (-b2 * v2 - y * r1 * v1 * c2 + y * v2 * ck);
                        fp += v2 * (g2 * v2 - y * r1 * v1 * s2 + y * v2 * sk);
                        fq += q2;
                        qcl += q2;
                        d00 += wc;
                        d01 += 2 * g2 * v2 - y * r1 * v1 * s2 + 2 * y * v2 * sk;
                        d10 += -ws;
                        d11 += -2 * b2 * v2 - y * r1 * v1 * c2 + 2 * y * v2 * ck;
                        o00 += -wc;
                        o01 += -y * r1 * v2 * s2;
                        o10 += ws;
                        o11 += -y * r1 * v2 * c2;
                    }
                }
                for (int t = net.obPtr[node]; t < net.obPtr[node + 1]; t++) {
                    const int2 ob = net.obList[t];
                    const uint32_t word = b.disabled[(size_t)(net.ncb + ob.x) * words + (s >> 5)];
                    if ((word >> (s & 31)) & 1u) continue;
                    const double* p = net.obPar + (size_t)ob.x * 7;
                    const double y = p[0], ksi = p[1], g1 = p[2], b1 = p[3], g2 = p[4], b2 = p[5], r1 = p[6];
                    double sk, ck;
                    sincos(ksi, &sk, &ck);
                    if (ob.y == 0) {
                        const double dd = (g2 + y * sk) * (g2 + y * sk) + (-b2 + y * ck) * (-b2 + y * ck);
                        const double gp = g1 + y * y * g2 / dd + (b2 * b2 + g2 * g2) * y * sk / dd;
                        const double bq = b1 + y * y * b2 / dd - (b2 * b2 + g2 * g2) * y * ck / dd;
                        fp += r1 * r1 * vi * vi * gp;
                        fq += -r1 * r1 * vi * vi * bq;
                        d01 += 2 * r1 * r1 * vi * gp;
                        d11 += -2 * vi * r1 * r1 * bq;
                    } else {
                        const double dd = (g1 + y * sk) * (g1 + y * sk) + (-b1 + y * ck) * (-b1 + y * ck);
                        const double gp = g2 + y * y * g1 / dd + (b1 * b1 + g1 * g1) * y * sk / dd;
                        const double bq = b2 + y * y * b1 / dd - (b1 * b1 + g1 * g1) * y * ck / dd;
                        fp += vi * vi * gp;
                        fq += -vi * vi * bq;
                        d01 += 2 * vi * gp;
                        d11 += -2 * vi * bq;
                    }
                }
                for (int t = net.shPtr[node]; t < net.shPtr[node + 1]; t++) {
                    const int e = net.shList[t];
                    const uint32_t word = b.disabled[(size_t)(net.ncb + net.nob + e) * words + (s >> 5)];
                    if ((word >> (s & 31)) & 1u) continue;
                    const double g = net.shPar[2 * e], bb = net.shPar[2 * e + 1];
                    fp += g * vi * vi;
                    fq += -bb * vi * vi;
                    d01 += 2 * g * vi;
                    d11 += -2 * bb * vi;
                }
                double FP = fp - b.target[cP * S + s];
                double FQ = fq - b.target[cV * S + s];
                if (idP) FP = thi - b.target[cP * S + s];
                if (idQ) FQ = vi - b.target[cV * S + s];
                b.F[cP * S + s] = FP;
                b.F[cV * S + s] = FQ;
                if (rlOn) b.qbuf[cV * S + s] = qcl;
                double* J = b.J + (size_t)net.aDiag[node] * 4 * S + s;
                J[0] = idP ? 1.0 : d00;
                J[S] = idP ? 0.0 : d01;
                J[2 * S] = idQ ? 0.0 : d10;
                J[3 * S] = idQ ? 1.0 : d11;
                fmax = absMaxP(absMaxP(fmax, FP), FQ);
            }
        }
        fred[slot][lane] = fmax;
        __syncthreads();
        // ---------------- test (newton_iteration.cu:276-397) ----------------
        if (tid < L) {
            double nrm = 0.0;
            for (int k = 0; k < slots; k++) nrm = absMaxP(nrm, fred[k][tid]);
            ts.solving[tid] = 0;
            ts.pending[tid] = 0;
            ts.restart[tid] = 0;
            const int troubled = ts.trouble[tid];
            ts.trouble[tid] = 0;
            if (ts.active[tid]) {
                const int it = ts.iter[tid];
                b.normOut[s0 + tid] = nrm;
                int st = ST_RUNNING;
                // a lane whose last factorization met a near-singular pivot took no step: it ends here
                if (troubled) st = ST_LINEAR_SOLVE_FAILED;
                else if (!isfinite(nrm)) st = ST_DIVERGED;
                else if (it > 0 && nrm < cfg.tol && it < cfg.maxIter) {
                    if (cfg.polishBelow > 0.0 && b.fallbackLeft[s0 + tid] && nrm > cfg.polishBelow &&
                        it + 1 < cfg.maxIter) {
                        b.fallbackLeft[s0 + tid] = 0;   // one more step from inside the tolerance ball
                    } else if (rlOn && ts.outer[tid] < cfg.maxOuter) {
                        ts.pending[tid] = 1;
                        ts.remainingPv[tid] = 0;
                        ts.any[tid] = 0;
                    } else {
                        st = ST_CONVERGED;
                    }
                } else if (it == cfg.maxIter) {
                    st = ST_MAX_ITERATION_REACHED;
                }
                if (st != ST_RUNNING && st != ST_CONVERGED && b.fallbackLeft[s0 + tid]) {
                    b.fallbackLeft[s0 + tid] = 0;      // restart once from the fallback start (next round)
                    b.fellBack[s0 + tid] = 1;
                    ts.iter[tid] = 0;
                    ts.restart[tid] = 1;
                } else if (st != ST_RUNNING && st != ST_CONVERGED && b.fp64Left && b.fp64Left[s0 + tid]) {
                    // mixed precision: a failed lane restarts once from its start with every solve refined to the
                    // correction bound (precision64 marks it), so it follows the FP64 trajectory
                    b.fp64Left[s0 + tid] = 0;
                    b.precision64[s0 + tid] = 1;
                    ts.iter[tid] = 0;
                    ts.restart[tid] = 2;
                } else if (st != ST_RUNNING) {
                    ts.status[tid] = st;
                    ts.active[tid] = 0;
                } else if (!ts.pending[tid]) {
                    ts.solving[tid] = 1;
                }
            }
        }
        __syncthreads();
        if (ts.restart[lane] == 1 || (ts.restart[lane] == 2 && !b.restartFull)) {
            for (int r = slot; r < b.nFallback; r += slots) b.x[(size_t)r * S + s] = b.fallbackX[r];
        } else if (ts.restart[lane] == 2) {
            const int n = b.nFallback;
            for (int r = slot; r < n; r += slots) b.x[(size_t)r * S + s] = b.restartFull[(size_t)s * n + r];
        }
        // ---------------- reactive limits (reactive_limits.cu:321-359, 417-448) ----------------
        if (rlOn) {
            bool anyPending = false;
            for (int k = 0; k < L; k++) anyPending |= ts.pending[k] != 0;
            if (anyPending) {
                if (ts.pending[lane]) {
                    for (int i = slot; i < rl.nRl; i += slots) {
                        const size_t e = (size_t)i * S + s;
                        rl.passSwitched[e] = 0;
                        const size_t ri = (size_t)rl.voltageRow[i] * S + s;
                        if (b.mode[ri] == MODE_FIXED_VARIABLE && rl.limitType[e] == 0) {
                            const double q = b.qbuf[ri] + rl.loadQ[i];
                            if (q < rl.minQ[i] - cfg.rlTol || q > rl.maxQ[i] + cfg.rlTol) {
                                const bool low = q < rl.minQ[i] - cfg.rlTol;
                                rl.savedTarget[e] = b.target[ri];
                                rl.savedMode[e] = b.mode[ri];
                                b.mode[ri] = MODE_EQUATION;
                                b.target[ri] = (low ? rl.minQ[i] : rl.maxQ[i]) - rl.loadQ[i];
                                rl.limitType[e] = low ? 1 : 2;
                                rl.switchCount[e]++;
                                rl.passSwitched[e] = 1;
                            } else {
                                atomicAdd(&ts.remainingPv[lane], 1);
                            }
                        } else if (rl.limitType[e] != 0) {
                            const double v = b.x[ri];
                            const double tv = rl.targetV[i];
                            const bool wants = (rl.limitType[e] == 2 && v > tv) || (rl.limitType[e] == 1 && v < tv);
                            if (wants && rl.switchCount[e] < cfg.maxSwitch) {
                                b.mode[ri] = MODE_FIXED_VARIABLE;
                                b.target[ri] = tv;
                                rl.limitType[e] = 0;
                                rl.passSwitched[e] = 2;
                            }
                        }
                    }
                }
                __syncthreads();
                // forced-PV election: one thread per pending lane (no bus stayed PV in this check)
                if (tid < L && ts.pending[tid]) {
                    const int sl = s0 + tid;
                    int anySwitched = 0;
                    if (ts.remainingPv[tid] == 0) {
                        int best = -1, bestId = 0x7fffffff;
                        double bestV = -1.0, bestP = -1e300;
                        for (int i = 0; i < rl.nRl; i++) {
                            const size_t e = (size_t)i * S + sl;
                            if (rl.passSwitched[e] != 1) continue;
                            const double v = rl.nomV[i];
                            const double p = rl.pRow[i] >= 0 ? b.target[(size_t)rl.pRow[i] * S + sl] : rl.staticP[i];
                            const bool better = best < 0 || v > bestV ||
                                                (v == bestV && (p > bestP || (p == bestP && rl.idRank[i] < bestId)));
                            if (better) {
                                best = i;
                                bestV = v;
                                bestP = p;
                                bestId = rl.idRank[i];
                            }
                        }
                        if (best >= 0) {
                            const size_t e = (size_t)best * S + sl;
                            const size_t ri = (size_t)rl.voltageRow[best] * S + sl;
                            b.mode[ri] = rl.savedMode[e];
                            b.target[ri] = rl.savedTarget[e];
                            rl.limitType[e] = 0;
                            rl.switchCount[e]--;
                            rl.passSwitched[e] = 0;
                        }
                    }
                    for (int i = 0; i < rl.nRl && !anySwitched; i++) anySwitched = rl.passSwitched[(size_t)i * S + sl] != 0;
                    if (anySwitched) {
                        ts.iter[tid] = 0;          // restart at the new targets and modes (newton_iteration.cu:472-487)
                        ts.outer[tid]++;
                    } else {
                        ts.status[tid] = ST_CONVERGED;
                        ts.active[tid] = 0;
                    }
                }
                __syncthreads();
            }
        }
        // ---------------- factorization: level by level, P slots per task ----------------
        const bool solve = ts.solving[lane] != 0;
        bool anySolve = false;
        for (int k = 0; k < L; k++) anySolve |= ts.solving[k] != 0;
        if (anySolve) {
            factorLevels<T, L>(net, b, lu, plan.levelPtr, plan.levelLongest, 0, plan.nLevels, solve, lane, slot, slots, s,
                               red, &ts.trouble[lane]);
            // ---------------- solves (one pass, then the refinement passes in mixed precision) ----------------
            if (tid == 0) {
                int r = 0;
                for (int k = 0; k < L; k++) {
                    ts.refining[k] = ts.solving[k] && (b.normOut[s0 + k] < cfg.refineBelow || b.precision64[s0 + k]);
                    r |= ts.refining[k];
                }
                ts.refine = r;
            }
            __syncthreads();
            const int passes = 1 + (sizeof(T) == 4 && ts.refine ? cfg.refinementSteps : 0);
            for (int pass = 0; pass < passes; pass++) {
                // pass 0: every solving lane; a refinement pass: the lanes still refining
                const bool mine = pass == 0 ? solve : (solve && ts.refining[lane] != 0);
                if (pass > 0) {
                    // FP64 residual r = -F - J dx
                    if (mine) {
                        for (int node = slot; node < net.nb; node += slots) {
                            const int cP = net.nodeCol[2 * node], cV = net.nodeCol[2 * node + 1];
                            double r0 = -b.F[cP * S + s], r1 = -b.F[cV * S + s];
                            for (int t = net.aPtr[node]; t < net.aPtr[node + 1]; t++) {
                                const int j = net.aCol[t];
                                const double* J = b.J + (size_t)t * 4 * S + s;
                                const double x0 = b.dx[(size_t)net.nodeCol[2 * j] * S + s];
                                const double x1 = b.dx[(size_t)net.nodeCol[2 * j + 1] * S + s];
                                r0 -= J[0] * x0 + J[S] * x1;
                                r1 -= J[2 * S] * x0 + J[3 * S] * x1;
                            }
                            b.res[cP * S + s] = r0;
                            b.res[cV * S + s] = r1;
                        }
                    }
                    __syncthreads();
                }
                // right-hand side in elimination positions
                if (mine) {
                    for (int i = slot; i < net.nb; i += slots) {
                        const int node = net.perm[i];
                        const int cP = net.nodeCol[2 * node], cV = net.nodeCol[2 * node + 1];
                        const double r0 = pass == 0 ? -b.F[cP * S + s] : b.res[cP * S + s];
                        const double r1 = pass == 0 ? -b.F[cV * S + s] : b.res[cV * S + s];
                        w[(2 * (size_t)i) * S + s] = (T)r0;
                        w[(2 * (size_t)i + 1) * S + s] = (T)r1;
                    }
                }
                __syncthreads();
                solveLevels<T, L>(net, b, lu, w, plan.fwdPtr, plan.fwdPos, plan.fwdLongest, 0, 0, plan.nFwd, mine, lane,
                                  slot, slots, s, red);
                solveLevels<T, L>(net, b, lu, w, plan.bwdPtr, plan.bwdPos, plan.bwdLongest, 1, 0, plan.nBwd, mine, lane,
                                  slot, slots, s, red);
                // back to columns: dx = w (first pass) or dx += w (refinement)
                double dmax = 0.0;
                if (mine) {
                    for (int node = slot; node < net.nb; node += slots) {
                        const int i = net.iperm[node];
                        const int cP = net.nodeCol[2 * node], cV = net.nodeCol[2 * node + 1];
                        const double d0 = (double)w[(2 * (size_t)i) * S + s], d1 = (double)w[(2 * (size_t)i + 1) * S + s];
                        if (pass == 0) {
                            b.dx[cP * S + s] = d0;
                            b.dx[cV * S + s] = d1;
                        } else {
                            b.dx[cP * S + s] += d0;
                            b.dx[cV * S + s] += d1;
                            dmax = absMaxP(absMaxP(dmax, d0), d1);
                        }
                    }
                }
                if (pass > 0) {
                    // a lane stops refining once its correction is at or below the bound (a NaN one stops too)
                    fred[slot][lane] = dmax;
                    __syncthreads();
                    if (tid < L) {
                        double m = 0.0;
                        for (int k = 0; k < slots; k++) m = absMaxP(m, fred[k][tid]);
                        ts.refining[tid] = ts.refining[tid] && m > cfg.corrBound;
                    }
                    __syncthreads();
                    if (tid == 0) {
                        int r = 0;
                        for (int k = 0; k < L; k++) r |= ts.refining[k];
                        ts.refine = r;
                    }
                }
                __syncthreads();
                if (pass > 0 && !ts.refine) break;
            }
            // ---------------- step (not for a lane whose factorization failed) ----------------
            if (solve && !ts.trouble[lane]) {
                for (int r = slot; r < net.n; r += slots) b.x[(size_t)r * S + s] += b.dx[(size_t)r * S + s];
            }
        }
        __syncthreads();
        if (tid < L) {
            if (ts.solving[tid] && !ts.trouble[tid]) {
                ts.iter[tid]++;
                b.totalIter[s0 + tid]++;
            }
            ts.pending[tid] = 0;
        }
        __syncthreads();
    }
    if (tid < L) {
        const int sl = s0 + tid;
        b.iter[sl] = ts.iter[tid];
        b.outer[sl] = ts.outer[tid];
        b.status[sl] = ts.active[tid] ? ST_REJECTED : ts.status[tid];   // still iterating at the cap: REJECTED
        b.active[sl] = 0;
        b.trouble[sl] = ts.trouble[tid];
    }
}

template <typename T, int L>
__global__ void __launch_bounds__(512) newtonPersistentKernel(DevNet net, DevBatch b, DevRl rl, Settings cfg,
                                                              PersistentPlan plan) {
    newtonTile<T, L>(net, b, rl, cfg, plan, blockIdx.x);
}

// One launch over several grids: CTA k runs tile (k - tileBegin) of the item whose tile range holds k.
template <typename T, int L>
__global__ void __launch_bounds__(512) newtonMultiKernel(const MultiItem* items, int nItems) {
    __shared__ MultiItem it;    // the item's descriptors staged once per CTA (read on every access of the loop)
    if (threadIdx.x == 0) {
        int k = 0;
        while (k + 1 < nItems && static_cast<int>(blockIdx.x) >= items[k + 1].tileBegin) k++;
        it = items[k];
    }
    __syncthreads();
    newtonTile<T, L>(it.net, it.b, it.rl, it.cfg, it.plan, blockIdx.x - it.tileBegin);
}

void launchMulti(const MultiItem* itemsDevice, int nItems, int totalTiles, int lanesPerTile, int threads, bool fp32,
                 cudaStream_t st) {
#define OLF_MULTI(T_, L_) newtonMultiKernel<T_, L_><<<totalTiles, threads, 0, st>>>(itemsDevice, nItems)
    if (fp32) {
        switch (lanesPerTile) {
            case 1: OLF_MULTI(float, 1); break;
            case 2: OLF_MULTI(float, 2); break;
            case 4: OLF_MULTI(float, 4); break;
            default: OLF_MULTI(float, 8); break;
        }
    } else {
        switch (lanesPerTile) {
            case 1: OLF_MULTI(double, 1); break;
            case 2: OLF_MULTI(double, 2); break;
            case 4: OLF_MULTI(double, 4); break;
            default: OLF_MULTI(double, 8); break;
        }
    }
#undef OLF_MULTI
}

// Factorization levels [l0, l1) for every tile (the narrow top of the elimination tree in the level schedule).
template <typename T, int L>
__global__ void __launch_bounds__(512) factorRangeKernel(DevNet net, DevBatch b, PersistentPlan plan, int l0, int l1) {
    __shared__ T red[MAX_SLOTS / L][4][L];
    const int tid = threadIdx.x, lane = tid % L, slot = tid / L, slots = blockDim.x / L;
    const int s = blockIdx.x * L + lane;
    T* lu = sizeof(T) == 8 ? reinterpret_cast<T*>(b.lu64) : reinterpret_cast<T*>(b.lu32);
    const bool solve = b.active[s] && !b.pending[s] && (!b.laneMask || b.laneMask[s]);
    factorLevels<T, L>(net, b, lu, plan.levelPtr, plan.levelLongest, l0, l1, solve, lane, slot, slots, s, red,
                       &b.trouble[s]);
}

// Triangular-solve levels [l0, l1) in direction dir for every tile.
template <typename T, int L>
__global__ void __launch_bounds__(512) solveRangeKernel(DevNet net, DevBatch b, PersistentPlan plan, int dir, int l0,
                                                        int l1) {
    __shared__ T red[MAX_SLOTS / L][4][L];
    const int tid = threadIdx.x, lane = tid % L, slot = tid / L, slots = blockDim.x / L;
    const int s = blockIdx.x * L + lane;
    const T* lu = sizeof(T) == 8 ? reinterpret_cast<const T*>(b.lu64) : reinterpret_cast<const T*>(b.lu32);
    T* w = sizeof(T) == 8 ? reinterpret_cast<T*>(b.w64) : reinterpret_cast<T*>(b.w32);
    const bool solve = b.active[s] && !b.pending[s] && (!b.laneMask || b.laneMask[s]);
    if (dir == 0) {
        solveLevels<T, L>(net, b, lu, w, plan.fwdPtr, plan.fwdPos, plan.fwdLongest, 0, l0, l1, solve, lane, slot,
                          slots, s, red);
    } else {
        solveLevels<T, L>(net, b, lu, w, plan.bwdPtr, plan.bwdPos, plan.bwdLongest, 1, l0, l1, solve, lane, slot,
                          slots, s, red);
    }
}

void launchFactorRange(const DevNet& net, const DevBatch& b, const PersistentPlan& plan, int l0, int l1, int lanes,
                       bool fp32, cudaStream_t st) {
    if (l0 >= l1) return;
    const int tiles = b.S / lanes;
#define OLF_RANGE(T_, L_) factorRangeKernel<T_, L_><<<tiles, 256, 0, st>>>(net, b, plan, l0, l1)
    if (fp32) {
        if (lanes == 1) OLF_RANGE(float, 1);
        else if (lanes == 2) OLF_RANGE(float, 2);
        else OLF_RANGE(float, 4);
    } else {
        if (lanes == 1) OLF_RANGE(double, 1);
        else if (lanes == 2) OLF_RANGE(double, 2);
        else OLF_RANGE(double, 4);
    }
#undef OLF_RANGE
}

void launchSolveRange(const DevNet& net, const DevBatch& b, const PersistentPlan& plan, int dir, int l0, int l1,
                      int lanes, bool fp32, cudaStream_t st) {
    if (l0 >= l1) return;
    const int tiles = b.S / lanes;
#define OLF_RANGE(T_, L_) solveRangeKernel<T_, L_><<<tiles, 256, 0, st>>>(net, b, plan, dir, l0, l1)
    if (fp32) {
        if (lanes == 1) OLF_RANGE(float, 1);
        else if (lanes == 2) OLF_RANGE(float, 2);
        else OLF_RANGE(float, 4);
    } else {
        if (lanes == 1) OLF_RANGE(double, 1);
        else if (lanes == 2) OLF_RANGE(double, 2);
        else OLF_RANGE(double, 4);
    }
#undef OLF_RANGE
}

void launchPersistent(const DevNet& net, const DevBatch& b, const DevRl& rl, const Settings& cfg,
                      const PersistentPlan& plan, int lanesPerTile, int threads, bool fp32, cudaStream_t st) {
    const int tiles = b.S / lanesPerTile;
#define OLF_PERSISTENT(T_, L_) newtonPersistentKernel<T_, L_><<<tiles, threads, 0, st>>>(net, b, rl, cfg, plan)
    if (fp32) {
        switch (lanesPerTile) {
            case 1: OLF_PERSISTENT(float, 1); break;
            case 2: OLF_PERSISTENT(float, 2); break;
            case 4: OLF_PERSISTENT(float, 4); break;
            default: OLF_PERSISTENT(float, 8); break;
        }
    } else {
        switch (lanesPerTile) {
            case 1: OLF_PERSISTENT(double, 1); break;
            case 2: OLF_PERSISTENT(double, 2); break;
            case 4: OLF_PERSISTENT(double, 4); break;
            default: OLF_PERSISTENT(double, 8); break;
        }
    }
#undef OLF_PERSISTENT
}

}  // namespace olfb200
