// Device kernels of the batched Newton-Raphson engine (sm_100a).  See kernels.cuh for the layouts.
#include "kernels.cuh"

#include <cmath>

namespace olfb200 {

namespace {

__device__ __forceinline__ bool solving(const DevBatch& b, int s) {
    return b.active[s] && !b.pending[s] && (!b.laneMask || b.laneMask[s]);
}

// NaN-propagating running maximum of |v| (a NaN stays: it orders above +inf as unsigned bits).
__device__ __forceinline__ double absMax(double m, double v) {
    const double a = fabs(v);
    return (a > m || a != a) ? a : m;   // a NaN in either argument stays
}

}  // namespace

// ---------------------------------------------------------------------------------------------------------------
// Fused Jacobian / mismatch fill: one thread per (bus, lane).  The thread owns its bus's two rows, so every value
// is written once, in a fixed order, with no atomics; the FIXED_VARIABLE row modes are applied in the same pass.
// Terms: closed branches (equations/generated/closed_branch.cuh:161-229), open branches (open_branch.cuh:65-87),
// shunts (shunt.cuh:47-60); F = terms - target (fill_launch.cu:117-126); identity rows (fill_launch.cu:96-103).
// The per-lane max |F| is reduced in the block and folded into norm[s] with one atomic per block and lane.  Five
// resident CTAs per SM: the fill is latency-bound, and occupancy pays more than a few spilled registers (measured per
// 500-lane fill: 2 CTAs 535 us, 4 CTAs 324 us; per step, 3 CTAs 2 % slower and 5 CTAs 0.5 % faster than 4).
// ---------------------------------------------------------------------------------------------------------------
template <bool WITH_J, bool WITH_Q>
__global__ void __launch_bounds__(256, 5) fillKernel(DevNet net, DevBatch b) {
    const int s = blockIdx.x * 32 + threadIdx.x;
    const int node = blockIdx.y * blockDim.y + threadIdx.y;
    const size_t S = b.S;
    __shared__ double red[8][33];
    double fmax = 0.0;
    const bool live = node < net.nb && s < b.S && b.active[s];
    if (live) {
        const int cP = net.nodeCol[2 * node], cV = net.nodeCol[2 * node + 1];
        const double thi = b.x[cP * S + s], vi = b.x[cV * S + s];
        const bool idP = b.mode[cP * S + s] == MODE_FIXED_VARIABLE;
        const bool idQ = b.mode[cV * S + s] == MODE_FIXED_VARIABLE;
        const int words = b.S >> 5;
        double fp = 0.0, fq = 0.0, pcl = 0.0, qcl = 0.0;
        double d00 = 0.0, d01 = 0.0, d10 = 0.0, d11 = 0.0;
        double o00 = 0.0, o01 = 0.0, o10 = 0.0, o11 = 0.0;
        int curNb = -1, curBlk = -1;
        auto flushOff = [&]() {
            if (WITH_J && curBlk >= 0) {
                double* J = b.J + (size_t)curBlk * 4 * S + s;
                J[0] = idP ? 0.0 : o00;
                J[S] = idP ? 0.0 : o01;
                J[2 * S] = idQ ? 0.0 : o10;
                J[3 * S] = idQ ? 0.0 : o11;
            }
        };
        for (int t = net.sidePtr[node]; t < net.sidePtr[node + 1]; t++) {
            const Side sd = net.side[t];
            if (sd.neighbour != curNb) {
                flushOff();
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
                // the bus is side 1: v1 = vi, ph1 = thi, v2 = vj, ph2 = thj
                const double v1 = vi, v2 = vj;
                const double th1 = ksi - a1 - thi + thj;
                double s1, c1;
                sincos(th1, &s1, &c1);
                const double wc = y * r1 * v1 * v2 * c1, ws = y * r1 * v1 * v2 * s1;
                const double p1 = r1 * v1 * (g1 * r1 * v1 + y * r1 * v1 * sk - y * v2 * s1);
                const double q1 = r1 * v1 * (-b1 * r1 * v1 + y * r1 * v1 * ck - y * v2 * c1);
                fp += p1;
                fq += q1;
                pcl += p1;
                qcl += q1;
                if (WITH_J) {
                    d00 += wc;                                                             // dp1dph1
                    d01 += r1 * (2 * g1 * r1 * v1 + 2 * y * r1 * v1 * sk - y * v2 * s1);   // dp1dv1
                    d10 += -ws;                                                            // dq1dph1
                    d11 += r1 * (-2 * b1 * r1 * v1 + 2 * y * r1 * v1 * ck - y * v2 * c1);  // dq1dv1
                    o00 += -wc;                                                            // dp1dph2
                    o01 += -y * r1 * v1 * s1;                                              // dp1dv2
                    o10 += ws;                                                             // dq1dph2
                    o11 += -y * r1 * v1 * c1;                                              // dq1dv2
                }
            } else {
                // the bus is side 2: v2 = vi, ph2 = thi, v1 = vj, ph1 = thj
                const double v1 = vj, v2 = vi;
                const double th2 = ksi + a1 + thj - thi;
                double s2, c2;
                sincos(th2, &s2, &c2);
                const double wc = y * r1 * v1 * v2 * c2, ws = y * r1 * v1 * v2 * s2;
                const double p2 = v2 * (g2 * v2 - y * r1 * v1 * s2 + y * v2 * sk);
                const double q2 = v2 * (-b2 * v2 - y * r1 * v1 * c2 + y * v2 * ck);
                fp += p2;
                fq += q2;
                pcl += p2;
                qcl += q2;
                if (WITH_J) {
                    d00 += wc;                                             // dp2dph2
                    d01 += 2 * g2 * v2 - y * r1 * v1 * s2 + 2 * y * v2 * sk;  // dp2dv2
                    d10 += -ws;                                            // dq2dph2
                    d11 += -2 * b2 * v2 - y * r1 * v1 * c2 + 2 * y * v2 * ck;  // dq2dv2
                    o00 += -wc;                                            // dp2dph1
                    o01 += -y * r1 * v2 * s2;                              // dp2dv1
                    o10 += ws;                                             // dq2dph1
                    o11 += -y * r1 * v2 * c2;                              // dq2dv1
                }
            }
        }
        flushOff();
        for (int t = net.obPtr[node]; t < net.obPtr[node + 1]; t++) {
            const int2 ob = net.obList[t];
            const uint32_t word = b.disabled[(size_t)(net.ncb + ob.x) * words + (s >> 5)];
            if ((word >> (s & 31)) & 1u) continue;
            const double* p = net.obPar + (size_t)ob.x * 7;
            const double y = p[0], ksi = p[1], g1 = p[2], b1 = p[3], g2 = p[4], b2 = p[5], r1 = p[6];
            double sk, ck;
            sincos(ksi, &sk, &ck);
            if (ob.y == 0) {
                // side 1 connected, side 2 open: p1/q1 at this bus, variable v1
                const double d2 = (g2 + y * sk) * (g2 + y * sk) + (-b2 + y * ck) * (-b2 + y * ck);
                const double gp1 = g1 + y * y * g2 / d2 + (b2 * b2 + g2 * g2) * y * sk / d2;
                const double bq1 = b1 + y * y * b2 / d2 - (b2 * b2 + g2 * g2) * y * ck / d2;
                fp += r1 * r1 * vi * vi * gp1;
                fq += -r1 * r1 * vi * vi * bq1;
                if (WITH_J) {
                    d01 += 2 * r1 * r1 * vi * gp1;
                    d11 += -2 * vi * r1 * r1 * bq1;
                }
            } else {
                const double d1 = (g1 + y * sk) * (g1 + y * sk) + (-b1 + y * ck) * (-b1 + y * ck);
                const double gp2 = g2 + y * y * g1 / d1 + (b1 * b1 + g1 * g1) * y * sk / d1;
                const double bq2 = b2 + y * y * b1 / d1 - (b1 * b1 + g1 * g1) * y * ck / d1;
                fp += vi * vi * gp2;
                fq += -vi * vi * bq2;
                if (WITH_J) {
                    d01 += 2 * vi * gp2;
                    d11 += -2 * vi * bq2;
                }
            }
        }
        for (int t = net.shPtr[node]; t < net.shPtr[node + 1]; t++) {
            const int e = net.shList[t];
            const uint32_t word = b.disabled[(size_t)(net.ncb + net.nob + e) * words + (s >> 5)];
            if ((word >> (s & 31)) & 1u) continue;
            const double g = net.shPar[2 * e], bb = net.shPar[2 * e + 1];
            fp += g * vi * vi;
            fq += -bb * vi * vi;
            if (WITH_J) {
                d01 += 2 * g * vi;
                d11 += -2 * bb * vi;
            }
        }
        double FP = fp - b.target[cP * S + s];
        double FQ = fq - b.target[cV * S + s];
        if (idP) FP = thi - b.target[cP * S + s];
        if (idQ) FQ = vi - b.target[cV * S + s];
        b.F[cP * S + s] = FP;
        b.F[cV * S + s] = FQ;
        if (WITH_Q) {   // the closed-branch flows on the bus's rows (reactive limits read Q, distributed slack P)
            b.qbuf[cP * S + s] = pcl;
            b.qbuf[cV * S + s] = qcl;
        }
        if (WITH_J) {
            double* J = b.J + (size_t)net.aDiag[node] * 4 * S + s;
            J[0] = idP ? 1.0 : d00;
            J[S] = idP ? 0.0 : d01;
            J[2 * S] = idQ ? 0.0 : d10;
            J[3 * S] = idQ ? 1.0 : d11;
        }
        fmax = absMax(absMax(0.0, FP), FQ);
    }
    red[threadIdx.y][threadIdx.x] = fmax;
    __syncthreads();
    if (threadIdx.y == 0 && s < b.S) {
        double m = red[0][threadIdx.x];
        for (int k = 1; k < blockDim.y; k++) m = absMax(m, red[k][threadIdx.x]);
        if (b.active[s] && m != 0.0) atomicMax(&b.norm[s], (unsigned long long)__double_as_longlong(m));
    }
}

void launchFill(const DevNet& net, const DevBatch& b, bool withJacobian, bool withQbuf, cudaStream_t st) {
    dim3 block(32, 8);
    dim3 grid(b.S / 32, (net.nb + 7) / 8);
    if (withJacobian) {
        if (withQbuf) fillKernel<true, true><<<grid, block, 0, st>>>(net, b);
        else fillKernel<true, false><<<grid, block, 0, st>>>(net, b);
    } else {
        if (withQbuf) fillKernel<false, true><<<grid, block, 0, st>>>(net, b);
        else fillKernel<false, false><<<grid, block, 0, st>>>(net, b);
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Convergence test and retirement (newton_iteration.cu:276-397): >= 1 iteration; a test that passes at the budget
// is MAX_ITERATION_REACHED; a non-finite mismatch is DIVERGED.  A converged lane with reactive limits to check is
// marked pending instead (its outer loop decides).
// ---------------------------------------------------------------------------------------------------------------
// A lane whose solve failed: restarts from the fallback start when it still may (pending for this iteration, so it
// neither factorizes nor counts an iteration; the next iteration fills at the fallback state), else retires.
// The restart of a lane: its iteration count, trouble and scored ratio reset, pending for this iteration (it neither
// factorizes nor counts an iteration; the next iteration fills at the restored state).
__device__ void restartLane(const DevBatch& b, int s) {
    b.iter[s] = 0;
    b.trouble[s] = 0;
    b.pending[s] = 1;
    b.solveRatio[s] = 0.0;
}

// A lane whose solve failed: restarts from the fallback start when it still may; else, in mixed precision, restarts
// once with FP64 factorizations and solves from its start (the FP64 engine's trajectory for that scenario, so a
// scenario that fails does so as it does in FP64); else retires with the status.
__device__ void failLane(const DevBatch& b, int s, int status) {
    const size_t S = b.S;
    if (b.fallbackLeft[s]) {
        b.fallbackLeft[s] = 0;
        b.fellBack[s] = 1;
        restartLane(b, s);
        for (int r = 0; r < b.nFallback; r++) b.x[(size_t)r * S + s] = b.fallbackX[r];
        return;
    }
    if (b.fp64Left && b.fp64Left[s]) {
        b.fp64Left[s] = 0;
        b.precision64[s] = 1;
        restartLane(b, s);
        const int n = b.nFallback;
        if (b.restartFull) {
            for (int r = 0; r < n; r++) b.x[(size_t)r * S + s] = b.restartFull[(size_t)s * n + r];
        } else {
            for (int r = 0; r < n; r++) b.x[(size_t)r * S + s] = b.fallbackX[r];
        }
        return;
    }
    b.status[s] = status;
    b.active[s] = 0;
    atomicSub(b.nActive, 1);
}

// OLF's realistic-voltage check of a converged state (realistic_voltage_check.cu:23-44): a checked voltage row
// outside [minV, maxV] makes the state UNREALISTIC_STATE.
__device__ bool unrealisticState(const DevBatch& b, const Settings& cfg, int s) {
    if (!cfg.realistic || !b.vCheck) return false;
    const size_t S = b.S;
    for (int r = 0; r < b.nFallback; r++) {
        if (!b.vCheck[r]) continue;
        const double v = b.x[(size_t)r * S + s];
        if (v < cfg.minV || v > cfg.maxV) return true;
    }
    return false;
}

// A converged lane leaves the loop CONVERGED, or UNREALISTIC_STATE when the realistic-voltage band rejects it.
__device__ void retireConverged(const DevBatch& b, const Settings& cfg, int s) {
    b.status[s] = unrealisticState(b, cfg, s) ? ST_UNREALISTIC_STATE : ST_CONVERGED;
    b.active[s] = 0;
    atomicSub(b.nActive, 1);
}

__global__ void testKernel(DevBatch b, Settings cfg, int* remainingPv) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.S || !b.active[s]) return;
    const double nrm = __longlong_as_double((long long)b.norm[s]);
    b.norm[s] = 0ull;
    const int it = b.iter[s];
    b.normOut[s] = nrm;
    if (b.trouble[s]) {
        // the last factorization met a near-singular 2x2 pivot, or its solve failed the linear-solve guard: the lane
        // took no step (its iteration did not advance) and ends here
        failLane(b, s, ST_LINEAR_SOLVE_FAILED);
        return;
    }
    if (!isfinite(nrm)) {
        failLane(b, s, ST_DIVERGED);
        return;
    }
    bool converged;
    if (cfg.norm2Threshold > 0.0) {
        const size_t S = b.S;
        double ssq = 0.0;
        for (int k = 0; k < SSQ_STRANDS; k++) ssq += b.ssqPart[(size_t)k * S + s];
        converged = sqrt(ssq) < cfg.norm2Threshold;
    } else {
        converged = nrm < cfg.tol;
    }
    if (it > 0 && converged && it < cfg.maxIter) {
        if (cfg.polishBelow > 0.0 && b.fallbackLeft[s] && nrm > cfg.polishBelow && it + 1 < cfg.maxIter) {
            b.fallbackLeft[s] = 0;   // one more step from inside the tolerance ball (the lane has converged: no restart)
            return;
        }
        if ((cfg.reactiveLimits || cfg.distributedSlack) && b.outer[s] < cfg.maxOuter) {
            b.pending[s] = 1;
            if (remainingPv) remainingPv[s] = 0;
        } else {
            retireConverged(b, cfg, s);
        }
        return;
    }
    if (it == cfg.maxIter) {
        // a budget spent on a solve that did not solve its system is a reject (newton_iteration.cu:371-392)
        const bool badSolve = !(b.solveRatio[s] <= LIN_SOLVE_FAIL_RATIO);
        failLane(b, s, badSolve ? (cfg.batchOfOne ? ST_LINEAR_SOLVE_FAILED : ST_REJECTED) : ST_MAX_ITERATION_REACHED);
    }
}

// Per lane, the sum of squares of F over the rows of strand blockIdx.y * 8 + threadIdx.y (rows r = strand mod
// SSQ_STRANDS, in row order): 32 lanes x 8 strands per CTA.
__global__ void ssqKernel(DevNet net, DevBatch b) {
    const int s = blockIdx.x * 32 + threadIdx.x;
    const int k = blockIdx.y * 8 + threadIdx.y;
    const size_t S = b.S;
    if (s >= b.S || k >= SSQ_STRANDS || !b.active[s]) return;
    double acc = 0.0;
    for (int r = k; r < net.n; r += SSQ_STRANDS) {
        const double f = b.F[(size_t)r * S + s];
        acc += f * f;
    }
    b.ssqPart[(size_t)k * S + s] = acc;
}

void launchNorm2(const DevNet& net, const DevBatch& b, cudaStream_t st) {
    ssqKernel<<<dim3(b.S / 32, SSQ_STRANDS / 8), dim3(32, 8), 0, st>>>(net, b);
}

void launchTest(const DevNet&, const DevBatch& b, const Settings& cfg, int* remainingPv, cudaStream_t st) {
    testKernel<<<(b.S + 127) / 128, 128, 0, st>>>(b, cfg, remainingPv);
}

// ---------------------------------------------------------------------------------------------------------------
// Reactive-limit outer loop, local controllers (reactive_limits.cu:321-359) and the forced-PV election
// (reactive_limits.cu:417-448).  q = closed-branch flows on the V row + load Q.
// ---------------------------------------------------------------------------------------------------------------
__global__ void rlCheckKernel(DevBatch b, DevRl rl, Settings cfg) {
    const size_t S = b.S;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int s = (int)(tid % S);
    const int i = (int)(tid / S);
    if (i >= rl.nRl || !b.pending[s] || (b.dsRestart && b.dsRestart[s])) return;
    const size_t e = (size_t)i * S + s;
    rl.passSwitched[e] = 0;
    const int r = rl.voltageRow[i];
    const size_t ri = (size_t)r * S + s;
    if (b.mode[ri] == MODE_FIXED_VARIABLE && rl.limitType[e] == 0) {
        const double q = b.qbuf[ri] + rl.loadQ[i];
        if (q < rl.minQ[i] - cfg.rlTol) {
            rl.savedTarget[e] = b.target[ri];
            rl.savedMode[e] = b.mode[ri];
            b.mode[ri] = MODE_EQUATION;
            b.target[ri] = rl.minQ[i] - rl.loadQ[i];
            rl.limitType[e] = 1;
            rl.switchCount[e]++;
            rl.passSwitched[e] = 1;
        } else if (q > rl.maxQ[i] + cfg.rlTol) {
            rl.savedTarget[e] = b.target[ri];
            rl.savedMode[e] = b.mode[ri];
            b.mode[ri] = MODE_EQUATION;
            b.target[ri] = rl.maxQ[i] - rl.loadQ[i];
            rl.limitType[e] = 2;
            rl.switchCount[e]++;
            rl.passSwitched[e] = 1;
        } else {
            atomicAdd(&rl.remainingPv[s], 1);
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

__global__ void rlFinalizeKernel(DevBatch b, DevRl rl, Settings cfg) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.S || !b.pending[s] || (b.dsRestart && b.dsRestart[s])) return;
    const size_t S = b.S;
    if (rl.remainingPv[s] == 0) {
        int best = -1, bestId = 0x7fffffff;
        double bestV = -1.0, bestP = -1e300;
        for (int i = 0; i < rl.nRl; i++) {
            const size_t e = (size_t)i * S + s;
            if (rl.passSwitched[e] != 1) continue;
            const double v = rl.nomV[i];
            const double p = rl.pRow[i] >= 0 ? b.target[(size_t)rl.pRow[i] * S + s] : rl.staticP[i];
            const bool better = best < 0 || v > bestV || (v == bestV && (p > bestP || (p == bestP && rl.idRank[i] < bestId)));
            if (better) {
                best = i;
                bestV = v;
                bestP = p;
                bestId = rl.idRank[i];
            }
        }
        if (best >= 0) {
            const size_t e = (size_t)best * S + s;
            const size_t ri = (size_t)rl.voltageRow[best] * S + s;
            b.mode[ri] = rl.savedMode[e];
            b.target[ri] = rl.savedTarget[e];
            rl.limitType[e] = 0;
            rl.switchCount[e]--;
            rl.passSwitched[e] = 0;
        }
    }
    bool any = false;
    for (int i = 0; i < rl.nRl && !any; i++) any = rl.passSwitched[(size_t)i * S + s] != 0;
    if (any) {
        // restart the Newton solve at the new targets and modes (newton_iteration.cu:472-487)
        b.iter[s] = 0;
        b.outer[s]++;
    } else {
        b.pending[s] = 0;
        retireConverged(b, cfg, s);
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Distributed slack (DistributedSlackOuterLoop; distributed_slack.cu:211-616, the bus-level water-fill), one thread
// per lane that converged this iteration.  The slack bus's closed-branch P minus its target is the mismatch; above
// slackDistTol, every participant is reset to its base target and the whole amount (the mismatch plus what the
// participants had absorbed) is water-filled over them in proportion to their factors, each clamped to its bounds and
// the factors renormalised over the unsaturated ones, until less than P_RESIDUE_EPS is left.  Targets that moved by
// more than 0.9 P_RESIDUE_EPS in total make the lane re-solve (an outer iteration); an unplaced remainder above
// P_RESIDUE_EPS is a distribution failure (REJECTED when the request asks, else left on the slack).  A lane that does
// not re-solve goes on to the reactive-limit check, or retires.
// ---------------------------------------------------------------------------------------------------------------
__global__ void dsCheckKernel(DevBatch b, DevDs ds, Settings cfg) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.S || !b.pending[s]) return;
    const size_t S = b.S;
    const double mis = b.qbuf[(size_t)ds.slackRow * S + s] - ds.slackTargetP;
    bool moved = false;
    if (fabs(mis) > cfg.slackDistTol && fabs(mis) > P_RESIDUE_EPS) {
        double absorbed = 0.0;
        for (int i = 0; i < ds.nDs; i++) {
            const size_t idx = (size_t)ds.row[i] * S + s;
            absorbed += b.target[idx] - ds.baseTarget[i];
            ds.prevTarget[(size_t)i * S + s] = b.target[idx];
            b.target[idx] = ds.baseTarget[i];
        }
        double rem = mis + absorbed;
        for (int it = 0; it < ds.nDs && fabs(rem) > P_RESIDUE_EPS; it++) {
            double fsum = 0.0;
            for (int i = 0; i < ds.nDs; i++) {
                const double cum = b.target[(size_t)ds.row[i] * S + s] - ds.baseTarget[i];
                const bool sat = rem > 0 ? cum >= ds.maxDelta[i] : cum <= ds.minDelta[i];
                if (!sat) fsum += ds.factor[i];
            }
            if (fsum <= 0.0) break;   // every participant saturated: the rest stays at the slack
            double done = 0.0;
            for (int i = 0; i < ds.nDs; i++) {
                const size_t idx = (size_t)ds.row[i] * S + s;
                const double cum = b.target[idx] - ds.baseTarget[i];
                const bool sat = rem > 0 ? cum >= ds.maxDelta[i] : cum <= ds.minDelta[i];
                if (sat) continue;
                const double next = fmin(fmax(cum + rem * (ds.factor[i] / fsum), ds.minDelta[i]), ds.maxDelta[i]);
                if (next != cum) {
                    b.target[idx] = ds.baseTarget[i] + next;
                    done += next - cum;
                }
            }
            rem -= done;
        }
        double shift = 0.0;
        for (int i = 0; i < ds.nDs; i++)
            shift += fabs(b.target[(size_t)ds.row[i] * S + s] - ds.prevTarget[(size_t)i * S + s]);
        moved = shift > 0.9 * P_RESIDUE_EPS;
        ds.failed[s] = fabs(rem) > P_RESIDUE_EPS ? 1 : 0;
        if (ds.failed[s] && cfg.rejectDsFailure) {
            b.status[s] = ST_REJECTED;
            b.active[s] = 0;
            b.pending[s] = 0;
            atomicSub(b.nActive, 1);
            return;
        }
    }
    if (moved) {
        // re-solve at the new targets (newton_iteration.cu:472-487); still pending for this iteration
        b.iter[s] = 0;
        b.outer[s]++;
        b.dsRestart[s] = 1;
    } else if (!cfg.reactiveLimits) {
        b.pending[s] = 0;
        retireConverged(b, cfg, s);
    }
}

void launchDistributedSlack(const DevBatch& b, const DevDs& ds, const Settings& cfg, cudaStream_t st) {
    if (ds.nDs == 0) return;
    dsCheckKernel<<<(b.S + 127) / 128, 128, 0, st>>>(b, ds, cfg);
}

void launchReactiveLimits(const DevNet&, const DevBatch& b, const DevRl& rl, const Settings& cfg, cudaStream_t st) {
    if (rl.nRl == 0) return;
    const size_t threads = (size_t)rl.nRl * b.S;
    rlCheckKernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(b, rl, cfg);
    rlFinalizeKernel<<<(b.S + 127) / 128, 128, 0, st>>>(b, rl, cfg);
}

// ---------------------------------------------------------------------------------------------------------------
// Batched block LU, one level of tasks per launch: one thread per (LU block, lane).
//   U(k, j) = A(k, j) - sum_m L(k, m) U(m, j);    L(i, k) = (A(i, k) - sum_m L(i, m) U(m, k)) inv(D_k)
// with D_m = U(m, m), whose slot stores its inverse.  Deferred-L plan: the L blocks stay unscaled (L~) during the
// factorization and every update applies its pivot's inverse, L~(k, m) inv(D_m) U(m, j), so an L block does not wait
// for its own column's pivot (about one level per pivot instead of two); scaleLKernel finally turns every L~ into L.
// The updates come in ascending m (a fixed summation order).
// A near-singular 2x2 pivot (|det| <= 1e-13 of its terms, lu_pivot.cuh:12-18) flags the lane.
// ---------------------------------------------------------------------------------------------------------------
// Mixed precision: flags the lane for an FP64 refactor when an FP32 pivot block D (inverse det^-1 adj D) is badly
// conditioned (max|D| max|inv D|) or grew against its Jacobian block (max|D| / max|A_kk|) beyond growthLimit.
template <typename T>
__device__ __forceinline__ void pivotGrowth(const DevBatch& b, int s, T a00, T a01, T a10, T a11, T inv, T amax) {
    if (!b.precision64) return;     // a batch without per-lane precision flags (the allocation-free solve)
    const float dmax = fmaxf(fmaxf(fabsf((float)a00), fabsf((float)a01)), fmaxf(fabsf((float)a10), fabsf((float)a11)));
    const float imax = dmax * fabsf((float)inv);      // max |adj D| = max |D| for a 2x2 block
    const float kappa = dmax * imax;
    const float grow = amax > 0 ? dmax / (float)amax : 1.0f;
    if (!(kappa <= (float)b.growthLimit) || !(grow <= (float)b.growthLimit)) b.precision64[s] = 1;
}

template <typename T>
__device__ __forceinline__ void load4(const T* base, size_t blk, size_t S, int s, T& a, T& b_, T& c, T& d) {
    const T* p = base + blk * 4 * S + s;
    a = p[0];
    b_ = p[S];
    c = p[2 * S];
    d = p[3 * S];
}

template <typename T>
__device__ __forceinline__ void store4(T* base, size_t blk, size_t S, int s, T a, T b_, T c, T d) {
    T* p = base + blk * 4 * S + s;
    p[0] = a;
    p[S] = b_;
    p[2 * S] = c;
    p[3 * S] = d;
}

// Register cap of the factorization level kernels: blocks of 32 x max(4, P) threads, at least as many resident per SM
// as this many registers a thread allow.
#ifndef OLF_FACTOR_MAX_REGS
#define OLF_FACTOR_MAX_REGS 64
#endif

// Launch geometry of one level: P threads share each task (or row) of the level, splitting its update list P ways;
// blocks are 32 lanes x max(4, P) threads (4 rows measured 1.5 % faster than 8 on the 500-lane batch, 16 rows 5 %
// slower).  The P partial sums are added in a fixed order (part 0 first), so the result does not depend on
// scheduling.
template <int P>
struct Split {
    static constexpr int ROWS = P >= 4 ? P : 4;     // blockDim.y
    static constexpr int TPB = P >= 4 ? 1 : 4 / P;  // tasks per block
};

template <typename T, int P>
__global__ void __launch_bounds__(32 * Split<P>::ROWS, 65536 / (OLF_FACTOR_MAX_REGS * 32 * Split<P>::ROWS))
    factorLevelKernel(DevNet net, DevBatch b, T* lu, int first, int count) {
    constexpr int TPB = Split<P>::TPB, ROWS = Split<P>::ROWS;
    __shared__ T red[ROWS][4][32];
    const size_t S = b.S;
    const int lane = threadIdx.x, ty = threadIdx.y;
    const int tib = ty / P, part = ty % P;
    const int s = blockIdx.y * 32 + lane;
    const int k = blockIdx.x * TPB + tib;
    pdlTrigger();
    const bool ok = k < count && s < b.S && solving(b, s);
    T a00 = 0, a01 = 0, a10 = 0, a11 = 0, amax = 0;
    int t = 0;
    Task tk{};
    int4 op0 = make_int4(-1, -1, -1, 0);
    if (ok) {
        t = net.levelTask[first + k];
        tk = net.task[t];
        // before the wait: the Jacobian block (written by the fill, which precedes the factorization's launches) and
        // the thread's first update record (static); the LU blocks of earlier levels are read after it
        if (part == 0 && tk.aBlock >= 0) {
            const double* p = b.J + (size_t)tk.aBlock * 4 * S + s;
            a00 = (T)p[0];
            a01 = (T)p[S];
            a10 = (T)p[2 * S];
            a11 = (T)p[3 * S];
            amax = fmax(fmax(fabs(a00), fabs(a01)), fmax(fabs(a10), fabs(a11)));
        }
        if (tk.opBegin + part < tk.opEnd) op0 = net.ops[tk.opBegin + part];
    }
    pdlWait();   // the previous level's blocks are read from here on
    if (ok) {
#pragma unroll 4
        for (int q = tk.opBegin + part; q < tk.opEnd; q += P) {
            const int4 op = q == tk.opBegin + part ? op0 : net.ops[q];
            T m00, m01, m10, m11, u00, u01, u10, u11;
            load4(lu, (size_t)op.x, S, s, m00, m01, m10, m11);
            load4(lu, (size_t)op.y, S, s, u00, u01, u10, u11);
            if (op.z >= 0) {   // deferred-L plan: L~(a,m) inv(D_m)
                T d00, d01, d10, d11;
                load4(lu, (size_t)op.z, S, s, d00, d01, d10, d11);
                const T l00 = m00, l01 = m01, l10 = m10, l11 = m11;
                m00 = dot2(l00, d00, l01, d10);
                m01 = dot2(l00, d01, l01, d11);
                m10 = dot2(l10, d00, l11, d10);
                m11 = dot2(l10, d01, l11, d11);
            }
            a00 = rnSub(a00, dot2(m00, u00, m01, u10));
            a01 = rnSub(a01, dot2(m00, u01, m01, u11));
            a10 = rnSub(a10, dot2(m10, u00, m11, u10));
            a11 = rnSub(a11, dot2(m10, u01, m11, u11));
        }
    }
    if (P > 1) {
        red[ty][0][lane] = a00;
        red[ty][1][lane] = a01;
        red[ty][2][lane] = a10;
        red[ty][3][lane] = a11;
        __syncthreads();
        if (part == 0) {
            for (int q = 1; q < P; q++) {
                a00 += red[ty + q][0][lane];
                a01 += red[ty + q][1][lane];
                a10 += red[ty + q][2][lane];
                a11 += red[ty + q][3][lane];
            }
        }
    }
    if (!ok || part != 0) return;
    if (tk.diag == -2) {
        const T det = rnFma(a00, a11, -rnMul(a01, a10));
        const T scale = fabs(a00 * a11) + fabs(a01 * a10);
        if (!(fabs(det) > (T)1e-13 * scale) || !isfinite(det)) b.trouble[s] = 1;
        const T inv = (T)1 / det;
        if (sizeof(T) == 4) pivotGrowth(b, s, a00, a01, a10, a11, inv, amax);
        store4(lu, (size_t)t, S, s, a11 * inv, -a01 * inv, -a10 * inv, a00 * inv);
    } else if (tk.diag >= 0 && !net.deferredL) {
        // default plan: L(i,k) = (...) inv(D_k), the pivot inverted one level earlier
        T i00, i01, i10, i11;
        load4(lu, (size_t)tk.diag, S, s, i00, i01, i10, i11);
        store4(lu, (size_t)t, S, s, dot2(a00, i00, a01, i10), dot2(a00, i01, a01, i11), dot2(a10, i00, a11, i10),
               dot2(a10, i01, a11, i11));
    } else {
        store4(lu, (size_t)t, S, s, a00, a01, a10, a11);
    }
}

// The last pass of a factorization: L(i, k) = L~(i, k) inv(D_k) for every L block (ids nU .. nLu - 1).  One thread
// per (L block, lane): 32 lanes x 8 blocks per CTA.
template <typename T>
__global__ void scaleLKernel(DevNet net, DevBatch b, T* lu) {
    const size_t S = b.S;
    const int s = blockIdx.y * 32 + threadIdx.x;
    const int id = net.nU + blockIdx.x * 8 + threadIdx.y;
    if (id >= net.nLu || s >= b.S || !solving(b, s)) return;
    T a00, a01, a10, a11, i00, i01, i10, i11;
    load4(lu, (size_t)id, S, s, a00, a01, a10, a11);
    load4(lu, (size_t)net.task[id].diag, S, s, i00, i01, i10, i11);
    store4(lu, (size_t)id, S, s, dot2(a00, i00, a01, i10), dot2(a00, i01, a01, i11), dot2(a10, i00, a11, i10),
           dot2(a10, i01, a11, i11));
}

__global__ void clearTroubleKernel(DevBatch b) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < b.S && solving(b, s)) b.trouble[s] = 0;
}

// Launches a per-level kernel template with the level's split factor, as a programmatic dependent launch: its CTAs
// may start while the previous level finishes (every level kernel loads its index records, then waits in pdlWait
// for the previous grid before it touches factor or solution data).
template <typename... KArgs, typename... Args>
static void launchLevel(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

#define OLF_SPLIT_CASE(N, KERNEL, T_, ...)                                                             \
    case N: {                                                                                           \
        dim3 blk(32, Split<N>::ROWS), grd((count + Split<N>::TPB - 1) / Split<N>::TPB, b.S / 32);       \
        launchLevel(KERNEL<T_, N>, grd, blk, st, __VA_ARGS__);                                          \
        break;                                                                                          \
    }
#define OLF_SPLIT_DISPATCH(P_, KERNEL, T_, ...)                                                         \
    switch (P_) {                                                                                       \
        OLF_SPLIT_CASE(1, KERNEL, T_, __VA_ARGS__)                                                      \
        OLF_SPLIT_CASE(2, KERNEL, T_, __VA_ARGS__)                                                      \
        OLF_SPLIT_CASE(4, KERNEL, T_, __VA_ARGS__)                                                      \
        OLF_SPLIT_CASE(8, KERNEL, T_, __VA_ARGS__)                                                      \
        default: OLF_SPLIT_CASE(16, KERNEL, T_, __VA_ARGS__)                                            \
    }

// ---------------------------------------------------------------------------------------------------------------
// Subtree bins of the wide levels: one CTA per (bin, 32 lanes), 8 warps; the bin's levels in order with a CTA barrier
// between them.  In a level with fewer tasks than warps, P warps share a task (its updates split P ways, partial sums
// added in part order through shared memory), as the level kernels' split does.  Every barrier sits in control flow
// that is uniform over the CTA (bin, level and round counts are the same for all its threads).
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ int binSplit(int cnt) {
    int P = 1;
    while (P < 8 && cnt * P * 2 <= 8) P *= 2;
    return P;
}

template <typename T>
__global__ void __launch_bounds__(256) subtreeFactorKernel(DevNet net, DevBatch b, T* lu, SubtreePlan sp, int binBase) {
    __shared__ T red[8][4][32];
    const size_t S = b.S;
    const int lane = threadIdx.x, warp = threadIdx.y;
    const int s = blockIdx.y * 32 + lane;
    const bool ok = s < b.S && solving(b, s);
    const int bin = binBase + blockIdx.x;
    const int v0 = sp.levPtr[bin], v1 = sp.levPtr[bin + 1];
    for (int v = v0; v < v1; v++) {
        const int first = sp.levOff[v], cnt = sp.levOff[v + 1] - first;
        const int P = binSplit(cnt), per = 8 / P, part = warp % P, slot = warp / P;
        for (int base = 0; base < cnt; base += per) {
            const int k = base + slot;
            const bool has = ok && k < cnt;
            T a00 = 0, a01 = 0, a10 = 0, a11 = 0, amax = 0;
            int t = 0;
            Task tk{};
            if (has) {
                t = sp.task[first + k];
                tk = net.task[t];
                if (part == 0 && tk.aBlock >= 0) {
                    const double* pa = b.J + (size_t)tk.aBlock * 4 * S + s;
                    a00 = (T)pa[0];
                    a01 = (T)pa[S];
                    a10 = (T)pa[2 * S];
                    a11 = (T)pa[3 * S];
                    amax = fmax(fmax(fabs(a00), fabs(a01)), fmax(fabs(a10), fabs(a11)));
                }
#pragma unroll 4
                for (int q = tk.opBegin + part; q < tk.opEnd; q += P) {
                    const int4 op = net.ops[q];
                    T m00, m01, m10, m11, u00, u01, u10, u11;
                    load4(lu, (size_t)op.x, S, s, m00, m01, m10, m11);
                    load4(lu, (size_t)op.y, S, s, u00, u01, u10, u11);
                    a00 -= m00 * u00 + m01 * u10;
                    a01 -= m00 * u01 + m01 * u11;
                    a10 -= m10 * u00 + m11 * u10;
                    a11 -= m10 * u01 + m11 * u11;
                }
            }
            if (P > 1) {
                red[warp][0][lane] = a00;
                red[warp][1][lane] = a01;
                red[warp][2][lane] = a10;
                red[warp][3][lane] = a11;
                __syncthreads();
                if (part == 0) {
                    for (int q = 1; q < P; q++) {
                        a00 += red[warp + q][0][lane];
                        a01 += red[warp + q][1][lane];
                        a10 += red[warp + q][2][lane];
                        a11 += red[warp + q][3][lane];
                    }
                }
                __syncthreads();
            }
            if (!has || part != 0) continue;
            if (tk.diag == -2) {
                const T det = rnFma(a00, a11, -rnMul(a01, a10));
                const T scale = fabs(a00 * a11) + fabs(a01 * a10);
                if (!(fabs(det) > (T)1e-13 * scale) || !isfinite(det)) b.trouble[s] = TROUBLE_PIVOT;
                const T inv = (T)1 / det;
                if (sizeof(T) == 4) pivotGrowth(b, s, a00, a01, a10, a11, inv, amax);
                store4(lu, (size_t)t, S, s, a11 * inv, -a01 * inv, -a10 * inv, a00 * inv);
            } else if (tk.diag >= 0) {
                T i00, i01, i10, i11;
                load4(lu, (size_t)tk.diag, S, s, i00, i01, i10, i11);
                store4(lu, (size_t)t, S, s, a00 * i00 + a01 * i10, a00 * i01 + a01 * i11, a10 * i00 + a11 * i10,
                       a10 * i01 + a11 * i11);
            } else {
                store4(lu, (size_t)t, S, s, a00, a01, a10, a11);
            }
        }
        __syncthreads();   // this level's blocks are written before the next level reads them
    }
}

// The bins' forward (DIR 0: w_i -= L(i,j) w_j over the bin's positions from the leaves up) or backward sweep (DIR 1:
// w_i = inv(D_i) (w_i - U(i,j) w_j) from the bins' roots down; every ancestor outside the bin is final before).
template <typename T, int DIR>
__global__ void __launch_bounds__(256) subtreeSolveKernel(DevNet net, DevBatch b, const T* lu, T* w, SubtreePlan sp,
                                                           int binBase) {
    __shared__ T red[8][2][32];
    const size_t S = b.S;
    const int lane = threadIdx.x, warp = threadIdx.y;
    const int s = blockIdx.y * 32 + lane;
    const bool ok = s < b.S && solving(b, s);
    const int* ptr = DIR == 0 ? sp.fwdPtr : sp.bwdPtr;
    const int* off = DIR == 0 ? sp.fwdOff : sp.bwdOff;
    const int* pos = DIR == 0 ? sp.fwdPos : sp.bwdPos;
    const int v0 = ptr[binBase + blockIdx.x], v1 = ptr[binBase + blockIdx.x + 1];
    for (int v = v0; v < v1; v++) {
        const int first = off[v], cnt = off[v + 1] - first;
        const int P = binSplit(cnt), per = 8 / P, part = warp % P, slot = warp / P;
        for (int base = 0; base < cnt; base += per) {
            const int k = base + slot;
            const bool has = ok && k < cnt;
            T w0 = 0, w1 = 0;
            int i = 0, d = 0;
            if (has) {
                i = pos[first + k];
                if (part == 0) {
                    w0 = w[(2 * (size_t)i) * S + s];
                    w1 = w[(2 * (size_t)i + 1) * S + s];
                }
                if (DIR == 0) {
                    const int q1 = net.lrowEnd[i];
                    for (int q = net.lrowPtr[i] + part; q < q1; q += P) {
                        const int2 e = net.lrow[q];
                        T l00, l01, l10, l11;
                        load4(lu, (size_t)e.x, S, s, l00, l01, l10, l11);
                        const T y0 = w[(2 * (size_t)e.y) * S + s], y1 = w[(2 * (size_t)e.y + 1) * S + s];
                        w0 -= l00 * y0 + l01 * y1;
                        w1 -= l10 * y0 + l11 * y1;
                    }
                } else {
                    d = net.uPtr[i];
                    const int q1 = net.uPtr[i + 1];
                    for (int q = d + 1 + part; q < q1; q += P) {
                        const int j = net.uCol[q];
                        T u00, u01, u10, u11;
                        load4(lu, (size_t)q, S, s, u00, u01, u10, u11);
                        const T x0 = w[(2 * (size_t)j) * S + s], x1 = w[(2 * (size_t)j + 1) * S + s];
                        w0 -= u00 * x0 + u01 * x1;
                        w1 -= u10 * x0 + u11 * x1;
                    }
                }
            }
            if (P > 1) {
                red[warp][0][lane] = w0;
                red[warp][1][lane] = w1;
                __syncthreads();
                if (part == 0) {
                    for (int q = 1; q < P; q++) {
                        w0 += red[warp + q][0][lane];
                        w1 += red[warp + q][1][lane];
                    }
                }
                __syncthreads();
            }
            if (!has || part != 0) continue;
            if (DIR == 0) {
                w[(2 * (size_t)i) * S + s] = w0;
                w[(2 * (size_t)i + 1) * S + s] = w1;
            } else {
                T i00, i01, i10, i11;
                load4(lu, (size_t)d, S, s, i00, i01, i10, i11);
                w[(2 * (size_t)i) * S + s] = i00 * w0 + i01 * w1;
                w[(2 * (size_t)i + 1) * S + s] = i10 * w0 + i11 * w1;
            }
        }
        __syncthreads();   // this level's entries are final before the next level reads them
    }
}

// One launch per phase: the factorization and the forward sweep in phase order, the backward sweep in reverse.
void launchSubtreeFactor(const DevNet& net, const DevBatch& b, const SubtreePlan& sp, bool fp32, cudaStream_t st) {
    for (int f = 0; f < sp.nPhases; f++) {
        const int b0 = sp.phasePtr[f], nb = sp.phasePtr[f + 1] - b0;
        if (nb <= 0) continue;
        dim3 grid(nb, b.S / 32), block(32, 8);
        if (fp32) subtreeFactorKernel<float><<<grid, block, 0, st>>>(net, b, b.lu32, sp, b0);
        else subtreeFactorKernel<double><<<grid, block, 0, st>>>(net, b, b.lu64, sp, b0);
    }
}

void launchSubtreeSolve(const DevNet& net, const DevBatch& b, const SubtreePlan& sp, bool fp32, int dir,
                        cudaStream_t st) {
    const int nPhases = dir == 0 ? sp.nFwdPhases : sp.nBwdPhases;
    const int* phasePtr = dir == 0 ? sp.fwdPhasePtr : sp.bwdPhasePtr;
    for (int k = 0; k < nPhases; k++) {
        const int f = dir == 0 ? k : nPhases - 1 - k;
        const int b0 = phasePtr[f], nb = phasePtr[f + 1] - b0;
        if (nb <= 0) continue;
        dim3 grid(nb, b.S / 32), block(32, 8);
        if (fp32) {
            if (dir == 0) subtreeSolveKernel<float, 0><<<grid, block, 0, st>>>(net, b, b.lu32, b.w32, sp, b0);
            else subtreeSolveKernel<float, 1><<<grid, block, 0, st>>>(net, b, b.lu32, b.w32, sp, b0);
        } else {
            if (dir == 0) subtreeSolveKernel<double, 0><<<grid, block, 0, st>>>(net, b, b.lu64, b.w64, sp, b0);
            else subtreeSolveKernel<double, 1><<<grid, block, 0, st>>>(net, b, b.lu64, b.w64, sp, b0);
        }
    }
}

void launchFactor(const DevNet& net, const DevBatch& b, const int* levelPtr, const int* levelSplit, int nLevels,
                  bool fp32, const Hybrid* hybrid, cudaStream_t st) {
    clearTroubleKernel<<<(b.S + 127) / 128, 128, 0, st>>>(b);
    const bool region = hybrid && hybrid->regionSlots > 0;
    const bool range = hybrid && !region && hybrid->lanes > 0;
    const int wide = region ? hybrid->regionFrom : range ? hybrid->factorFrom : nLevels;
    // subtree bins: one launch for the bins, then the wide levels' top tasks only
    const SubtreePlan* sub = hybrid && hybrid->sub && hybrid->sub->nBins > 0 ? hybrid->sub : nullptr;
    DevNet top = net;
    if (sub) {
        launchSubtreeFactor(net, b, *sub, fp32, st);
        top.levelTask = sub->topLevelTask;
    }
    for (int l = 0; l < wide; l++) {
        const int* ptr = sub ? sub->topLevelPtr : levelPtr;
        const int split = sub ? sub->topLevelSplit[l] : levelSplit[l];
        const int first = ptr[l], count = ptr[l + 1] - ptr[l];
        if (count == 0) continue;
        if (fp32) {
            OLF_SPLIT_DISPATCH(split, factorLevelKernel, float, top, b, b.lu32, first, count)
        } else {
            OLF_SPLIT_DISPATCH(split, factorLevelKernel, double, top, b, b.lu64, first, count)
        }
    }
    if (region || range) {
        // the range kernel ends with the L scaling pass of its tiles (a deferred-L plan has no front and no region)
        if (region) launchRegionFactor(net, b, *hybrid, fp32, st);
        else launchFactorRange(net, b, hybrid->plan, wide, hybrid->factorTo, hybrid->lanes, fp32, st);
        for (int l = hybrid->factorTo; l < nLevels; l++) {
            const int first = levelPtr[l], count = levelPtr[l + 1] - levelPtr[l];
            if (count == 0) continue;
            if (fp32) {
                OLF_SPLIT_DISPATCH(levelSplit[l], factorLevelKernel, float, net, b, b.lu32, first, count)
            } else {
                OLF_SPLIT_DISPATCH(levelSplit[l], factorLevelKernel, double, net, b, b.lu64, first, count)
            }
        }
    } else if (net.deferredL) {
        const int nL = net.nLu - net.nU;
        dim3 blk(32, 8), grd((nL + 7) / 8, b.S / 32);
        if (fp32) {
            scaleLKernel<float><<<grd, blk, 0, st>>>(net, b, b.lu32);
        } else {
            scaleLKernel<double><<<grd, blk, 0, st>>>(net, b, b.lu64);
        }
    }
    launchDenseFront(net, b, fp32, st);   // after every level (a dense-front plan is never deferred-L)
}

// ---------------------------------------------------------------------------------------------------------------
// Triangular solves on the block factors, level by level; one thread per (position, lane).
// ---------------------------------------------------------------------------------------------------------------
template <typename T>
__global__ void rhsKernel(DevNet net, DevBatch b, T* w, bool fromResidual) {
    const size_t S = b.S;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int s = (int)(tid % S);
    const int i = (int)(tid / S);
    if (i >= net.nb || !solving(b, s)) return;
    const int node = net.perm[i];
    const int cP = net.nodeCol[2 * node], cV = net.nodeCol[2 * node + 1];
    if (fromResidual) {
        w[(2 * (size_t)i) * S + s] = (T)b.res[cP * S + s];
        w[(2 * (size_t)i + 1) * S + s] = (T)b.res[cV * S + s];
    } else {
        w[(2 * (size_t)i) * S + s] = (T)(-b.F[cP * S + s]);
        w[(2 * (size_t)i + 1) * S + s] = (T)(-b.F[cV * S + s]);
    }
}

template <typename T, int P>
__global__ void __launch_bounds__(1024) forwardLevelKernel(DevNet net, DevBatch b, const T* lu, T* w, const int* pos,
                                                           int first, int count) {
    constexpr int TPB = Split<P>::TPB, ROWS = Split<P>::ROWS;
    __shared__ T red[ROWS][2][32];
    const size_t S = b.S;
    const int lane = threadIdx.x, ty = threadIdx.y;
    const int tib = ty / P, part = ty % P;
    const int s = blockIdx.y * 32 + lane;
    const int k = blockIdx.x * TPB + tib;
    pdlTrigger();
    const bool ok = k < count && s < b.S && solving(b, s);
    T w0 = 0, w1 = 0;
    int i = 0, q0 = 0, q1 = 0;
    // the thread's first two L blocks, read before the wait: the factors are final for the whole solve (its first
    // kernel is a normal launch after the factorization) and only the solution entries depend on earlier levels
    int2 e0 = make_int2(0, -1), e1 = make_int2(0, -1);
    T a00 = 0, a01 = 0, a10 = 0, a11 = 0, c00 = 0, c01 = 0, c10 = 0, c11 = 0;
    if (ok) {
        i = pos[first + k];
        q0 = net.lrowPtr[i] + part;
        q1 = net.lrowEnd[i];
        if (q0 < q1) {
            e0 = net.lrow[q0];
            load4(lu, (size_t)e0.x, S, s, a00, a01, a10, a11);
        }
        if (q0 + P < q1) {
            e1 = net.lrow[q0 + P];
            load4(lu, (size_t)e1.x, S, s, c00, c01, c10, c11);
        }
    }
    pdlWait();   // the previous level's solution entries are read from here on
    if (ok) {
        if (part == 0) {
            w0 = w[(2 * (size_t)i) * S + s];
            w1 = w[(2 * (size_t)i + 1) * S + s];
        }
        if (e0.y >= 0) {
            const T y0 = w[(2 * (size_t)e0.y) * S + s], y1 = w[(2 * (size_t)e0.y + 1) * S + s];
            w0 = rnSub(w0, dot2(a00, y0, a01, y1));
            w1 = rnSub(w1, dot2(a10, y0, a11, y1));
        }
        if (e1.y >= 0) {
            const T y0 = w[(2 * (size_t)e1.y) * S + s], y1 = w[(2 * (size_t)e1.y + 1) * S + s];
            w0 = rnSub(w0, dot2(c00, y0, c01, y1));
            w1 = rnSub(w1, dot2(c10, y0, c11, y1));
        }
#pragma unroll 4
        for (int q = q0 + 2 * P; q < q1; q += P) {
            const int2 e = net.lrow[q];
            T l00, l01, l10, l11;
            load4(lu, (size_t)e.x, S, s, l00, l01, l10, l11);
            const T y0 = w[(2 * (size_t)e.y) * S + s], y1 = w[(2 * (size_t)e.y + 1) * S + s];
            w0 = rnSub(w0, dot2(l00, y0, l01, y1));
            w1 = rnSub(w1, dot2(l10, y0, l11, y1));
        }
    }
    if (P > 1) {
        red[ty][0][lane] = w0;
        red[ty][1][lane] = w1;
        __syncthreads();
        if (part == 0) {
            for (int q = 1; q < P; q++) {
                w0 += red[ty + q][0][lane];
                w1 += red[ty + q][1][lane];
            }
        }
    }
    if (!ok || part != 0) return;
    w[(2 * (size_t)i) * S + s] = w0;
    w[(2 * (size_t)i + 1) * S + s] = w1;
}

template <typename T, int P>
__global__ void __launch_bounds__(1024) backwardLevelKernel(DevNet net, DevBatch b, const T* lu, T* w, const int* pos,
                                                            int first, int count) {
    constexpr int TPB = Split<P>::TPB, ROWS = Split<P>::ROWS;
    __shared__ T red[ROWS][2][32];
    const size_t S = b.S;
    const int lane = threadIdx.x, ty = threadIdx.y;
    const int tib = ty / P, part = ty % P;
    const int s = blockIdx.y * 32 + lane;
    const int k = blockIdx.x * TPB + tib;
    pdlTrigger();
    const bool ok = k < count && s < b.S && solving(b, s);
    T w0 = 0, w1 = 0;
    int i = 0, d = 0, q1 = 0;
    // the pivot inverse and the thread's first two U blocks, read before the wait (the factors are final for the
    // whole solve; only the solution entries depend on earlier levels)
    int j0 = -1, j1 = -1;
    T i00 = 0, i01 = 0, i10 = 0, i11 = 0;
    T a00 = 0, a01 = 0, a10 = 0, a11 = 0, c00 = 0, c01 = 0, c10 = 0, c11 = 0;
    if (ok) {
        i = pos[first + k];
        d = net.uPtr[i];
        q1 = net.uPtr[i + 1];
        if (part == 0) load4(lu, (size_t)d, S, s, i00, i01, i10, i11);
        const int qa = d + 1 + part;
        if (qa < q1) {
            j0 = net.uCol[qa];
            load4(lu, (size_t)qa, S, s, a00, a01, a10, a11);
        }
        if (qa + P < q1) {
            j1 = net.uCol[qa + P];
            load4(lu, (size_t)(qa + P), S, s, c00, c01, c10, c11);
        }
    }
    pdlWait();   // the previous level's solution entries are read from here on
    if (ok) {
        if (part == 0) {
            w0 = w[(2 * (size_t)i) * S + s];
            w1 = w[(2 * (size_t)i + 1) * S + s];
        }
        if (j0 >= 0) {
            const T x0 = w[(2 * (size_t)j0) * S + s], x1 = w[(2 * (size_t)j0 + 1) * S + s];
            w0 = rnSub(w0, dot2(a00, x0, a01, x1));
            w1 = rnSub(w1, dot2(a10, x0, a11, x1));
        }
        if (j1 >= 0) {
            const T x0 = w[(2 * (size_t)j1) * S + s], x1 = w[(2 * (size_t)j1 + 1) * S + s];
            w0 = rnSub(w0, dot2(c00, x0, c01, x1));
            w1 = rnSub(w1, dot2(c10, x0, c11, x1));
        }
#pragma unroll 4
        for (int q = d + 1 + part + 2 * P; q < q1; q += P) {
            const int j = net.uCol[q];
            T u00, u01, u10, u11;
            load4(lu, (size_t)q, S, s, u00, u01, u10, u11);
            const T x0 = w[(2 * (size_t)j) * S + s], x1 = w[(2 * (size_t)j + 1) * S + s];
            w0 = rnSub(w0, dot2(u00, x0, u01, x1));
            w1 = rnSub(w1, dot2(u10, x0, u11, x1));
        }
    }
    if (P > 1) {
        red[ty][0][lane] = w0;
        red[ty][1][lane] = w1;
        __syncthreads();
        if (part == 0) {
            for (int q = 1; q < P; q++) {
                w0 += red[ty + q][0][lane];
                w1 += red[ty + q][1][lane];
            }
        }
    }
    if (!ok || part != 0) return;
    w[(2 * (size_t)i) * S + s] = dot2(i00, w0, i01, w1);
    w[(2 * (size_t)i + 1) * S + s] = dot2(i10, w0, i11, w1);
}

template <typename T>
__global__ void scatterKernel(DevNet net, DevBatch b, const T* w, bool accumulate) {
    const size_t S = b.S;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int s = (int)(tid % S);
    const int node = (int)(tid / S);
    if (node >= net.nb || !solving(b, s)) return;
    const int i = net.iperm[node];
    const int cP = net.nodeCol[2 * node], cV = net.nodeCol[2 * node + 1];
    const double d0 = (double)w[(2 * (size_t)i) * S + s], d1 = (double)w[(2 * (size_t)i + 1) * S + s];
    if (accumulate) {
        // a refinement correction: dx += d, and d kept in res for the correction check
        b.dx[cP * S + s] += d0;
        b.dx[cV * S + s] += d1;
        b.res[cP * S + s] = d0;
        b.res[cV * S + s] = d1;
    } else {
        b.dx[cP * S + s] = d0;
        b.dx[cV * S + s] = d1;
    }
}

template <typename T>
static void solveT(const DevNet& net, const DevBatch& b, T* w, const T* lu, const LevelSchedule& fwd,
                   const LevelSchedule& bwd, bool fromResidual, const Hybrid* hybrid, cudaStream_t st) {
    const size_t all = (size_t)net.nb * b.S;
    const bool fp32 = sizeof(T) == 4;
    rhsKernel<T><<<(unsigned)((all + 255) / 256), 256, 0, st>>>(net, b, w, fromResidual);
    const bool region = hybrid && hybrid->solveRegion;   // the narrow levels in shared memory, one CTA per lane
    // subtree bins: the bins' forward sweep first and their backward sweep last; the wide levels run their top
    // positions only
    const SubtreePlan* sub = hybrid && hybrid->sub && hybrid->sub->nBins > 0 ? hybrid->sub : nullptr;
    if (!region && hybrid && hybrid->lanes <= 0) hybrid = nullptr;   // no range launches in the solves
    const LevelSchedule fwdTop = sub ? LevelSchedule{fwd.levels, sub->topFwdPtr, sub->topFwdPos, sub->topFwdSplit} : fwd;
    const LevelSchedule bwdTop = sub ? LevelSchedule{bwd.levels, sub->topBwdPtr, sub->topBwdPos, sub->topBwdSplit} : bwd;
    auto forwardLevels = [&](const LevelSchedule& ls, int l0, int l1) {
        for (int l = l0; l < l1; l++) {
            const int first = ls.ptr[l], count = ls.ptr[l + 1] - ls.ptr[l];
            if (count == 0) continue;
            OLF_SPLIT_DISPATCH(ls.split[l], forwardLevelKernel, T, net, b, lu, w, ls.pos, first, count)
        }
    };
    auto backwardLevels = [&](const LevelSchedule& ls, int l0, int l1) {
        for (int l = l0; l < l1; l++) {
            const int first = ls.ptr[l], count = ls.ptr[l + 1] - ls.ptr[l];
            if (count == 0) continue;
            OLF_SPLIT_DISPATCH(ls.split[l], backwardLevelKernel, T, net, b, lu, w, ls.pos, first, count)
        }
    };
    if (sub) launchSubtreeSolve(net, b, *sub, sizeof(T) == 4, 0, st);
    const int fwdWide = hybrid ? hybrid->fwdFrom : fwd.levels;
    forwardLevels(fwdTop, 0, fwdWide);
    if (region && hybrid->fwdRegionSlots > 0) launchSolveRegion(net, b, *hybrid, fp32, 0, st);
    else if (region) forwardLevels(fwd, fwdWide, fwd.levels);
    else if (hybrid) launchSolveRange(net, b, hybrid->plan, 0, fwdWide, fwd.levels, hybrid->lanes, fp32, st);
    else if (sub) forwardLevels(fwdTop, fwdWide, fwd.levels);
    launchDenseFrontSolve(net, b, fp32, st);   // dense-front plans: the front rows, forward then backward
    const int bwdNarrow = hybrid ? hybrid->bwdUntil : 0;
    if (region && hybrid->bwdRegionSlots > 0) launchSolveRegion(net, b, *hybrid, fp32, 1, st);
    else if (region) backwardLevels(bwd, 0, bwdNarrow);
    else if (hybrid) launchSolveRange(net, b, hybrid->plan, 1, 0, bwdNarrow, hybrid->lanes, fp32, st);
    backwardLevels(bwdTop, bwdNarrow, bwd.levels);
    if (sub) launchSubtreeSolve(net, b, *sub, sizeof(T) == 4, 1, st);
    scatterKernel<T><<<(unsigned)((all + 255) / 256), 256, 0, st>>>(net, b, w, fromResidual);
}

void launchSolve(const DevNet& net, const DevBatch& b, const LevelSchedule& fwd, const LevelSchedule& bwd, bool fp32,
                 bool fromResidual, const Hybrid* hybrid, cudaStream_t st) {
    if (fp32) solveT<float>(net, b, b.w32, b.lu32, fwd, bwd, fromResidual, hybrid, st);
    else solveT<double>(net, b, b.w64, b.lu64, fwd, bwd, fromResidual, hybrid, st);
}

// ---------------------------------------------------------------------------------------------------------------
// Transposed solve J^T y = c on the same block factors (transposed_solve.cuh:1-30): the plain solve's operations
// transposed, in reverse order.  With P J P^T = L U (L unit lower, U upper with the pivot blocks D, whose slots hold
// inv(D)): U^T y' = c' forward, row i: y'_i = inv(D_i)^T (c'_i - sum_k U(k, i)^T y'_k) over the L pattern of row i;
// then L^T z = y' backward, row i: z_i = y'_i - sum_j L(j, i)^T z_j over the U pattern of row i.  The level schedules
// of the plain sweeps serve (the patterns coincide); a dense front's positions (the last frontF of the order) run in
// order, one thread per lane, after the forward levels and before the backward ones.
// ---------------------------------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void upperTransposedRow(const DevNet& net, const T* lu, T* w, int i, size_t S, int s) {
    T w0 = w[(2 * (size_t)i) * S + s], w1 = w[(2 * (size_t)i + 1) * S + s];
    for (int q = net.lrowPtr[i]; q < net.lrowPtr[i + 1]; q++) {
        const int k = net.lrow[q].y;
        T u00, u01, u10, u11;
        load4(lu, (size_t)net.lrowU[q], S, s, u00, u01, u10, u11);
        const T y0 = w[(2 * (size_t)k) * S + s], y1 = w[(2 * (size_t)k + 1) * S + s];
        w0 -= u00 * y0 + u10 * y1;
        w1 -= u01 * y0 + u11 * y1;
    }
    T i00, i01, i10, i11;
    load4(lu, (size_t)net.uPtr[i], S, s, i00, i01, i10, i11);
    w[(2 * (size_t)i) * S + s] = i00 * w0 + i10 * w1;
    w[(2 * (size_t)i + 1) * S + s] = i01 * w0 + i11 * w1;
}

template <typename T>
__device__ __forceinline__ void lowerTransposedRow(const DevNet& net, const T* lu, T* w, int i, size_t S, int s) {
    T w0 = w[(2 * (size_t)i) * S + s], w1 = w[(2 * (size_t)i + 1) * S + s];
    for (int q = net.uPtr[i] + 1; q < net.uPtr[i + 1]; q++) {
        const int j = net.uCol[q];
        T l00, l01, l10, l11;
        load4(lu, (size_t)net.uRowL[q], S, s, l00, l01, l10, l11);
        const T z0 = w[(2 * (size_t)j) * S + s], z1 = w[(2 * (size_t)j + 1) * S + s];
        w0 -= l00 * z0 + l10 * z1;
        w1 -= l01 * z0 + l11 * z1;
    }
    w[(2 * (size_t)i) * S + s] = w0;
    w[(2 * (size_t)i + 1) * S + s] = w1;
}

// one level of a transposed sweep: 8 rows x 32 lanes per CTA (DIR 0: U^T forward, 1: L^T backward); front rows skipped
template <typename T, int DIR>
__global__ void transposedLevelKernel(DevNet net, DevBatch b, const T* lu, T* w, const int* pos, int first, int count) {
    const int k = blockIdx.x * 8 + threadIdx.y;
    const int s = blockIdx.y * 32 + threadIdx.x;
    if (k >= count || s >= b.S || !solving(b, s)) return;
    const int i = pos[first + k];
    if (net.frontF > 0 && i >= net.frontStart) return;
    if (DIR == 0) upperTransposedRow(net, lu, w, i, b.S, s);
    else lowerTransposedRow(net, lu, w, i, b.S, s);
}

// the dense front's rows in order, one thread per lane (DIR 0: ascending U^T rows, 1: descending L^T rows)
template <typename T, int DIR>
__global__ void transposedFrontKernel(DevNet net, DevBatch b, const T* lu, T* w) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.S || !solving(b, s)) return;
    for (int r = 0; r < net.frontF; r++) {
        const int i = DIR == 0 ? net.frontStart + r : net.nb - 1 - r;
        if (DIR == 0) upperTransposedRow(net, lu, w, i, b.S, s);
        else lowerTransposedRow(net, lu, w, i, b.S, s);
    }
}

template <typename T>
static void solveTransposedT(const DevNet& net, const DevBatch& b, T* w, const T* lu, const LevelSchedule& fwd,
                             const LevelSchedule& bwd, cudaStream_t st) {
    const size_t all = (size_t)net.nb * b.S;
    rhsKernel<T><<<(unsigned)((all + 255) / 256), 256, 0, st>>>(net, b, w, true);
    dim3 blk(32, 8);
    for (int l = 0; l < fwd.levels; l++) {
        const int first = fwd.ptr[l], count = fwd.ptr[l + 1] - first;
        if (count > 0) transposedLevelKernel<T, 0><<<dim3((count + 7) / 8, b.S / 32), blk, 0, st>>>(net, b, lu, w, fwd.pos, first, count);
    }
    if (net.frontF > 0) {
        transposedFrontKernel<T, 0><<<b.S / 32, 32, 0, st>>>(net, b, lu, w);
        transposedFrontKernel<T, 1><<<b.S / 32, 32, 0, st>>>(net, b, lu, w);
    }
    for (int l = 0; l < bwd.levels; l++) {
        const int first = bwd.ptr[l], count = bwd.ptr[l + 1] - first;
        if (count > 0) transposedLevelKernel<T, 1><<<dim3((count + 7) / 8, b.S / 32), blk, 0, st>>>(net, b, lu, w, bwd.pos, first, count);
    }
    scatterKernel<T><<<(unsigned)((all + 255) / 256), 256, 0, st>>>(net, b, w, false);
}

void launchSolveTransposed(const DevNet& net, const DevBatch& b, const LevelSchedule& fwd, const LevelSchedule& bwd,
                           bool fp32, cudaStream_t st) {
    if (fp32) solveTransposedT<float>(net, b, b.w32, b.lu32, fwd, bwd, st);
    else solveTransposedT<double>(net, b, b.w64, b.lu64, fwd, bwd, st);
}

// ---------------------------------------------------------------------------------------------------------------
// FP64 refinement residual r = -F - J dx, one thread per (bus, lane), J in its block rows.
// ---------------------------------------------------------------------------------------------------------------
__global__ void residualKernel(DevNet net, DevBatch b) {
    const size_t S = b.S;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int s = (int)(tid % S);
    const int node = (int)(tid / S);
    if (node >= net.nb || !solving(b, s)) return;
    const int cP = net.nodeCol[2 * node], cV = net.nodeCol[2 * node + 1];
    double r0 = -b.F[cP * S + s], r1 = -b.F[cV * S + s];
    for (int t = net.aPtr[node]; t < net.aPtr[node + 1]; t++) {
        const int j = net.aCol[t];
        const double* J = b.J + (size_t)t * 4 * S + s;
        const double x0 = b.dx[(size_t)net.nodeCol[2 * j] * S + s], x1 = b.dx[(size_t)net.nodeCol[2 * j + 1] * S + s];
        r0 -= J[0] * x0 + J[S] * x1;
        r1 -= J[2 * S] * x0 + J[3 * S] * x1;
    }
    b.res[cP * S + s] = r0;
    b.res[cV * S + s] = r1;
}

void launchResidual(const DevNet& net, const DevBatch& b, cudaStream_t st) {
    const size_t all = (size_t)net.nb * b.S;
    residualKernel<<<(unsigned)((all + 255) / 256), 256, 0, st>>>(net, b);
}

// ---------------------------------------------------------------------------------------------------------------
// Newton step for the lanes that solved this iteration: x += dx (state_vector_scaling.cu:48-51, plain NR), or
// x += f dx with the MAX_VOLTAGE_CHANGE factor f = min(1, maxDv / max |dV|, maxDphi / max |dphi|)
// (state_vector_scaling.cu:53-97).  A lane whose factorization or solve failed (trouble) takes no step and does not
// advance its iteration: the next test ends it.  The per-lane iteration counters advance; a pending lane (reactive
// limits decided) is released.
// ---------------------------------------------------------------------------------------------------------------
__global__ void stepMaxKernel(DevNet net, DevBatch b) {
    __shared__ double red[2][8][32];
    const int s = blockIdx.x * 32 + threadIdx.x;
    const size_t S = b.S;
    double mdv = 0.0, mdphi = 0.0;
    if (s < b.S && solving(b, s)) {
        for (int r = blockIdx.y * 8 + threadIdx.y; r < net.n; r += 8 * gridDim.y) {
            const double a = fabs(b.dx[(size_t)r * S + s]);
            if (b.varType[r] == VAR_BUS_V) mdv = fmax(mdv, a);
            else if (b.varType[r] == VAR_BUS_PHI) mdphi = fmax(mdphi, a);
        }
    }
    red[0][threadIdx.y][threadIdx.x] = mdv;
    red[1][threadIdx.y][threadIdx.x] = mdphi;
    __syncthreads();
    if (threadIdx.y == 0 && s < b.S) {
        for (int k = 1; k < 8; k++) {
            mdv = fmax(mdv, red[0][k][threadIdx.x]);
            mdphi = fmax(mdphi, red[1][k][threadIdx.x]);
        }
        if (mdv != 0.0) atomicMax(&b.stepMax[s], (unsigned long long)__double_as_longlong(mdv));
        if (mdphi != 0.0) atomicMax(&b.stepMax[S + s], (unsigned long long)__double_as_longlong(mdphi));
    }
}

__global__ void stepKernel(DevNet net, DevBatch b, Settings cfg) {
    const size_t S = b.S;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int s = (int)(tid % S);
    const int r = (int)(tid / S);
    if (r >= net.n || !solving(b, s) || b.trouble[s]) return;
    if (cfg.svsMode == SVS_MAX_VOLTAGE_CHANGE) {
        const double mdv = __longlong_as_double((long long)b.stepMax[s]);
        const double mdphi = __longlong_as_double((long long)b.stepMax[S + s]);
        double f = 1.0;
        if (mdv > cfg.maxDv) f = fmin(f, cfg.maxDv / mdv);
        if (mdphi > cfg.maxDphi) f = fmin(f, cfg.maxDphi / mdphi);
        b.x[(size_t)r * S + s] += f * b.dx[(size_t)r * S + s];
    } else {
        b.x[(size_t)r * S + s] += b.dx[(size_t)r * S + s];
    }
}

__global__ void advanceKernel(DevBatch b) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.S || !b.active[s] || b.pending[s] || b.trouble[s]) return;
    b.iter[s]++;
    b.totalIter[s]++;
}

// Start of an iteration: the lanes an outer-loop check restarted last iteration solve again.
__global__ void releasePendingKernel(DevBatch b) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.S) return;
    b.pending[s] = 0;
    if (b.dsRestart) b.dsRestart[s] = 0;
}

// After the test: how many lanes factorize this iteration (the host skips the factor/solve graph when none does) and
// how many of those are close enough to convergence for the refinement steps (mode 0); or, after a mixed-precision
// factorization, how many factorizing lanes are flagged for an FP64 refactor (mode 1).
__global__ void countLanesKernel(DevBatch b, double refineBelow, int mode, int maxIter) {
    __shared__ int part[3][32];
    int c0 = 0, c1 = 0, c2 = 0;
    for (int s = threadIdx.x; s < b.S; s += blockDim.x) {
        const bool sv = b.active[s] && !b.pending[s];
        if (mode == 0) {
            // mixed precision: the lanes near convergence start this iteration's refinement (a lane already redone
            // in FP64 needs none)
            const bool near = sv && b.normOut[s] < refineBelow && !(b.precision64 && b.precision64[s]);
            c0 += sv ? 1 : 0;
            c1 += near ? 1 : 0;
            if (b.refine) b.refine[s] = near ? 1 : 0;
            // lanes whose solve is scored this iteration (the guard's second iteration of a first solve, or the
            // iteration before the budget)
            const int it = b.iter[s];
            c2 += sv && ((b.outer[s] == 0 && it == 1) || it == maxIter - 1) ? 1 : 0;
        } else {
            c0 += sv && b.precision64[s] ? 1 : 0;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        c0 += __shfl_down_sync(0xffffffffu, c0, o);
        c1 += __shfl_down_sync(0xffffffffu, c1, o);
        c2 += __shfl_down_sync(0xffffffffu, c2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        part[0][threadIdx.x >> 5] = c0;
        part[1][threadIdx.x >> 5] = c1;
        part[2][threadIdx.x >> 5] = c2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int t0 = 0, t1 = 0, t2 = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            t0 += part[0][w];
            t1 += part[1][w];
            t2 += part[2][w];
        }
        if (mode == 0) {
            b.nActive[1] = t0;
            b.nActive[2] = t1;
            b.nActive[4] = t2;
        } else {
            b.nActive[3] = t0;
        }
    }
}

void launchIterationStart(const DevBatch& b, cudaStream_t st) {
    releasePendingKernel<<<(b.S + 127) / 128, 128, 0, st>>>(b);
}

void launchCountSolving(const DevBatch& b, double refineBelow, int maxIter, cudaStream_t st) {
    countLanesKernel<<<1, 1024, 0, st>>>(b, refineBelow, 0, maxIter);
}

void launchCountFp64(const DevBatch& b, cudaStream_t st) { countLanesKernel<<<1, 1024, 0, st>>>(b, 0.0, 1, 0); }

// Per-lane max |res| over the rows: 32 lanes x 8 row strands per CTA, reduced in shared memory, one atomic per CTA
// and lane (non-negative doubles order like their bit patterns; a NaN residual sorts above every number).
__global__ void residualMaxKernel(DevNet net, DevBatch b) {
    __shared__ double red[8][32];
    const int s = blockIdx.x * 32 + threadIdx.x;
    const size_t S = b.S;
    double m = 0.0;
    if (s < b.S && solving(b, s)) {
        for (int r = blockIdx.y * 8 + threadIdx.y; r < net.n; r += 8 * gridDim.y) m = absMax(m, b.res[(size_t)r * S + s]);
    }
    red[threadIdx.y][threadIdx.x] = m;
    __syncthreads();
    if (threadIdx.y == 0 && s < b.S) {
        for (int k = 1; k < 8; k++) m = absMax(m, red[k][threadIdx.x]);
        if (m != 0.0) atomicMax(&b.resNorm[s], (unsigned long long)__double_as_longlong(m));
    }
}

// Lanes near convergence (max |F| below refineBelow) whose linear residual is above the threshold: a lane further
// out takes another Newton step anyway, and its FP32 solve error shrinks with its mismatch.
__global__ void countResidualKernel(DevBatch b, double threshold, double refineBelow) {
    __shared__ int part[32];
    int c = 0;
    for (int s = threadIdx.x; s < b.S; s += blockDim.x) {
        const double r = __longlong_as_double((long long)b.resNorm[s]);
        c += (b.active[s] && !b.pending[s] && b.normOut[s] < refineBelow && !(r <= threshold)) ? 1 : 0;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[w];
        b.nActive[2] = t;
    }
}

void launchResidualCheck(const DevNet& net, const DevBatch& b, double threshold, double refineBelow,
                         cudaStream_t st) {
    cudaMemsetAsync(b.resNorm, 0, sizeof(unsigned long long) * b.S, st);
    residualMaxKernel<<<dim3(b.S / 32, 64), dim3(32, 8), 0, st>>>(net, b);
    countResidualKernel<<<1, 1024, 0, st>>>(b, threshold, refineBelow);
}

// After a correction solve: the lanes still refining are those whose correction max |d| (in b.res, reduced into
// b.resNorm) is above the bound; a NaN correction stops the lane's refinement (its next test decides its status).
__global__ void correctionCountKernel(DevBatch b, double bound) {
    __shared__ int part[32];
    int c = 0;
    for (int s = threadIdx.x; s < b.S; s += blockDim.x) {
        if (!b.refine[s]) continue;
        const double d = __longlong_as_double((long long)b.resNorm[s]);
        const bool more = d > bound;
        b.refine[s] = more ? 1 : 0;
        c += more ? 1 : 0;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[w];
        b.nActive[2] = t;
    }
}

void launchCorrectionCheck(const DevNet& net, const DevBatch& b, double bound, cudaStream_t st) {
    cudaMemsetAsync(b.resNorm, 0, sizeof(unsigned long long) * b.S, st);
    residualMaxKernel<<<dim3(b.S / 32, 64), dim3(32, 8), 0, st>>>(net, b);
    correctionCountKernel<<<1, 1024, 0, st>>>(b, bound);
}

// The lanes whose solve is scored this iteration: the second iteration of the first solve (no reactive-limit restart
// yet: the linear-solve guard, newton_iteration.cu:176-183,615-647) and the iteration before the budget (its ratio is
// read by the budget's test, newton_iteration.cu:371-392,534-546).
__device__ __forceinline__ bool scored(const DevBatch& b, const Settings& cfg, int s) {
    if (!solving(b, s) || b.trouble[s]) return false;
    const int it = b.iter[s];
    return (b.outer[s] == 0 && it == 1) || it == cfg.maxIter - 1;
}

__global__ void scoreResidualKernel(DevNet net, DevBatch b, Settings cfg) {
    const size_t S = b.S;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int s = (int)(tid % S);
    const int node = (int)(tid / S);
    if (node >= net.nb || !scored(b, cfg, s)) return;
    const int cP = net.nodeCol[2 * node], cV = net.nodeCol[2 * node + 1];
    double r0 = -b.F[cP * S + s], r1 = -b.F[cV * S + s];
    for (int t = net.aPtr[node]; t < net.aPtr[node + 1]; t++) {
        const int j = net.aCol[t];
        const double* J = b.J + (size_t)t * 4 * S + s;
        const double x0 = b.dx[(size_t)net.nodeCol[2 * j] * S + s], x1 = b.dx[(size_t)net.nodeCol[2 * j + 1] * S + s];
        r0 -= J[0] * x0 + J[S] * x1;
        r1 -= J[2 * S] * x0 + J[3 * S] * x1;
    }
    b.res[cP * S + s] = r0;
    b.res[cV * S + s] = r1;
}

// ratio = max |r| / max |F| (1e300 when F is zero or r is not finite, linResidScoreBatch in iterative_refinement.cu);
// a guard lane above LIN_SOLVE_FAIL_RATIO (NaN included) gets TROUBLE_GUARD, a budget lane keeps the ratio.
__global__ void scoreFinishKernel(DevBatch b, Settings cfg) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= b.S || !scored(b, cfg, s)) return;
    const double r = __longlong_as_double((long long)b.resNorm[s]);
    const double f = b.normOut[s];
    const double ratio = (f > 0.0 && isfinite(r)) ? r / f : 1e300;
    const int it = b.iter[s];
    if (it == cfg.maxIter - 1) b.solveRatio[s] = ratio;
    if (b.outer[s] == 0 && it == 1 && !(ratio <= LIN_SOLVE_FAIL_RATIO)) b.trouble[s] = TROUBLE_GUARD;
}

void launchScoreSolve(const DevNet& net, const DevBatch& b, const Settings& cfg, cudaStream_t st) {
    const size_t all = (size_t)net.nb * b.S;
    scoreResidualKernel<<<(unsigned)((all + 255) / 256), 256, 0, st>>>(net, b, cfg);
    cudaMemsetAsync(b.resNorm, 0, sizeof(unsigned long long) * b.S, st);
    residualMaxKernel<<<dim3(b.S / 32, 64), dim3(32, 8), 0, st>>>(net, b);
    scoreFinishKernel<<<(b.S + 127) / 128, 128, 0, st>>>(b, cfg);
}

void launchStep(const DevNet& net, const DevBatch& b, const Settings& cfg, cudaStream_t st) {
    const size_t all = (size_t)net.n * b.S;
    if (cfg.svsMode == SVS_MAX_VOLTAGE_CHANGE && b.varType) {
        cudaMemsetAsync(b.stepMax, 0, sizeof(unsigned long long) * 2 * b.S, st);
        stepMaxKernel<<<dim3(b.S / 32, 64), dim3(32, 8), 0, st>>>(net, b);
    }
    Settings c = cfg;
    if (!b.varType) c.svsMode = SVS_NONE;
    stepKernel<<<(unsigned)((all + 255) / 256), 256, 0, st>>>(net, b, c);
    advanceKernel<<<(b.S + 127) / 128, 128, 0, st>>>(b);
}


}  // namespace olfb200
