// Cooperative level sweeps: the factorization (every level) and the triangular solves (rhs, forward, backward,
// scatter) of all lanes, each phase in ONE cooperative launch whose CTAs meet at a grid barrier between dependency
// levels.  Same arithmetic and summation order as the per-level launches of kernels.cu (one task or row per
// (thread row, lane), P threads splitting its update list, partial sums added part 0 first), without a kernel launch
// per level: the narrow levels at the top of the elimination tree cost a barrier instead of a launch.
#include <cooperative_groups.h>

#include "coop.cuh"

namespace cg = cooperative_groups;

namespace olfb200 {

namespace {

constexpr int ROWS = 16;   // thread rows per CTA: TPB = ROWS / P tasks of a level per virtual block

__device__ __forceinline__ bool coopSolving(const DevBatch& b, int s) {
    return b.active[s] && !b.pending[s] && (!b.laneMask || b.laneMask[s]);
}

template <typename T>
__device__ __forceinline__ void ld4c(const T* base, size_t blk, size_t S, int s, T& a, T& b_, T& c, T& d) {
    const T* p = base + blk * 4 * S + s;
    a = p[0];
    b_ = p[S];
    c = p[2 * S];
    d = p[3 * S];
}

template <typename T>
__device__ __forceinline__ void st4c(T* base, size_t blk, size_t S, int s, T a, T b_, T c, T d) {
    T* p = base + blk * 4 * S + s;
    p[0] = a;
    p[S] = b_;
    p[2 * S] = c;
    p[3 * S] = d;
}

// One virtual block of a factorization level: ROWS / P tasks x 32 lanes (lane group vby).
template <typename T>
__device__ void factorVBlock(const DevNet& net, const DevBatch& b, T* lu, int first, int count, int P, int vbx,
                             int vby, T (*red)[4][32]) {
    const size_t S = b.S;
    const int lane = threadIdx.x, ty = threadIdx.y;
    const int tib = ty / P, part = ty % P;
    const int s = vby * 32 + lane;
    const int k = vbx * (ROWS / P) + tib;
    const bool ok = k < count && s < b.S && coopSolving(b, s);
    T a00 = 0, a01 = 0, a10 = 0, a11 = 0, amax = 0;
    int t = 0;
    Task tk{};
    if (ok) {
        t = net.levelTask[first + k];
        tk = net.task[t];
        if (part == 0 && tk.aBlock >= 0) {
            const double* p = b.J + (size_t)tk.aBlock * 4 * S + s;
            a00 = (T)p[0];
            a01 = (T)p[S];
            a10 = (T)p[2 * S];
            a11 = (T)p[3 * S];
            amax = fmax(fmax(fabs(a00), fabs(a01)), fmax(fabs(a10), fabs(a11)));
        }
#pragma unroll 4
        for (int q = tk.opBegin + part; q < tk.opEnd; q += P) {
            const int4 op = net.ops[q];
            T m00, m01, m10, m11, u00, u01, u10, u11;
            ld4c(lu, (size_t)op.x, S, s, m00, m01, m10, m11);
            ld4c(lu, (size_t)op.y, S, s, u00, u01, u10, u11);
            if (op.z >= 0) {   // deferred-L plan: L~(a,m) inv(D_m)
                T d00, d01, d10, d11;
                ld4c(lu, (size_t)op.z, S, s, d00, d01, d10, d11);
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
        __syncthreads();   // red is reused by the next virtual block
    }
    if (!ok || part != 0) return;
    if (tk.diag == -2) {
        const T det = rnFma(a00, a11, -rnMul(a01, a10));
        const T scale = fabs(a00 * a11) + fabs(a01 * a10);
        if (!(fabs(det) > (T)1e-13 * scale) || !isfinite(det)) b.trouble[s] = 1;
        const T inv = (T)1 / det;
        if (sizeof(T) == 4 && b.precision64) {
            const float dmax = fmaxf(fmaxf(fabsf((float)a00), fabsf((float)a01)), fmaxf(fabsf((float)a10), fabsf((float)a11)));
            const float kappa = dmax * dmax * fabsf((float)inv);
            const float grow = amax > 0 ? dmax / (float)amax : 1.0f;
            if (!(kappa <= (float)b.growthLimit) || !(grow <= (float)b.growthLimit)) b.precision64[s] = 1;
        }
        st4c(lu, (size_t)t, S, s, a11 * inv, -a01 * inv, -a10 * inv, a00 * inv);
    } else if (tk.diag >= 0 && !net.deferredL) {
        T i00, i01, i10, i11;
        ld4c(lu, (size_t)tk.diag, S, s, i00, i01, i10, i11);
        st4c(lu, (size_t)t, S, s, dot2(a00, i00, a01, i10), dot2(a00, i01, a01, i11), dot2(a10, i00, a11, i10),
             dot2(a10, i01, a11, i11));
    } else {
        st4c(lu, (size_t)t, S, s, a00, a01, a10, a11);
    }
}

template <typename T>
__global__ void __launch_bounds__(512) factorCoopKernel(DevNet net, DevBatch b, T* lu, CoopPlan cp) {
    __shared__ T red[ROWS][4][32];
    cg::grid_group grid = cg::this_grid();
    const int nthreads = gridDim.x * blockDim.x * blockDim.y;
    const int gtid = (blockIdx.x * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
    for (int s = gtid; s < b.S; s += nthreads)
        if (coopSolving(b, s)) b.trouble[s] = 0;
    const int vy = b.S / 32;
    for (int l = 0; l < cp.nLevels; l++) {
        const int first = cp.levelPtr[l], count = cp.levelPtr[l + 1] - first;
        const int P = cp.levelSplit[l];
        const int vx = (count + ROWS / P - 1) / (ROWS / P);
        for (int vb = blockIdx.x; vb < vx * vy; vb += gridDim.x) factorVBlock<T>(net, b, lu, first, count, P, vb % vx, vb / vx, red);
        grid.sync();
    }
    if (net.deferredL) {
        // the last pass of the deferred-L plan: L = L~ inv(D_k)
        const size_t S = b.S;
        const long long cells = (long long)(net.nLu - net.nU) * b.S;
        for (long long c = gtid; c < cells; c += nthreads) {
            const int s = (int)(c % b.S);
            const int id = net.nU + (int)(c / b.S);
            if (!coopSolving(b, s)) continue;
            T a00, a01, a10, a11, i00, i01, i10, i11;
            ld4c(lu, (size_t)id, S, s, a00, a01, a10, a11);
            ld4c(lu, (size_t)net.task[id].diag, S, s, i00, i01, i10, i11);
            st4c(lu, (size_t)id, S, s, dot2(a00, i00, a01, i10), dot2(a00, i01, a01, i11), dot2(a10, i00, a11, i10),
                 dot2(a10, i01, a11, i11));
        }
    }
}

// One virtual block of a solve level: dir 0 forward (L rows), dir 1 backward (U rows, times the inverse diagonal).
template <typename T>
__device__ void solveVBlock(const DevNet& net, const DevBatch& b, const T* lu, T* w, const int* pos, int dir,
                            int first, int count, int P, int vbx, int vby, T (*red)[2][32]) {
    const size_t S = b.S;
    const int lane = threadIdx.x, ty = threadIdx.y;
    const int tib = ty / P, part = ty % P;
    const int s = vby * 32 + lane;
    const int k = vbx * (ROWS / P) + tib;
    const bool ok = k < count && s < b.S && coopSolving(b, s);
    T w0 = 0, w1 = 0;
    int i = 0;
    if (ok) {
        i = pos[first + k];
        if (part == 0) {
            w0 = w[(2 * (size_t)i) * S + s];
            w1 = w[(2 * (size_t)i + 1) * S + s];
        }
        if (dir == 0) {
#pragma unroll 4
            for (int q = net.lrowPtr[i] + part; q < net.lrowEnd[i]; q += P) {
                const int2 e = net.lrow[q];
                T l00, l01, l10, l11;
                ld4c(lu, (size_t)e.x, S, s, l00, l01, l10, l11);
                const T y0 = w[(2 * (size_t)e.y) * S + s], y1 = w[(2 * (size_t)e.y + 1) * S + s];
                w0 = rnSub(w0, dot2(l00, y0, l01, y1));
                w1 = rnSub(w1, dot2(l10, y0, l11, y1));
            }
        } else {
#pragma unroll 4
            for (int q = net.uPtr[i] + 1 + part; q < net.uPtr[i + 1]; q += P) {
                const int j = net.uCol[q];
                T u00, u01, u10, u11;
                ld4c(lu, (size_t)q, S, s, u00, u01, u10, u11);
                const T x0 = w[(2 * (size_t)j) * S + s], x1 = w[(2 * (size_t)j + 1) * S + s];
                w0 = rnSub(w0, dot2(u00, x0, u01, x1));
                w1 = rnSub(w1, dot2(u10, x0, u11, x1));
            }
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
        __syncthreads();
    }
    if (!ok || part != 0) return;
    if (dir == 0) {
        w[(2 * (size_t)i) * S + s] = w0;
        w[(2 * (size_t)i + 1) * S + s] = w1;
    } else {
        T i00, i01, i10, i11;
        ld4c(lu, (size_t)net.uPtr[i], S, s, i00, i01, i10, i11);
        w[(2 * (size_t)i) * S + s] = dot2(i00, w0, i01, w1);
        w[(2 * (size_t)i + 1) * S + s] = dot2(i10, w0, i11, w1);
    }
}

// rhs (from -F or from the refinement residual) -> forward levels -> backward levels -> dx (= or +=).
// mode 0: everything; 1: rhs and the forward levels; 2: the backward levels and dx (a dense front solve between).
template <typename T>
__global__ void __launch_bounds__(512) solveCoopKernel(DevNet net, DevBatch b, const T* lu, T* w, CoopPlan cp,
                                                       int fromResidual, int mode) {
    __shared__ T red[ROWS][2][32];
    cg::grid_group grid = cg::this_grid();
    const size_t S = b.S;
    const long long nthreads = (long long)gridDim.x * blockDim.x * blockDim.y;
    const long long gtid = ((long long)blockIdx.x * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
    const long long cells = (long long)net.nb * b.S;
    const int vy = b.S / 32;
    if (mode != 2) {
    for (long long c = gtid; c < cells; c += nthreads) {
        const int s = (int)(c % b.S), i = (int)(c / b.S);
        if (!coopSolving(b, s)) continue;
        const int node = net.perm[i];
        const int cP = net.nodeCol[2 * node], cV = net.nodeCol[2 * node + 1];
        const double r0 = fromResidual ? b.res[cP * S + s] : -b.F[cP * S + s];
        const double r1 = fromResidual ? b.res[cV * S + s] : -b.F[cV * S + s];
        w[(2 * (size_t)i) * S + s] = (T)r0;
        w[(2 * (size_t)i + 1) * S + s] = (T)r1;
    }
    grid.sync();
    for (int l = 0; l < cp.nFwd; l++) {
        const int first = cp.fwdPtr[l], count = cp.fwdPtr[l + 1] - first, P = cp.fwdSplit[l];
        const int vx = (count + ROWS / P - 1) / (ROWS / P);
        for (int vb = blockIdx.x; vb < vx * vy; vb += gridDim.x)
            solveVBlock<T>(net, b, lu, w, cp.fwdPos, 0, first, count, P, vb % vx, vb / vx, red);
        grid.sync();
    }
    }
    if (mode == 1) return;
    for (int l = 0; l < cp.nBwd; l++) {
        const int first = cp.bwdPtr[l], count = cp.bwdPtr[l + 1] - first, P = cp.bwdSplit[l];
        const int vx = (count + ROWS / P - 1) / (ROWS / P);
        for (int vb = blockIdx.x; vb < vx * vy; vb += gridDim.x)
            solveVBlock<T>(net, b, lu, w, cp.bwdPos, 1, first, count, P, vb % vx, vb / vx, red);
        grid.sync();
    }
    for (long long c = gtid; c < cells; c += nthreads) {
        const int s = (int)(c % b.S), node = (int)(c / b.S);
        if (!coopSolving(b, s)) continue;
        const int i = net.iperm[node];
        const int cP = net.nodeCol[2 * node], cV = net.nodeCol[2 * node + 1];
        const double d0 = (double)w[(2 * (size_t)i) * S + s], d1 = (double)w[(2 * (size_t)i + 1) * S + s];
        if (fromResidual) {
            b.dx[cP * S + s] += d0;
            b.dx[cV * S + s] += d1;
        } else {
            b.dx[cP * S + s] = d0;
            b.dx[cV * S + s] = d1;
        }
    }
}

// CTAs of a cooperative launch: as many as can be resident at once (a cooperative launch is refused otherwise).
template <typename K>
int coopGrid(K kernel) {
    int dev = 0, sms = 0, perSm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, 32 * ROWS, 0);
    return perSm * sms;
}

template <typename T>
cudaError_t factorCoopT(const DevNet& net, const DevBatch& b, T* lu, const CoopPlan& cp, cudaStream_t st) {
    static const int grid = coopGrid(factorCoopKernel<T>);
    if (grid <= 0) return cudaErrorLaunchOutOfResources;
    DevNet n2 = net;
    DevBatch b2 = b;
    CoopPlan c2 = cp;
    void* args[] = {&n2, &b2, &lu, &c2};
    return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(factorCoopKernel<T>), dim3(grid), dim3(32, ROWS), args, 0,
                                       st);
}

template <typename T>
cudaError_t solveCoopT(const DevNet& net, const DevBatch& b, const T* lu, T* w, const CoopPlan& cp, int fromResidual,
                       int mode, cudaStream_t st) {
    static const int grid = coopGrid(solveCoopKernel<T>);
    if (grid <= 0) return cudaErrorLaunchOutOfResources;
    DevNet n2 = net;
    DevBatch b2 = b;
    CoopPlan c2 = cp;
    void* args[] = {&n2, &b2, &lu, &w, &c2, &fromResidual, &mode};
    return cudaLaunchCooperativeKernel(reinterpret_cast<void*>(solveCoopKernel<T>), dim3(grid), dim3(32, ROWS), args, 0,
                                       st);
}

}  // namespace

cudaError_t launchFactorCoop(const DevNet& net, const DevBatch& b, const CoopPlan& cp, bool fp32, cudaStream_t st) {
    return fp32 ? factorCoopT<float>(net, b, b.lu32, cp, st) : factorCoopT<double>(net, b, b.lu64, cp, st);
}

cudaError_t launchSolveCoop(const DevNet& net, const DevBatch& b, const CoopPlan& cp, bool fp32, bool fromResidual,
                            cudaStream_t st) {
    const int fr = fromResidual ? 1 : 0;
    if (net.frontF <= 0) {
        return fp32 ? solveCoopT<float>(net, b, b.lu32, b.w32, cp, fr, 0, st)
                    : solveCoopT<double>(net, b, b.lu64, b.w64, cp, fr, 0, st);
    }
    // dense-front plan: forward levels, the front's dense solves, backward levels
    cudaError_t e = fp32 ? solveCoopT<float>(net, b, b.lu32, b.w32, cp, fr, 1, st)
                         : solveCoopT<double>(net, b, b.lu64, b.w64, cp, fr, 1, st);
    if (e != cudaSuccess) return e;
    launchDenseFrontSolve(net, b, fp32, st);
    return fp32 ? solveCoopT<float>(net, b, b.lu32, b.w32, cp, fr, 2, st)
                : solveCoopT<double>(net, b, b.lu64, b.w64, cp, fr, 2, st);
}

}  // namespace olfb200
