// Dense front of the block LU: the trailing F pivots of the elimination order (the root separators at the top of the
// elimination tree; absent blocks are structural zeros) factorized in shared memory, G lanes per CTA, instead of one
// dependency level per step.  The level tasks of the front blocks have already applied every update from the pivots
// before the front (in ascending pivot order); the front continues right-looking in ascending pivot order, so every
// block sees its updates in the same order as the left-looking level tasks, with the same 2x2 expressions.
#include "kernels.cuh"

namespace olfb200 {

namespace {

__device__ __forceinline__ bool frontSolving(const DevBatch& b, int s) {
    return b.active[s] && !b.pending[s] && (!b.laneMask || b.laneMask[s]);
}

template <typename T>
__global__ void __launch_bounds__(256) denseFrontKernel(DevNet net, DevBatch b, T* lu, int G) {
    extern __shared__ __align__(16) unsigned char smraw[];
    T* M = reinterpret_cast<T*>(smraw);
    const int F = net.frontF, N = 2 * F, LD = 2 * F + 1;
    const size_t S = b.S;
    const int s0 = blockIdx.x * G;
    // blocks of the G lanes into shared memory (the lane index runs fastest: neighbouring threads, neighbouring lanes)
    for (int idx = threadIdx.x; idx < G * F * F; idx += blockDim.x) {
        const int g = idx % G, blk = idx / G, i = blk / F, j = blk % F;
        const int s = s0 + g;
        if (s >= b.S) continue;
        const int id = net.frontBlocks[blk];
        T* m = M + (size_t)g * N * LD;
        if (id < 0) {   // a structural zero of the front stays an exact zero through the elimination
            m[(2 * i) * LD + 2 * j] = m[(2 * i) * LD + 2 * j + 1] = 0;
            m[(2 * i + 1) * LD + 2 * j] = m[(2 * i + 1) * LD + 2 * j + 1] = 0;
            continue;
        }
        const T* p = lu + (size_t)id * 4 * S + s;
        m[(2 * i) * LD + 2 * j] = p[0];
        m[(2 * i) * LD + 2 * j + 1] = p[S];
        m[(2 * i + 1) * LD + 2 * j] = p[2 * S];
        m[(2 * i + 1) * LD + 2 * j + 1] = p[3 * S];
    }
    __syncthreads();
    for (int k = 0; k < F; k++) {
        // the pivot block: inverted in place (one thread per lane)
        if (threadIdx.x < G) {
            const int g = threadIdx.x, s = s0 + g;
            if (s < b.S && frontSolving(b, s)) {
                T* m = M + (size_t)g * N * LD;
                T* d0 = m + (2 * k) * LD + 2 * k;
                T* d1 = d0 + LD;
                const T a00 = d0[0], a01 = d0[1], a10 = d1[0], a11 = d1[1];
                const T det = a00 * a11 - a01 * a10;
                const T scale = fabs(a00 * a11) + fabs(a01 * a10);
                if (!(fabs(det) > (T)1e-13 * scale) || !isfinite(det)) b.trouble[s] = 1;
                const T inv = (T)1 / det;
                if (sizeof(T) == 4 && b.precision64) {
                    // the mixed-precision pivot-growth check against the pivot's Jacobian block
                    const int ab = net.task[net.frontBlocks[k * F + k]].aBlock;
                    float amax = 0.f;
                    if (ab >= 0) {
                        const double* pj = b.J + (size_t)ab * 4 * S + s;
                        amax = fmaxf(fmaxf(fabsf((float)pj[0]), fabsf((float)pj[S])),
                                     fmaxf(fabsf((float)pj[2 * S]), fabsf((float)pj[3 * S])));
                    }
                    const float dmax = fmaxf(fmaxf(fabsf((float)a00), fabsf((float)a01)),
                                             fmaxf(fabsf((float)a10), fabsf((float)a11)));
                    const float kappa = dmax * dmax * fabsf((float)inv);
                    const float grow = amax > 0 ? dmax / amax : 1.0f;
                    if (!(kappa <= (float)b.growthLimit) || !(grow <= (float)b.growthLimit)) b.precision64[s] = 1;
                }
                d0[0] = a11 * inv;
                d0[1] = -a01 * inv;
                d1[0] = -a10 * inv;
                d1[1] = a00 * inv;
            }
        }
        __syncthreads();
        // the L column: L(i, k) = M(i, k) inv(D_k)
        const int rest = F - 1 - k;
        for (int idx = threadIdx.x; idx < G * rest; idx += blockDim.x) {
            const int g = idx % G, i = k + 1 + idx / G;
            const int s = s0 + g;
            if (s >= b.S || !frontSolving(b, s)) continue;
            T* m = M + (size_t)g * N * LD;
            const T* d0 = m + (2 * k) * LD + 2 * k;
            const T* d1 = d0 + LD;
            T* l0 = m + (2 * i) * LD + 2 * k;
            T* l1 = l0 + LD;
            const T i00 = d0[0], i01 = d0[1], i10 = d1[0], i11 = d1[1];
            const T a00 = l0[0], a01 = l0[1], a10 = l1[0], a11 = l1[1];
            l0[0] = a00 * i00 + a01 * i10;
            l0[1] = a00 * i01 + a01 * i11;
            l1[0] = a10 * i00 + a11 * i10;
            l1[1] = a10 * i01 + a11 * i11;
        }
        __syncthreads();
        // the trailing blocks: M(i, j) -= L(i, k) U(k, j)
        for (int idx = threadIdx.x; idx < G * rest * rest; idx += blockDim.x) {
            const int g = idx % G, t = idx / G, i = k + 1 + t / rest, j = k + 1 + t % rest;
            const int s = s0 + g;
            if (s >= b.S || !frontSolving(b, s)) continue;
            T* m = M + (size_t)g * N * LD;
            const T* l0 = m + (2 * i) * LD + 2 * k;
            const T* l1 = l0 + LD;
            const T* u0 = m + (2 * k) * LD + 2 * j;
            const T* u1 = u0 + LD;
            T* a0 = m + (2 * i) * LD + 2 * j;
            T* a1 = a0 + LD;
            const T l00 = l0[0], l01 = l0[1], l10 = l1[0], l11 = l1[1];
            const T u00 = u0[0], u01 = u0[1], u10 = u1[0], u11 = u1[1];
            a0[0] -= l00 * u00 + l01 * u10;
            a0[1] -= l00 * u01 + l01 * u11;
            a1[0] -= l10 * u00 + l11 * u10;
            a1[1] -= l10 * u01 + l11 * u11;
        }
        __syncthreads();
    }
    // back to the factor storage: U blocks (diagonal as its inverse) and scaled L blocks, as the level tasks store them
    for (int idx = threadIdx.x; idx < G * F * F; idx += blockDim.x) {
        const int g = idx % G, blk = idx / G, i = blk / F, j = blk % F;
        const int s = s0 + g;
        const int id = net.frontBlocks[blk];
        if (s >= b.S || id < 0 || !frontSolving(b, s)) continue;
        T* p = lu + (size_t)id * 4 * S + s;
        const T* m = M + (size_t)g * N * LD;
        p[0] = m[(2 * i) * LD + 2 * j];
        p[S] = m[(2 * i) * LD + 2 * j + 1];
        p[2 * S] = m[(2 * i + 1) * LD + 2 * j];
        p[3 * S] = m[(2 * i + 1) * LD + 2 * j + 1];
    }
}

// The triangular solves of the front positions, after the forward level tasks have applied every column before the
// front: forward y_i -= L(i, k) y_k (k ascending), then backward x_i = inv(D_i) y_i and y_r -= U(r, i) x_i (i
// descending), with the front's factor blocks and solution entries in shared memory.  In place on w.
template <typename T>
__global__ void __launch_bounds__(256) denseFrontSolveKernel(DevNet net, DevBatch b, const T* lu, T* w, int G) {
    extern __shared__ __align__(16) unsigned char smraw[];
    T* M = reinterpret_cast<T*>(smraw);
    const int F = net.frontF, N = 2 * F, LD = 2 * F + 1, k0 = net.frontStart;
    T* Y = M + (size_t)G * N * LD;   // [G][N]
    const size_t S = b.S;
    const int s0 = blockIdx.x * G;
    for (int idx = threadIdx.x; idx < G * F * F; idx += blockDim.x) {
        const int g = idx % G, blk = idx / G, i = blk / F, j = blk % F;
        const int s = s0 + g;
        const int id = net.frontBlocks[blk];
        if (s >= b.S || id < 0) continue;
        const T* p = lu + (size_t)id * 4 * S + s;
        T* m = M + (size_t)g * N * LD;
        m[(2 * i) * LD + 2 * j] = p[0];
        m[(2 * i) * LD + 2 * j + 1] = p[S];
        m[(2 * i + 1) * LD + 2 * j] = p[2 * S];
        m[(2 * i + 1) * LD + 2 * j + 1] = p[3 * S];
    }
    for (int idx = threadIdx.x; idx < G * N; idx += blockDim.x) {
        const int g = idx % G, r = idx / G, s = s0 + g;
        if (s < b.S) Y[g * N + r] = w[(2 * (size_t)k0 + r) * S + s];
    }
    __syncthreads();
    for (int k = 0; k < F; k++) {   // forward: the column of pivot k into the later rows
        for (int idx = threadIdx.x; idx < G * (F - 1 - k); idx += blockDim.x) {
            const int g = idx % G, i = k + 1 + idx / G, s = s0 + g;
            if (s >= b.S || !frontSolving(b, s)) continue;
            const T* m = M + (size_t)g * N * LD;
            const T* l0 = m + (2 * i) * LD + 2 * k;
            const T* l1 = l0 + LD;
            T* y = Y + g * N;
            const T y0 = y[2 * k], y1 = y[2 * k + 1];
            y[2 * i] -= l0[0] * y0 + l0[1] * y1;
            y[2 * i + 1] -= l1[0] * y0 + l1[1] * y1;
        }
        __syncthreads();
    }
    for (int i = F - 1; i >= 0; i--) {   // backward: pivot i, then its column of U into the earlier rows
        if (threadIdx.x < G) {
            const int g = threadIdx.x, s = s0 + g;
            if (s < b.S && frontSolving(b, s)) {
                const T* m = M + (size_t)g * N * LD;
                const T* d0 = m + (2 * i) * LD + 2 * i;
                const T* d1 = d0 + LD;
                T* y = Y + g * N;
                const T w0 = y[2 * i], w1 = y[2 * i + 1];
                y[2 * i] = d0[0] * w0 + d0[1] * w1;
                y[2 * i + 1] = d1[0] * w0 + d1[1] * w1;
            }
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < G * i; idx += blockDim.x) {
            const int g = idx % G, r = idx / G, s = s0 + g;
            if (s >= b.S || !frontSolving(b, s)) continue;
            const T* m = M + (size_t)g * N * LD;
            const T* u0 = m + (2 * r) * LD + 2 * i;
            const T* u1 = u0 + LD;
            T* y = Y + g * N;
            const T x0 = y[2 * i], x1 = y[2 * i + 1];
            y[2 * r] -= u0[0] * x0 + u0[1] * x1;
            y[2 * r + 1] -= u1[0] * x0 + u1[1] * x1;
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < G * N; idx += blockDim.x) {
        const int g = idx % G, r = idx / G, s = s0 + g;
        if (s < b.S && frontSolving(b, s)) w[(2 * (size_t)k0 + r) * S + s] = Y[g * N + r];
    }
}

template <typename T>
constexpr int lanesPerCta() { return sizeof(T) == 8 ? 2 : 4; }

template <typename T>
size_t frontBytes(int F) { return (size_t)lanesPerCta<T>() * (2 * F) * (2 * F + 1) * sizeof(T); }

template <typename T>
void frontT(const DevNet& net, const DevBatch& b, T* lu, cudaStream_t st) {
    const int G = lanesPerCta<T>();
    denseFrontKernel<T><<<(b.S + G - 1) / G, 256, frontBytes<T>(net.frontF), st>>>(net, b, lu, G);
}

template <typename T>
void frontSolveT(const DevNet& net, const DevBatch& b, const T* lu, T* w, cudaStream_t st) {
    const int G = lanesPerCta<T>();
    const size_t bytes = frontBytes<T>(net.frontF) + (size_t)G * 2 * net.frontF * sizeof(T);
    denseFrontSolveKernel<T><<<(b.S + G - 1) / G, 256, bytes, st>>>(net, b, lu, w, G);
}

}  // namespace

cudaError_t prepareDenseFront(int F) {
    const int y64 = lanesPerCta<double>() * 2 * F * 8, y32 = lanesPerCta<float>() * 2 * F * 4;
    cudaError_t e = cudaFuncSetAttribute(denseFrontKernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)frontBytes<double>(F));
    if (e == cudaSuccess) {
        e = cudaFuncSetAttribute(denseFrontKernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)frontBytes<float>(F));
    }
    if (e == cudaSuccess) {
        e = cudaFuncSetAttribute(denseFrontSolveKernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)frontBytes<double>(F) + y64);
    }
    if (e == cudaSuccess) {
        e = cudaFuncSetAttribute(denseFrontSolveKernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)frontBytes<float>(F) + y32);
    }
    return e;
}

void launchDenseFrontSolve(const DevNet& net, const DevBatch& b, bool fp32, cudaStream_t st) {
    if (net.frontF <= 0) return;
    if (fp32) frontSolveT<float>(net, b, b.lu32, b.w32, st);
    else frontSolveT<double>(net, b, b.lu64, b.w64, st);
}

void launchDenseFront(const DevNet& net, const DevBatch& b, bool fp32, cudaStream_t st) {
    if (net.frontF <= 0) return;
    if (fp32) frontT<float>(net, b, b.lu32, st);
    else frontT<double>(net, b, b.lu64, st);
}

}  // namespace olfb200
