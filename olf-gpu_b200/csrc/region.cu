// Narrow factorization levels in shared memory.  The top of the elimination tree (the levels of at most a few dozen
// tasks before the dense front) is a long chain of small dependent levels: one launch per level leaves the GPU idle
// between launches and every update waits on global-memory latency.  Here those levels run inside one CTA per lane
// with every LU block they produce held in shared memory ("slots", in level order), a barrier between levels and the
// P threads of a task splitting its update list.
//
// Two launches: regionPrefixKernel (one thread per (slot, lane), lanes coalesced) applies to each slot's task the
// leading updates whose operands both lie outside the region, all finished before the region starts, and stores the
// partial sums in the task's LU block; regionFactorKernel then loads the partials into shared memory and runs the
// region's levels, reading an update operand from its slot (ops.w: slot + 1 of the L block in the low 16 bits, of
// the U block in the high 16 bits, 0 outside the region) or from global memory, and writes each finished block to
// both.  The expressions per block are those of factorLevelKernel (pivot inverse, L scaled by the inverted pivot,
// the near-singular and pivot-growth checks); the P partial sums of a task are combined by a fixed butterfly.
//
// The solves' narrow levels (solveRegionKernel, schedule 4) follow the same pattern: the forward tail and the backward
// head of the triangular sweeps, one CTA per lane, the solution entries of their rows in shared memory.
#include "kernels.cuh"

namespace olfb200 {

namespace {

__device__ __forceinline__ bool regionSolving(const DevBatch& b, int s) {
    return b.active[s] && !b.pending[s] && (!b.laneMask || b.laneMask[s]);
}

template <typename T>
__device__ __forceinline__ void ld4g(const T* lu, int blk, size_t S, int s, T (&v)[4]) {
    const T* p = lu + (size_t)blk * 4 * S + s;
    v[0] = p[0];
    v[1] = p[S];
    v[2] = p[2 * S];
    v[3] = p[3 * S];
}

template <typename T>
__device__ __forceinline__ void st4g(T* lu, int blk, size_t S, int s, const T (&v)[4]) {
    T* p = lu + (size_t)blk * 4 * S + s;
    p[0] = v[0];
    p[S] = v[1];
    p[2 * S] = v[2];
    p[3 * S] = v[3];
}

// Partial sums of the slots' tasks: A - the updates [opBegin, mid) (both operands outside the region), one thread per
// (slot, lane).
template <typename T>
__global__ void __launch_bounds__(256) regionPrefixKernel(DevNet net, DevBatch b, T* lu, int nSlots,
                                                          const int4* rtask) {
    const int s = blockIdx.y * 32 + threadIdx.x;
    const int k = blockIdx.x * 8 + threadIdx.y;
    if (k >= nSlots || s >= b.S || !regionSolving(b, s)) return;
    const size_t S = b.S;
    const int4 rt = rtask[k];
    const Task tk = net.task[rt.x];
    T a[4] = {0, 0, 0, 0};
    if (tk.aBlock >= 0) {
        const double* p = b.J + (size_t)tk.aBlock * 4 * S + s;
        a[0] = (T)p[0];
        a[1] = (T)p[S];
        a[2] = (T)p[2 * S];
        a[3] = (T)p[3 * S];
    }
#pragma unroll 2
    for (int q = tk.opBegin; q < rt.z; q++) {
        const int4 op = net.ops[q];
        T m[4], u[4];
        ld4g(lu, op.x, S, s, m);
        ld4g(lu, op.y, S, s, u);
        a[0] -= m[0] * u[0] + m[1] * u[2];
        a[1] -= m[0] * u[1] + m[1] * u[3];
        a[2] -= m[2] * u[0] + m[3] * u[2];
        a[3] -= m[2] * u[1] + m[3] * u[3];
    }
    st4g(lu, rt.x, S, s, a);
}

template <typename T>
__device__ __forceinline__ void slotLoad(const T* blk, int slot, T (&v)[4]) {
    if (sizeof(T) == 8) {
        const double2* p = reinterpret_cast<const double2*>(blk + (size_t)slot * 4);
        const double2 x = p[0], y = p[1];
        v[0] = (T)x.x;
        v[1] = (T)x.y;
        v[2] = (T)y.x;
        v[3] = (T)y.y;
    } else {
        const float4 x = *reinterpret_cast<const float4*>(blk + (size_t)slot * 4);
        v[0] = (T)x.x;
        v[1] = (T)x.y;
        v[2] = (T)x.z;
        v[3] = (T)x.w;
    }
}

template <typename T>
__device__ __forceinline__ void slotStore(T* blk, int slot, const T (&v)[4]) {
    T* p = blk + (size_t)slot * 4;
    p[0] = v[0];
    p[1] = v[1];
    p[2] = v[2];
    p[3] = v[3];
}

// One thread's share of a level: the task (P threads per task, part = this thread's index among them), its first
// update and that update's operands outside the region, loaded one level ahead (they do not depend on the region).
template <typename T>
struct RegionItem {
    int4 rt;        // slot task; rt.x < 0: no task for this thread
    int slot;
    int4 op;        // the thread's first update (op.x < 0: none)
    T m[4], u[4];   // its operands outside the region
    T d[4];         // the inverted pivot outside the region (L tasks, part 0)
};

__device__ __forceinline__ int regionSplit(int count, int threads) {
    int P = 1;   // threads per task: a power of two <= 32, so a task's threads share a warp
    while (P < 32 && 2 * P * count <= threads) P *= 2;
    return P;
}

template <typename T>
__device__ __forceinline__ void regionFetch(const DevNet& net, const T* lu, size_t S, int s, const int* lvl, int li,
                                            int base, const int4* rtask, RegionItem<T>& it) {
    const int first = lvl[li], count = lvl[li + 1] - first;
    const int P = regionSplit(count, blockDim.x);
    const int k = threadIdx.x / P, part = threadIdx.x % P;
    it.rt.x = -1;
    it.op.x = -1;
    if (k >= count) return;
    it.slot = first - base + k;
    it.rt = rtask[it.slot];
    const int q = it.rt.z + part;
    if (q < it.rt.y) {
        it.op = net.ops[q];
        if ((it.op.w & 0xffff) == 0) ld4g(lu, it.op.x, S, s, it.m);
        if (((unsigned)it.op.w >> 16) == 0) ld4g(lu, it.op.y, S, s, it.u);
    }
    if (part == 0 && it.rt.w >= 0) ld4g(lu, it.rt.w, S, s, it.d);
}

// The region's levels [l0, l1) for lane blockIdx.x (every region level holds at most blockDim.x tasks: one round
// per level).  Shared memory: nSlots blocks of 4 T, (FP32) the max |A| of each slot's Jacobian block for the
// pivot-growth check, then the level boundaries.
template <typename T>
__global__ void __launch_bounds__(REGION_THREADS, 2) regionFactorKernel(DevNet net, DevBatch b, T* lu, const int* levelPtr,
                                                             int l0, int l1, int base, int nSlots, const int4* rtask) {
    extern __shared__ __align__(16) unsigned char regionSmem[];
    T* blk = reinterpret_cast<T*>(regionSmem);
    float* amaxS = reinterpret_cast<float*>(blk + (size_t)nSlots * 4);
    int* lvl = reinterpret_cast<int*>(amaxS + (sizeof(T) == 4 ? nSlots : 0));
    const int s = blockIdx.x;
    if (s >= b.S || !regionSolving(b, s)) return;   // the whole CTA: one lane
    const size_t S = b.S;
    for (int i = threadIdx.x; i <= l1 - l0; i += blockDim.x) lvl[i] = levelPtr[l0 + i];
    for (int k = threadIdx.x; k < nSlots; k += blockDim.x) {
        const int4 rt = rtask[k];
        T v[4];
        ld4g(lu, rt.x, S, s, v);
        slotStore(blk, k, v);
        if (sizeof(T) == 4) {
            float m = 0.f;
            if (rt.w == -2) {
                const int a = net.task[rt.x].aBlock;
                if (a >= 0) {
                    const double* p = b.J + (size_t)a * 4 * S + s;
                    m = fmaxf(fmaxf(fabsf((float)p[0]), fabsf((float)p[S])),
                              fmaxf(fabsf((float)p[2 * S]), fabsf((float)p[3 * S])));
                }
            }
            amaxS[k] = m;
        }
    }
    __syncthreads();
    RegionItem<T> next;
    regionFetch(net, lu, S, s, lvl, 0, base, rtask, next);
    for (int li = 0; li < l1 - l0; li++) {
        const RegionItem<T> cur = next;
        if (li + 1 < l1 - l0) regionFetch(net, lu, S, s, lvl, li + 1, base, rtask, next);
        const int count = lvl[li + 1] - lvl[li];
        const int P = regionSplit(count, blockDim.x);
        const int part = threadIdx.x % P;
        T acc[4] = {0, 0, 0, 0};
        if (cur.rt.x >= 0 && cur.op.x >= 0) {
            T m[4], u[4];
            const int sl = (cur.op.w & 0xffff) - 1, su = (int)((unsigned)cur.op.w >> 16) - 1;
            if (sl >= 0) slotLoad(blk, sl, m);
            else {
#pragma unroll
                for (int e = 0; e < 4; e++) m[e] = cur.m[e];
            }
            if (su >= 0) slotLoad(blk, su, u);
            else {
#pragma unroll
                for (int e = 0; e < 4; e++) u[e] = cur.u[e];
            }
            acc[0] = m[0] * u[0] + m[1] * u[2];
            acc[1] = m[0] * u[1] + m[1] * u[3];
            acc[2] = m[2] * u[0] + m[3] * u[2];
            acc[3] = m[2] * u[1] + m[3] * u[3];
#pragma unroll 2
            for (int q = cur.rt.z + part + P; q < cur.rt.y; q += P) {
                const int4 op = net.ops[q];
                const int ql = (op.w & 0xffff) - 1, qu = (int)((unsigned)op.w >> 16) - 1;
                if (ql >= 0) slotLoad(blk, ql, m);
                else ld4g(lu, op.x, S, s, m);
                if (qu >= 0) slotLoad(blk, qu, u);
                else ld4g(lu, op.y, S, s, u);
                acc[0] += m[0] * u[0] + m[1] * u[2];
                acc[1] += m[0] * u[1] + m[1] * u[3];
                acc[2] += m[2] * u[0] + m[3] * u[2];
                acc[3] += m[2] * u[1] + m[3] * u[3];
            }
        }
        for (int o = P >> 1; o > 0; o >>= 1) {
#pragma unroll
            for (int e = 0; e < 4; e++) acc[e] += __shfl_xor_sync(0xffffffffu, acc[e], o);
        }
        if (cur.rt.x >= 0 && part == 0) {
            const int slot = cur.slot, code = cur.rt.w;
            T a[4];
            slotLoad(blk, slot, a);
#pragma unroll
            for (int e = 0; e < 4; e++) a[e] -= acc[e];
            T v[4];
            if (code == -2) {
                const T det = a[0] * a[3] - a[1] * a[2];
                const T scale = fabs(a[0] * a[3]) + fabs(a[1] * a[2]);
                if (!(fabs(det) > (T)1e-13 * scale) || !isfinite(det)) b.trouble[s] = 1;
                const T inv = (T)1 / det;
                if (sizeof(T) == 4 && b.precision64) {
                    const float dmax = fmaxf(fmaxf(fabsf((float)a[0]), fabsf((float)a[1])),
                                             fmaxf(fabsf((float)a[2]), fabsf((float)a[3])));
                    const float kappa = dmax * dmax * fabsf((float)inv);
                    const float amax = amaxS[slot];
                    const float grow = amax > 0 ? dmax / amax : 1.0f;
                    if (!(kappa <= (float)b.growthLimit) || !(grow <= (float)b.growthLimit)) b.precision64[s] = 1;
                }
                v[0] = a[3] * inv;
                v[1] = -a[1] * inv;
                v[2] = -a[2] * inv;
                v[3] = a[0] * inv;
            } else if (code >= 0 || code <= -4) {
                // L(i, k) = (...) inv(D_k), the pivot inverted at an earlier level (outside the region, or a slot)
                T d[4];
                if (code <= -4) slotLoad(blk, -4 - code, d);
                else {
#pragma unroll
                    for (int e = 0; e < 4; e++) d[e] = cur.d[e];
                }
                v[0] = a[0] * d[0] + a[1] * d[2];
                v[1] = a[0] * d[1] + a[1] * d[3];
                v[2] = a[2] * d[0] + a[3] * d[2];
                v[3] = a[2] * d[1] + a[3] * d[3];
            } else {
                v[0] = a[0];
                v[1] = a[1];
                v[2] = a[2];
                v[3] = a[3];
            }
            slotStore(blk, slot, v);
            st4g(lu, cur.rt.x, S, s, v);
        }
        __syncthreads();
    }
}

// Shared memory of a region of nSlots slots and nLevels levels.
// The narrow solve levels of one sweep for lane blockIdx.x, in shared memory: DIR 0 the forward tail (L rows, levels
// [l0, l1) of the forward schedule), DIR 1 the backward head (U rows, then the inverted pivot).  Slot k holds the two
// solution entries of position pos[base + k]; an entry of a row reads its column from its slot (entrySlot[q] = slot
// + 1) or, outside the region (a wide level's or the dense front's position, final before this launch), from global
// memory.  Each thread loads its next level's row bounds, first entry and that entry's block one level ahead.
template <typename T, int DIR>
__global__ void __launch_bounds__(REGION_THREADS) solveRegionKernel(DevNet net, DevBatch b, const T* lu, T* w,
                                                                    const int* levelPtr, const int* pos, int l0,
                                                                    int l1, int base, int nSlots,
                                                                    const int* entrySlot, const int* rowStart) {
    extern __shared__ __align__(16) unsigned char regionSmem[];
    T* ws = reinterpret_cast<T*>(regionSmem);                                  // [nSlots][2]
    int* lvl = reinterpret_cast<int*>(ws + 2 * (size_t)nSlots + (nSlots & 1));   // [l1 - l0 + 1]
    const int s = blockIdx.x;
    if (s >= b.S || !regionSolving(b, s)) return;   // the whole CTA: one lane
    const size_t S = b.S;
    for (int i = threadIdx.x; i <= l1 - l0; i += blockDim.x) lvl[i] = levelPtr[l0 + i];
    for (int k = threadIdx.x; k < nSlots; k += blockDim.x) {
        const int i = pos[base + k];
        ws[2 * k] = w[(2 * (size_t)i) * S + s];
        ws[2 * k + 1] = w[(2 * (size_t)i + 1) * S + s];
    }
    __syncthreads();
    // next level's item: row position, entry range, first entry (block id, column, slot code) and its block
    int nPos = -1, nQ0 = 0, nQ1 = 0, nBlk = -1, nCol = 0, nCode = 0;
    T nM[4], nD[4];   // the first entry's block; (backward, part 0) the row's inverted pivot
    auto fetch = [&](int li) {
        const int first = lvl[li], count = lvl[li + 1] - first;
        const int P = regionSplit(count, blockDim.x);
        const int k = threadIdx.x / P, part = threadIdx.x % P;
        nPos = -1;
        nBlk = -1;
        if (k >= count) return;
        nPos = pos[first + k];
        if (DIR == 0) {
            nQ0 = rowStart[first - base + k];   // the entries before it went to the prefix launch
            nQ1 = net.lrowEnd[nPos];
        } else {
            nQ0 = net.uPtr[nPos] + 1;
            nQ1 = net.uPtr[nPos + 1];
        }
        const int q = nQ0 + part;
        if (q < nQ1) {
            if (DIR == 0) {
                const int2 e = net.lrow[q];
                nBlk = e.x;
                nCol = e.y;
            } else {
                nBlk = q;
                nCol = net.uCol[q];
            }
            nCode = entrySlot[q];
            ld4g(lu, nBlk, S, s, nM);
        }
        if (DIR == 1 && part == 0) ld4g(lu, nQ0 - 1, S, s, nD);
    };
    fetch(0);
    for (int li = 0; li < l1 - l0; li++) {
        const int iPos = nPos, q0 = nQ0, q1 = nQ1, blk0 = nBlk, col0 = nCol, code0 = nCode;
        T m0[4], d[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            m0[e] = nM[e];
            d[e] = nD[e];
        }
        if (li + 1 < l1 - l0) fetch(li + 1);
        const int first = lvl[li], count = lvl[li + 1] - first;
        const int P = regionSplit(count, blockDim.x);
        const int k = threadIdx.x / P, part = threadIdx.x % P;
        T a0 = 0, a1 = 0;
        if (iPos >= 0 && blk0 >= 0) {
            T y0, y1;
            if (code0 > 0) {
                y0 = ws[2 * (code0 - 1)];
                y1 = ws[2 * (code0 - 1) + 1];
            } else {
                y0 = w[(2 * (size_t)col0) * S + s];
                y1 = w[(2 * (size_t)col0 + 1) * S + s];
            }
            a0 = m0[0] * y0 + m0[1] * y1;
            a1 = m0[2] * y0 + m0[3] * y1;
#pragma unroll 2
            for (int q = q0 + part + P; q < q1; q += P) {
                int bq, c;
                if (DIR == 0) {
                    const int2 e = net.lrow[q];
                    bq = e.x;
                    c = e.y;
                } else {
                    bq = q;
                    c = net.uCol[q];
                }
                const int code = entrySlot[q];
                T m[4];
                ld4g(lu, bq, S, s, m);
                if (code > 0) {
                    y0 = ws[2 * (code - 1)];
                    y1 = ws[2 * (code - 1) + 1];
                } else {
                    y0 = w[(2 * (size_t)c) * S + s];
                    y1 = w[(2 * (size_t)c + 1) * S + s];
                }
                a0 += m[0] * y0 + m[1] * y1;
                a1 += m[2] * y0 + m[3] * y1;
            }
        }
        for (int o = P >> 1; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        }
        if (iPos >= 0 && part == 0) {
            const int slot = first - base + k;
            T v0 = ws[2 * slot] - a0, v1 = ws[2 * slot + 1] - a1;
            if (DIR == 1) {   // times the inverted pivot stored in the row's diagonal slot
                const T t0 = v0, t1 = v1;
                v0 = d[0] * t0 + d[1] * t1;
                v1 = d[2] * t0 + d[3] * t1;
            }
            ws[2 * slot] = v0;
            ws[2 * slot + 1] = v1;
            w[(2 * (size_t)iPos) * S + s] = v0;
            w[(2 * (size_t)iPos + 1) * S + s] = v1;
        }
        __syncthreads();
    }
}

// The forward tail's prefix: for each region row, the entries whose columns lie outside the region (final before it
// starts), w_i -= L(i, c) w_c, one thread per (row, lane), lanes coalesced.
template <typename T>
__global__ void __launch_bounds__(256) solvePrefixKernel(DevNet net, DevBatch b, const T* lu, T* w, const int* pos,
                                                         int base, int nSlots, const int* rowStart) {
    const int s = blockIdx.y * 32 + threadIdx.x;
    const int k = blockIdx.x * 8 + threadIdx.y;
    if (k >= nSlots || s >= b.S || !regionSolving(b, s)) return;
    const size_t S = b.S;
    const int i = pos[base + k];
    const int q1 = rowStart[k];
    T w0 = w[(2 * (size_t)i) * S + s], w1 = w[(2 * (size_t)i + 1) * S + s];
#pragma unroll 2
    for (int q = net.lrowPtr[i]; q < q1; q++) {
        const int2 e = net.lrow[q];
        T m[4];
        ld4g(lu, e.x, S, s, m);
        const T y0 = w[(2 * (size_t)e.y) * S + s], y1 = w[(2 * (size_t)e.y + 1) * S + s];
        w0 -= m[0] * y0 + m[1] * y1;
        w1 -= m[2] * y0 + m[3] * y1;
    }
    w[(2 * (size_t)i) * S + s] = w0;
    w[(2 * (size_t)i + 1) * S + s] = w1;
}

template <typename T>
size_t regionBytes(int nSlots, int nLevels) {
    return (size_t)nSlots * 4 * sizeof(T) + (sizeof(T) == 4 ? (size_t)nSlots * 4 : 0) + (size_t)(nLevels + 1) * 4;
}

template <typename T>
void regionT(const DevNet& net, const DevBatch& b, T* lu, const Hybrid& h, cudaStream_t st) {
    dim3 blk(32, 8), grd((h.regionSlots + 7) / 8, b.S / 32);
    regionPrefixKernel<T><<<grd, blk, 0, st>>>(net, b, lu, h.regionSlots, h.regionTask);
    regionFactorKernel<T><<<b.S, REGION_THREADS, regionBytes<T>(h.regionSlots, h.factorTo - h.regionFrom), st>>>(
        net, b, lu, h.plan.levelPtr, h.regionFrom, h.factorTo, h.regionBase, h.regionSlots, h.regionTask);
}

template <typename T>
size_t solveRegionBytes(int nSlots, int nLevels) {
    return (2 * (size_t)nSlots + (nSlots & 1)) * sizeof(T) + (size_t)(nLevels + 1) * 4;
}

template <typename T>
void solveRegionT(const DevNet& net, const DevBatch& b, const T* lu, T* w, const Hybrid& h, int dir, cudaStream_t st) {
    if (dir == 0) {
        if (h.fwdRegionSlots <= 0) return;
        dim3 blk(32, 8), grd((h.fwdRegionSlots + 7) / 8, b.S / 32);
        solvePrefixKernel<T><<<grd, blk, 0, st>>>(net, b, lu, w, h.plan.fwdPos, h.fwdRegionBase, h.fwdRegionSlots,
                                                 h.fwdRegionStart);
        solveRegionKernel<T, 0><<<b.S, REGION_THREADS, solveRegionBytes<T>(h.fwdRegionSlots, h.plan.nFwd - h.fwdFrom),
                                  st>>>(net, b, lu, w, h.plan.fwdPtr, h.plan.fwdPos, h.fwdFrom, h.plan.nFwd,
                                        h.fwdRegionBase, h.fwdRegionSlots, h.lrowSlot, h.fwdRegionStart);
    } else {
        if (h.bwdRegionSlots <= 0) return;
        solveRegionKernel<T, 1><<<b.S, REGION_THREADS, solveRegionBytes<T>(h.bwdRegionSlots, h.bwdUntil), st>>>(
            net, b, lu, w, h.plan.bwdPtr, h.plan.bwdPos, 0, h.bwdUntil, 0, h.bwdRegionSlots, h.uSlot, nullptr);
    }
}

}  // namespace

void launchSolveRegion(const DevNet& net, const DevBatch& b, const Hybrid& h, bool fp32, int dir, cudaStream_t st) {
    if (fp32) solveRegionT<float>(net, b, b.lu32, b.w32, h, dir, st);
    else solveRegionT<double>(net, b, b.lu64, b.w64, h, dir, st);
}

cudaError_t prepareRegion(int nSlots, int nLevels) {
    cudaError_t e = cudaFuncSetAttribute(regionFactorKernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)regionBytes<double>(nSlots, nLevels));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(regionFactorKernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)regionBytes<float>(nSlots, nLevels));
}

void launchRegionFactor(const DevNet& net, const DevBatch& b, const Hybrid& h, bool fp32, cudaStream_t st) {
    if (h.regionSlots <= 0) return;
    if (fp32) regionT<float>(net, b, b.lu32, h, st);
    else regionT<double>(net, b, b.lu64, h, st);
}

}  // namespace olfb200
