// Kernels of the learned warm start: a message-passing graph network over the bus graph, BF16 weights and
// activations with FP32 accumulation.  The dense layers' GEMMs run on the fifth-generation tensor cores (tcgen05.mma,
// accumulators in tensor memory; gemmTcKernel); their weight gradients on mma.sync m16n8k16 tiles; CUDA-core gather
// kernels for the messages.  Every reduction runs in a fixed order, so forward and backward are deterministic.
//
// Shapes: M rows = samples x buses; feature widths K, N are multiples of 16 / 8 (<= 128).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>

#include "../../include/olfgpu_b200.h"

namespace olfb200 {
namespace gnn {

namespace {

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// ---------------------------------------------------------------------------------------------------------------
// Y[M x N] = [A1 | A2][M x (K1 + K2)] . W[(K1 + K2) x N] (+ bias), z = relu ? max(Y, 0) : Y, saved to saveZ when given;
// out = z (+ residual) to outB (bf16) and / or outF (fp32), on the fifth-generation tensor cores.
// A persistent CTA of 4 warps walks 128-row tiles (grid-stride).  W^T and the bias stay in shared memory; the tiles of
// [A1 | A2] stream through two shared-memory buffers with cp.async (16-byte copies, rows past M zero-filled), the next
// tile's copies in flight while the current tile multiplies and runs its epilogue.  Both operands use the K-major
// canonical layout without swizzle (8-row x 16-byte core matrices; between the two 8-column halves of a 16-wide K step
// LBO bytes, between 8-row groups SBO = 128 bytes); eight consecutive threads copy the eight rows of one core matrix,
// so their shared-memory writes fill one 128-byte line.  One thread issues the K / 16 MMAs (M = 128, N, K = 16,
// BF16 x BF16 -> FP32) into a tensor-memory accumulator of 128 lanes x N columns and commits them to an mbarrier;
// every warp then reads its 32 lanes (rows) with tcgen05.ld and writes 16 columns per 16-byte store.  The mbarrier
// wait is bounded: on timeout the CTA records it (gTcTimeouts), drains its copies, frees its tensor memory and leaves.
// The launch pads the dynamic shared memory so that no more CTAs share an SM than its 512 tensor-memory columns hold
// (N columns each): their allocations never wait on one another.
// ---------------------------------------------------------------------------------------------------------------
__device__ int gTcTimeouts = 0;

// Shared memory of one CTA: two A buffers (128 x K), W^T (N x K), the bias (N floats), the mbarrier and the
// tensor-memory address.
constexpr int tcSmemBytes(int K, int N) { return 2 * 128 * K * 2 + N * K * 2 + N * 4 + 16; }
// The dynamic shared memory a launch asks for: at least the tile's, and enough that at most 512 / columns CTAs fit
// on one SM (228 KB of shared memory, 1 KB reserved per CTA).
constexpr int tcLaunchSmem(int K, int N) {
    return tcSmemBytes(K, N) > 233472 / (512 / (N < 32 ? 32 : N) + 1) ? tcSmemBytes(K, N)
                                                                       : 233472 / (512 / (N < 32 ? 32 : N) + 1);
}

__device__ __forceinline__ void cpAsync16(uint32_t dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}

__device__ __forceinline__ uint32_t packBf2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

__device__ __forceinline__ uint32_t smemU32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Shared-memory matrix descriptor (K-major, no swizzle): start >> 4 at [0,14), LBO >> 4 at [16,30), SBO >> 4 at
// [32,46), descriptor version 1 at [46,48), base offset 0, layout type 0 (no swizzle) at [61,64).
__device__ __forceinline__ uint64_t ummaDesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A and B (bits 7-9, 10-12 = 1), both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24 (M = 128).
template <int N>
constexpr uint32_t ummaInstrDesc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ bool mbarWait(uint32_t mbar, uint32_t parity) {
    for (int i = 0; i < (1 << 22); i++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(mbar), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

template <int K1, int K2, int N>
__global__ void __launch_bounds__(128) gemmTcKernel(int M, const __nv_bfloat16* __restrict__ A1,
                                                    const __nv_bfloat16* __restrict__ A2,
                                                    const __nv_bfloat16* __restrict__ W, const float* __restrict__ bias,
                                                    int relu, const __nv_bfloat16* __restrict__ residual,
                                                    __nv_bfloat16* outB, float* outF, int ldo,
                                                    __nv_bfloat16* saveZ) {
    constexpr int K = K1 + K2;
    constexpr int KC = K / 8;                           // 16-byte chunks of a row
    constexpr int CL = KC < 4 ? KC : 4;                 // chunks of one row that a warp copies together
    constexpr int CH = KC / CL;
    constexpr int TMEM_COLS = N < 32 ? 32 : N;          // a power of two >= 32
    static_assert(K % 16 == 0 && K1 % 8 == 0 && N % 16 == 0 && N <= 256, "tcgen05 tile: K multiple of 16, N of 16");
    static_assert((TMEM_COLS & (TMEM_COLS - 1)) == 0, "tensor-memory allocation: a power of two columns");
    static_assert(tcSmemBytes(K, N) <= 227 * 1024, "tile does not fit the shared memory");
    extern __shared__ __align__(1024) unsigned char tcSmem[];
    // A buffer b: 128 x K, core matrix (row / 8, chunk) at (chunk * 16 + row / 8) * 128
    unsigned char* sB = tcSmem + 2 * 128 * K * 2;       // W^T, N x K, core matrix (n / 8, chunk) at (chunk * N / 8 + n / 8) * 128
    float* sBias = reinterpret_cast<float*>(sB + N * K * 2);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sBias + N);
    uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(mbar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles = (M + 127) / 128;
    const uint32_t sA0 = smemU32(tcSmem);
    auto copyTile = [&](int tile, int buf) {
        const int base = tile * 128;
        const uint32_t dst0 = sA0 + (uint32_t)(buf * 128 * K * 2);
#pragma unroll
        for (int it = 0; it < KC; it++) {
            const int i = it * 128 + tid;
            const int rest = (i >> 3) / CL;
            const int c = (rest % CH) * CL + (i >> 3) % CL, r = (rest / CH) * 8 + (i & 7);
            const bool valid = base + r < M;
            const size_t row = valid ? (size_t)(base + r) : 0;
            const __nv_bfloat16* src = c * 8 < K1 ? A1 + row * K1 + c * 8 : A2 + row * K2 + (c * 8 - K1);
            cpAsync16(dst0 + (uint32_t)((c * 16 + (r >> 3)) * 128 + (r & 7) * 16), src, valid);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    if (blockIdx.x < tiles) copyTile(blockIdx.x, 0);
    for (int i = tid; i < K * N; i += 128) {
        const int k = i / N, n = i % N;
        *reinterpret_cast<__nv_bfloat16*>(sB + ((k >> 3) * (N / 8) + (n >> 3)) * 128 + (n & 7) * 16 + (k & 7) * 2) = W[i];
    }
    for (int i = tid; i < N; i += 128) sBias[i] = bias ? bias[i] : 0.f;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smemU32(mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemU32(tmemSlot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmemSlot;
    uint32_t parity = 0;
    int buf = 0;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, buf ^= 1) {
        // the other buffer was read by the previous tile's MMAs, which have completed
        if (tile + (int)gridDim.x < tiles) {
            copyTile(tile + gridDim.x, buf ^ 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        // the tile's copies become visible to the tensor cores' reads
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = sA0 + (uint32_t)(buf * 128 * K * 2), b0 = smemU32(sB);
#pragma unroll
            for (int ks = 0; ks < K / 16; ks++) {
                const uint64_t da = ummaDesc(a0 + 2 * ks * 16 * 128, 16 * 128, 128);
                const uint64_t db = ummaDesc(b0 + 2 * ks * (N / 8) * 128, (N / 8) * 128, 128);
                asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                             "l"(da), "l"(db), "r"(ummaInstrDesc<N>()), "r"(ks > 0 ? 1u : 0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smemU32(mbar))
                         : "memory");
        }
        __syncwarp();
        const bool done = mbarWait(smemU32(mbar), parity);
        if (__syncthreads_or(!done)) {   // the whole CTA leaves together, its copies drained
            if (tid == 0) atomicAdd(&gTcTimeouts, 1);
            asm volatile("cp.async.wait_group 0;" ::: "memory");
            break;
        }
        parity ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int r = tile * 128 + warp * 32 + lane;
#pragma unroll
        for (int cb = 0; cb < N / 16; cb++) {
            uint32_t v[16];
            const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 16);
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                         "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                           "=r"(v[14]), "=r"(v[15])
                         : "r"(addr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (r >= M) continue;
            float f[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
                f[j] = __uint_as_float(v[j]) + sBias[cb * 16 + j];
                if (relu) f[j] = fmaxf(f[j], 0.f);
            }
            const size_t rowN = (size_t)r * N + cb * 16;
            if (saveZ) {
                uint4* z = reinterpret_cast<uint4*>(saveZ + rowN);
                z[0] = make_uint4(packBf2(f[0], f[1]), packBf2(f[2], f[3]), packBf2(f[4], f[5]), packBf2(f[6], f[7]));
                z[1] = make_uint4(packBf2(f[8], f[9]), packBf2(f[10], f[11]), packBf2(f[12], f[13]),
                                  packBf2(f[14], f[15]));
            }
            if (residual) {
                const uint4* rp = reinterpret_cast<const uint4*>(residual + rowN);
                const uint4 q[2] = {rp[0], rp[1]};
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const uint32_t w4[4] = {q[h].x, q[h].y, q[h].z, q[h].w};
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const float2 rv = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w4[j]));
                        f[h * 8 + 2 * j] += rv.x;
                        f[h * 8 + 2 * j + 1] += rv.y;
                    }
                }
            }
            const size_t rowO = (size_t)r * ldo + cb * 16;
            if (outB) {
                uint4* o = reinterpret_cast<uint4*>(outB + rowO);
                o[0] = make_uint4(packBf2(f[0], f[1]), packBf2(f[2], f[3]), packBf2(f[4], f[5]), packBf2(f[6], f[7]));
                o[1] = make_uint4(packBf2(f[8], f[9]), packBf2(f[10], f[11]), packBf2(f[12], f[13]),
                                  packBf2(f[14], f[15]));
            }
            if (outF) {
                float4* o = reinterpret_cast<float4*>(outF + rowO);
#pragma unroll
                for (int j = 0; j < 4; j++) o[j] = make_float4(f[4 * j], f[4 * j + 1], f[4 * j + 2], f[4 * j + 3]);
            }
        }
        // every warp's tensor-memory reads are done before the next tile's MMAs overwrite the accumulator
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

template <int K1, int K2, int N>
void launchGemmTc(int M, const __nv_bfloat16* a1, const __nv_bfloat16* a2, const __nv_bfloat16* w, const float* bias,
                  int relu, const __nv_bfloat16* res, __nv_bfloat16* ob, float* of, int ldo, __nv_bfloat16* sz,
                  cudaStream_t st) {
    constexpr int smem = tcLaunchSmem(K1 + K2, N);
    // CTAs resident on the device: per SM the fewest that the shared memory (228 KB, 1 KB reserved per CTA), the
    // tensor memory (512 columns), the registers (64 K, 8-register granules) and the threads (2048) allow
    static const int resident = [] {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaFuncSetAttribute(gemmTcKernel<K1, K2, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
                cudaSuccess ||
            cudaFuncSetAttribute(gemmTcKernel<K1, K2, N>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared) != cudaSuccess)
            return -1;
        cudaFuncAttributes fa{};
        if (cudaFuncGetAttributes(&fa, gemmTcKernel<K1, K2, N>) != cudaSuccess) return -1;
        const int regs = (fa.numRegs + 7) / 8 * 8;
        int perSm = 2048 / 128;
        perSm = std::min(perSm, 233472 / (smem + 1024));
        perSm = std::min(perSm, 512 / (N < 32 ? 32 : N));
        perSm = std::min(perSm, 65536 / (regs * 128));
        return sms * std::max(perSm, 1);
    }();
    if (resident < 0) throw std::runtime_error("tcgen05 GEMM set-up: shared-memory attribute refused");
    if (M <= 0) return;
    // 16-byte copies and stores: row pointers and the output stride must keep 16-byte alignment
    auto misaligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) != 0; };
    if (misaligned(a1) || (K2 > 0 && misaligned(a2)) || misaligned(res) || misaligned(ob) || misaligned(of) ||
        misaligned(sz) || (ob && ldo % 8 != 0) || (of && ldo % 4 != 0) || ldo < N)
        throw std::runtime_error("GEMM operands must be 16-byte aligned, ldo >= N and ldo * element size a multiple of 16");
    const long long tiles = (M + 127) / 128;
    const int grid = (int)(tiles < resident ? tiles : resident);
    gemmTcKernel<K1, K2, N><<<grid, 128, smem, st>>>(M, a1, a2, w, bias, relu, res, ob, of, ldo, sz);
}

// Partial weight gradients: chunk c of the rows contributes P_c[K x N] = [A1|A2]_c^T dZ_c and colsum(dZ_c); one CTA
// per chunk.  32-row slices stream through two shared-memory buffers with cp.async (16-byte copies, rows past the
// chunk zero-filled), the next slice in flight while the tensor-core tiles (m over K, n over N, k over rows) consume
// the current one.
template <int K1, int K2, int N>
__global__ void __launch_bounds__(128) gemmDwKernel(int M, int rowsPerChunk, const __nv_bfloat16* __restrict__ A1,
                                                    const __nv_bfloat16* __restrict__ A2,
                                                    const __nv_bfloat16* __restrict__ dZ, float* partial) {
    constexpr int K = K1 + K2;
    constexpr int MT = K / 16, NT = N / 8, TILES = MT * NT;
    constexpr int PER_WARP = (TILES + 3) / 4;
    constexpr int SR = 32;                              // rows per slice
    __shared__ __align__(16) __nv_bfloat16 as[2][SR][K + 8];
    __shared__ __align__(16) __nv_bfloat16 ds[2][SR][N + 8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int row0 = blockIdx.x * rowsPerChunk;
    const int row1 = min(M, row0 + rowsPerChunk);
    auto stage = [&](int base, int buf) {
        for (int i = threadIdx.x; i < SR * (K / 8); i += 128) {
            const int r = i / (K / 8), c = i % (K / 8), row = base + r;
            const bool valid = row < row1;
            const size_t rr = valid ? (size_t)row : (size_t)row0;
            const __nv_bfloat16* src = c * 8 < K1 ? A1 + rr * K1 + c * 8 : A2 + rr * K2 + (c * 8 - K1);
            cpAsync16(smemU32(&as[buf][r][c * 8]), src, valid);
        }
        for (int i = threadIdx.x; i < SR * (N / 8); i += 128) {
            const int r = i / (N / 8), c = i % (N / 8), row = base + r;
            const bool valid = row < row1;
            cpAsync16(smemU32(&ds[buf][r][c * 8]), dZ + (valid ? (size_t)row : (size_t)row0) * N + c * 8, valid);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    float acc[PER_WARP][4];
#pragma unroll
    for (int i = 0; i < PER_WARP; i++) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
    float colsum = 0.f;   // thread tid < N sums column tid of dZ
    if (row0 < row1) stage(row0, 0);
    int buf = 0;
    for (int base = row0; base < row1; base += SR, buf ^= 1) {
        // the other buffer was consumed in the previous slice, before its closing barrier
        if (base + SR < row1) {
            stage(base + SR, buf ^ 1);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        if (threadIdx.x < N) {
            for (int r = 0; r < SR; r++) colsum += __bfloat162float(ds[buf][r][threadIdx.x]);
        }
#pragma unroll
        for (int s0 = 0; s0 < SR; s0 += 16) {
            const __nv_bfloat16(*a16)[K + 8] = &as[buf][s0];
            const __nv_bfloat16(*d16)[N + 8] = &ds[buf][s0];
#pragma unroll
            for (int i = 0; i < PER_WARP; i++) {
                const int tile = warp * PER_WARP + i;
                if (tile >= TILES) break;
                const int m0 = (tile / NT) * 16, n0 = (tile % NT) * 8;
                uint32_t a[4], b[2];
                // A_mma(m, kk) = a16[kk][m0 + m]; B_mma(kk, n) = d16[kk][n0 + n]
                a[0] = pack2(a16[2 * t][m0 + g], a16[2 * t + 1][m0 + g]);
                a[1] = pack2(a16[2 * t][m0 + g + 8], a16[2 * t + 1][m0 + g + 8]);
                a[2] = pack2(a16[2 * t + 8][m0 + g], a16[2 * t + 9][m0 + g]);
                a[3] = pack2(a16[2 * t + 8][m0 + g + 8], a16[2 * t + 9][m0 + g + 8]);
                b[0] = pack2(d16[2 * t][n0 + g], d16[2 * t + 1][n0 + g]);
                b[1] = pack2(d16[2 * t + 8][n0 + g], d16[2 * t + 9][n0 + g]);
                mma16816(acc[i], a, b);
            }
        }
        __syncthreads();
    }
    float* out = partial + (size_t)blockIdx.x * (K * N + N);
#pragma unroll
    for (int i = 0; i < PER_WARP; i++) {
        const int tile = warp * PER_WARP + i;
        if (tile >= TILES) break;
        const int m0 = (tile / NT) * 16, n0 = (tile % NT) * 8;
        out[(m0 + g) * N + n0 + 2 * t] = acc[i][0];
        out[(m0 + g) * N + n0 + 2 * t + 1] = acc[i][1];
        out[(m0 + g + 8) * N + n0 + 2 * t] = acc[i][2];
        out[(m0 + g + 8) * N + n0 + 2 * t + 1] = acc[i][3];
    }
    if (threadIdx.x < N) out[K * N + threadIdx.x] = colsum;
}

// dW[K x N], db[N] = sums of the chunk partials in chunk order.
__global__ void reducePartialsKernel(int chunks, int KN, int N, const float* partial, float* dW, float* db) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= KN + N) return;
    float s = 0.f;
    for (int c = 0; c < chunks; c++) s += partial[(size_t)c * (KN + N) + i];
    if (i < KN) dW[i] = s;
    else if (db) db[i - KN] = s;
}

// Messages into bus i of sample b: agg[b, i] = sum over directed edges e = (j -> i) of
// relu(P[b, j] + Q[b, i] + C[e] + bmsg), the edge dropped in the sample whose outaged branch it belongs to.
// PQ rows hold [P | Q] (128 features).  One warp per (sample, bus), two features per lane.
__global__ void messageForwardKernel(int B, int nb, const int* inPtr, const int* inEdge, const int* edgeSrc,
                                     const int* edgeBranch, const int* outage, const __nv_bfloat16* PQ, const float* C,
                                     const float* bmsg, __nv_bfloat16* agg) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= B * nb) return;
    const int b = warp / nb, i = warp % nb;
    const int f = 2 * lane;
    // each lane owns a feature pair: one 4-byte bf16x2 / 8-byte float2 access per row (a warp reads 128 / 256 bytes)
    const float2 q = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(PQ + ((size_t)b * nb + i) * 128 + 64 + f));
    const float2 bm = *reinterpret_cast<const float2*>(bmsg + f);
    const float q0 = q.x + bm.x, q1 = q.y + bm.y;
    float a0 = 0.f, a1 = 0.f;
    const int out = outage[b];
    const int p1 = inPtr[i + 1];
    for (int p = inPtr[i]; p < p1; p++) {
        const int e = inEdge[p];
        if (edgeBranch[e] == out) continue;
        const float2 pj = __bfloat1622float2(
            *reinterpret_cast<const __nv_bfloat162*>(PQ + ((size_t)b * nb + edgeSrc[e]) * 128 + f));
        const float2 c = *reinterpret_cast<const float2*>(C + (size_t)e * 64 + f);
        a0 += fmaxf(pj.x + q0 + c.x, 0.f);
        a1 += fmaxf(pj.y + q1 + c.y, 0.f);
    }
    *reinterpret_cast<__nv_bfloat162*>(agg + ((size_t)b * nb + i) * 64 + f) = __floats2bfloat162_rn(a0, a1);
}

// The same messages for a compact set of rows (sample rowSample[r], bus rowNode[r]): the buses within reach of each
// sample's outage.  A neighbour j outside the set takes its P row from PQbase (the outage-free sample, identical there);
// inside, from PQ at rowOf[sample * nb + j].  Same edges, same order, same arithmetic as messageForwardKernel.
__global__ void messageForwardCompactKernel(int R, int nb, const int* rowNode, const int* rowSample, const int* rowOf,
                                            const int* inPtr, const int* inEdge, const int* edgeSrc,
                                            const int* edgeBranch, const int* outage, const __nv_bfloat16* PQ,
                                            const __nv_bfloat16* PQbase, const float* C, const float* bmsg,
                                            __nv_bfloat16* agg) {
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (r >= R) return;
    const int i = rowNode[r], b = rowSample[r];
    const int f = 2 * lane;
    const float2 q = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(PQ + (size_t)r * 128 + 64 + f));
    const float2 bm = *reinterpret_cast<const float2*>(bmsg + f);
    const float q0 = q.x + bm.x, q1 = q.y + bm.y;
    float a0 = 0.f, a1 = 0.f;
    const int out = outage[b];
    const int p1 = inPtr[i + 1];
    for (int p = inPtr[i]; p < p1; p++) {
        const int e = inEdge[p];
        if (edgeBranch[e] == out) continue;
        const int j = edgeSrc[e];
        const int rj = rowOf[(size_t)b * nb + j];
        const __nv_bfloat16* src = rj >= 0 ? PQ + (size_t)rj * 128 : PQbase + (size_t)j * 128;
        const float2 pj = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(src + f));
        const float2 c = *reinterpret_cast<const float2*>(C + (size_t)e * 64 + f);
        a0 += fmaxf(pj.x + q0 + c.x, 0.f);
        a1 += fmaxf(pj.y + q1 + c.y, 0.f);
    }
    *reinterpret_cast<__nv_bfloat162*>(agg + (size_t)r * 64 + f) = __floats2bfloat162_rn(a0, a1);
}

// Backward of the messages.  dQ[b, i] = sum over e into i of g_e; dP[b, j] = sum over e out of j of g_e, with
// g_e = dAgg[b, dst(e)] * [pre_e > 0] recomputed from the saved P, Q.  Written into dPQ [rows x 128] (fp32).
__global__ void messageBackwardNodesKernel(int B, int nb, const int* inPtr, const int* inEdge, const int* outPtr,
                                           const int* outEdge, const int* edgeSrc, const int* edgeDst,
                                           const int* edgeBranch, const int* outage, const __nv_bfloat16* PQ,
                                           const float* C, const float* bmsg, const float* dAgg, float* dPQ) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= B * nb) return;
    const int b = warp / nb, v = warp % nb;
    const int f = 2 * lane;
    const int out = outage[b];
    const size_t rowV = (size_t)b * nb + v;
    // as destination: dQ[v]
    {
        const float q0 = __bfloat162float(PQ[rowV * 128 + 64 + f]) + bmsg[f];
        const float q1 = __bfloat162float(PQ[rowV * 128 + 64 + f + 1]) + bmsg[f + 1];
        const float d0 = dAgg[rowV * 64 + f], d1 = dAgg[rowV * 64 + f + 1];
        float s0 = 0.f, s1 = 0.f;
        for (int p = inPtr[v]; p < inPtr[v + 1]; p++) {
            const int e = inEdge[p];
            if (edgeBranch[e] == out) continue;
            const size_t pj = ((size_t)b * nb + edgeSrc[e]) * 128 + f;
            if (__bfloat162float(PQ[pj]) + q0 + C[(size_t)e * 64 + f] > 0.f) s0 += d0;
            if (__bfloat162float(PQ[pj + 1]) + q1 + C[(size_t)e * 64 + f + 1] > 0.f) s1 += d1;
        }
        dPQ[rowV * 128 + 64 + f] = s0;
        dPQ[rowV * 128 + 64 + f + 1] = s1;
    }
    // as source: dP[v]
    {
        const float p0 = __bfloat162float(PQ[rowV * 128 + f]), p1 = __bfloat162float(PQ[rowV * 128 + f + 1]);
        float s0 = 0.f, s1 = 0.f;
        for (int p = outPtr[v]; p < outPtr[v + 1]; p++) {
            const int e = outEdge[p];
            if (edgeBranch[e] == out) continue;
            const size_t rowI = (size_t)b * nb + edgeDst[e];
            const float pre0 = p0 + __bfloat162float(PQ[rowI * 128 + 64 + f]) + bmsg[f] + C[(size_t)e * 64 + f];
            const float pre1 = p1 + __bfloat162float(PQ[rowI * 128 + 64 + f + 1]) + bmsg[f + 1] + C[(size_t)e * 64 + f + 1];
            if (pre0 > 0.f) s0 += dAgg[rowI * 64 + f];
            if (pre1 > 0.f) s1 += dAgg[rowI * 64 + f + 1];
        }
        dPQ[rowV * 128 + f] = s0;
        dPQ[rowV * 128 + f + 1] = s1;
    }
}

// dC[e] = sum over samples of g_e (one warp per directed edge, two features per lane); dbmsg from the partials of
// dC summed over edges in edge order by the caller's reduction.
__global__ void messageBackwardEdgesKernel(int B, int nb, int nEdges, const int* edgeSrc, const int* edgeDst,
                                           const int* edgeBranch, const int* outage, const __nv_bfloat16* PQ,
                                           const float* C, const float* bmsg, const float* dAgg, float* dC) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= nEdges) return;
    const int e = warp, f = 2 * lane;
    const int j = edgeSrc[e], i = edgeDst[e];
    float s0 = 0.f, s1 = 0.f;
    for (int b = 0; b < B; b++) {
        if (edgeBranch[e] == outage[b]) continue;
        const size_t rj = ((size_t)b * nb + j) * 128, ri = ((size_t)b * nb + i) * 128;
        const float pre0 = __bfloat162float(PQ[rj + f]) + __bfloat162float(PQ[ri + 64 + f]) + bmsg[f] + C[(size_t)e * 64 + f];
        const float pre1 = __bfloat162float(PQ[rj + f + 1]) + __bfloat162float(PQ[ri + 64 + f + 1]) + bmsg[f + 1] +
                           C[(size_t)e * 64 + f + 1];
        const size_t ai = ((size_t)b * nb + i) * 64 + f;
        if (pre0 > 0.f) s0 += dAgg[ai];
        if (pre1 > 0.f) s1 += dAgg[ai + 1];
    }
    dC[(size_t)e * 64 + f] = s0;
    dC[(size_t)e * 64 + f + 1] = s1;
}

// C[e] = Estatic[e] (4 features) . We[4 x 64] (fp32, edge-wise).
__global__ void edgeProjectKernel(int nEdges, const float* Es, const float* We, float* C) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nEdges * 64) return;
    const int e = i / 64, f = i % 64;
    float s = 0.f;
    for (int k = 0; k < 4; k++) s += Es[e * 4 + k] * We[k * 64 + f];
    C[i] = s;
}

// dWe[4 x 64] = Es^T dC, dbmsg[64] = column sums of dC.  One CTA per 8 columns: thread t sums the edges t, t + 256,
// t + 512, ... in that order (two 16-byte loads of dC and one of Es per edge), then a fixed-shape tree adds the 256
// partial sums, so the result does not depend on timing.
constexpr int EPB_THREADS = 256;
__global__ void __launch_bounds__(EPB_THREADS) edgeProjectBackwardKernel(int nEdges, const float* __restrict__ Es,
                                                                          const float* __restrict__ dC, float* dWe,
                                                                          float* dbmsg) {
    __shared__ float part[40][EPB_THREADS];   // (k, column) x thread
    const int t = threadIdx.x, f0 = blockIdx.x * 8;
    float acc[5][8] = {};
    for (int e = t; e < nEdges; e += EPB_THREADS) {
        const float4 es = *reinterpret_cast<const float4*>(Es + (size_t)e * 4);
        const float4 c0 = *reinterpret_cast<const float4*>(dC + (size_t)e * 64 + f0);
        const float4 c1 = *reinterpret_cast<const float4*>(dC + (size_t)e * 64 + f0 + 4);
        const float ev[4] = {es.x, es.y, es.z, es.w};
        const float cv[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
#pragma unroll
        for (int j = 0; j < 8; j++) {
#pragma unroll
            for (int k = 0; k < 4; k++) acc[k][j] = fmaf(ev[k], cv[j], acc[k][j]);
            acc[4][j] += cv[j];
        }
    }
#pragma unroll
    for (int k = 0; k < 5; k++)
#pragma unroll
        for (int j = 0; j < 8; j++) part[k * 8 + j][t] = acc[k][j];
    __syncthreads();
    for (int stride = EPB_THREADS / 2; stride > 0; stride >>= 1) {
        if (t < stride)
            for (int q = 0; q < 40; q++) part[q][t] += part[q][t + stride];
        __syncthreads();
    }
    if (t < 40) {
        const int k = t / 8, j = t % 8;
        if (k < 4) dWe[k * 64 + f0 + j] = part[t][0];
        else dbmsg[f0 + j] = part[t][0];
    }
}

// dz = dOut * [z > 0] (relu) or dOut, stored bf16 [M x N] from fp32 [M x ldd]; optionally adds dOut to accum.
__global__ void reluGradKernel(size_t count, int N, int ldd, const float* dOut, const __nv_bfloat16* z,
                               __nv_bfloat16* dz, float* dzF) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const size_t r = i / N;
    const int c = (int)(i % N);
    float v = dOut[r * ldd + c];
    if (z && __bfloat162float(z[i]) <= 0.f) v = 0.f;
    if (dz) dz[i] = __float2bfloat16(v);
    if (dzF) dzF[i] = v;
}

// Adam on fp32 master weights; writes the bf16 copy and the bf16 transpose (K x N -> N x K) the kernels read.
__global__ void adamKernel(int count, int K, int N, float* w, const float* grad, float* m, float* v, float lr,
                           float beta1, float beta2, float eps, float c1, float c2, __nv_bfloat16* wB,
                           __nv_bfloat16* wT) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gr = grad[i];
    const float mi = beta1 * m[i] + (1.f - beta1) * gr;
    const float vi = beta2 * v[i] + (1.f - beta2) * gr * gr;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wB) wB[i] = __float2bfloat16(wi);
    if (wT) {
        const int k = i / N, n = i % N;
        wT[n * K + k] = __float2bfloat16(wi);
    }
}

// Mean squared error over the first 2 columns of out [M x ldo] against target [M x 2]; dOut [M x ldo] (zero beyond
// column 1) and per-block partial sums of the squared error.
__global__ void mseKernel(int M, int ldo, const float* out, const float* target, float* dOut, float* partial,
                          float scale) {
    __shared__ float red[256];
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    float s = 0.f;
    if (r < M) {
        for (int c = 0; c < ldo; c++) {
            float d = 0.f;
            if (c < 2) {
                const float e = out[(size_t)r * ldo + c] - target[(size_t)r * 2 + c];
                s += e * e;
                d = 2.f * e * scale;
            }
            dOut[(size_t)r * ldo + c] = d;
        }
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// dst[r, dstCol0 + c] (+)= src[r, srcCol0 + c] for c < ncols (fp32).
__global__ void copyColsKernel(long long count, int ncols, const float* src, int lds, int srcCol0, float* dst, int ldd,
                               int dstCol0, int accumulate) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const long long r = i / ncols;
    const int c = (int)(i % ncols);
    const float v = src[r * lds + srcCol0 + c];
    float* d = dst + r * ldd + dstCol0 + c;
    *d = accumulate ? *d + v : v;
}


}  // namespace

}  // namespace gnn
}  // namespace olfb200

using namespace olfb200::gnn;

namespace {
thread_local std::string gnnError;

template <typename F>
int gnnGuard(F&& f) {
    try {
        gnnError.clear();
        f();
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error ") + cudaGetErrorString(e));
        return 0;
    } catch (const std::exception& e) {
        gnnError = e.what();
    }
    return -1;
}
}  // namespace

// Node inputs of the compact rows: row r copies the outage-free inputs of its bus (16 BF16 columns, 32 B) and, at an
// end of its scenario's outaged branch, sets the outage columns: flag 1 at column nFeat, the branch's base-case P and
// Q flow (flows[o][0..1]) at the next two, negated at the to end.  rowOf[sample * nb + bus] = r (the entries of the
// other buses are left as they are: -1, set by the caller).
__global__ void compactInputsKernel(int R, int nb, int nFeat, const int* rowNode, const int* rowSample,
                                    const int* outage, const int* branchFrom, const int* branchTo,
                                    const __nv_bfloat16* xBase, const float* flows, __nv_bfloat16* x, int* rowOf) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    const int b = rowNode[r];
    const int sample = rowSample[r];
    const int o = outage[sample];
    rowOf[(size_t)sample * nb + b] = r;
    const uint4* src = reinterpret_cast<const uint4*>(xBase + (size_t)b * 16);
    uint4 lo = src[0], hi = src[1];
    __nv_bfloat16 v[16];
    memcpy(v, &lo, 16);
    memcpy(v + 8, &hi, 16);
    const bool atFrom = b == branchFrom[o], atTo = b == branchTo[o];
    if (atFrom || atTo) {
        const float sign = atTo ? -1.0f : 1.0f;
        v[nFeat] = __float2bfloat16_rn(1.0f);
        v[nFeat + 1] = __float2bfloat16_rn(sign * flows[2 * o]);
        v[nFeat + 2] = __float2bfloat16_rn(sign * flows[2 * o + 1]);
    }
    memcpy(&lo, v, 16);
    memcpy(&hi, v + 8, 16);
    uint4* dst = reinterpret_cast<uint4*>(x + (size_t)r * 16);
    dst[0] = lo;
    dst[1] = hi;
}

// Learned start states of the buses in the compact set: x0[s][2b], x0[s][2b + 1] from the compact output row (the
// identity rows keep their targets, already written by the full composition).
__global__ void scatterStartKernel(int R, int nb, const int* rowNode, const int* rowSample, const float* pred, int ldp,
                                   double stdVm, double stdVa, const double* xBase, const unsigned char* identity,
                                   double* x0) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    const int b = rowNode[r];
    const size_t base = (size_t)rowSample[r] * 2 * nb;
    const float* o = pred + (size_t)r * ldp;
    if (!identity[2 * b]) x0[base + 2 * b] = xBase[2 * b] + (double)o[1] * stdVa;
    if (!identity[2 * b + 1]) x0[base + 2 * b + 1] = xBase[2 * b + 1] + (double)o[0] * stdVm;
}

// Start states from the network's output: per scenario s and bus b, x0[s][2b] (angle) = xBase + dVa * stdVa and
// x0[s][2b + 1] (magnitude) = xBase + dVm * stdVm, the identity rows (slack angle, PV magnitudes) at their targets.
__global__ void composeStartKernel(int nS, int nb, const float* pred, int ldp, long long sampleStride, double stdVm,
                                   double stdVa, const double* xBase, const unsigned char* identity,
                                   const double* target, double* x0) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int n = 2 * nb;
    if (tid >= (long long)nS * n) return;
    const int s = (int)(tid / n), r = (int)(tid % n), b = r >> 1;
    double v;
    if (identity[r]) {
        v = target[r];
    } else {
        const float* o = pred + (long long)s * sampleStride + (long long)b * ldp;
        v = xBase[r] + ((r & 1) ? (double)o[0] * stdVm : (double)o[1] * stdVa);
    }
    x0[tid] = v;
}

extern "C" const char* olfgpu_gnn_last_error(void) { return gnnError.c_str(); }

extern "C" int olfgpu_gnn_tc_timeouts(int* count) {
    return gnnGuard([&] {
        if (!count) throw std::runtime_error("null output");
        const cudaError_t e = cudaMemcpyFromSymbol(count, gTcTimeouts, sizeof(int));
        if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
    });
}

extern "C" int olfgpu_gnn_gemm(int M, int K1, int K2, int N, const void* A1, const void* A2, const void* W,
                               const float* bias, int relu, const void* residual, void* outBf16, float* outF32,
                               int ldo, void* saveZ, void* stream) {
    return gnnGuard([&] {
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        auto a1 = static_cast<const __nv_bfloat16*>(A1);
        auto a2 = static_cast<const __nv_bfloat16*>(A2);
        auto w = static_cast<const __nv_bfloat16*>(W);
        auto res = static_cast<const __nv_bfloat16*>(residual);
        auto ob = static_cast<__nv_bfloat16*>(outBf16);
        auto sz = static_cast<__nv_bfloat16*>(saveZ);
#define OLF_GEMM(a, b2, c) launchGemmTc<a, b2, c>(M, a1, a2, w, bias, relu, res, ob, outF32, ldo, sz, st)
        if (K1 == 16 && K2 == 0 && N == 64) OLF_GEMM(16, 0, 64);
        else if (K1 == 64 && K2 == 0 && N == 128) OLF_GEMM(64, 0, 128);
        else if (K1 == 64 && K2 == 64 && N == 64) OLF_GEMM(64, 64, 64);
        else if (K1 == 64 && K2 == 0 && N == 16) OLF_GEMM(64, 0, 16);
        else if (K1 == 128 && K2 == 0 && N == 64) OLF_GEMM(128, 0, 64);
        else throw std::runtime_error("unsupported GEMM shape");
#undef OLF_GEMM
    });
}

extern "C" int olfgpu_gnn_gemm_dw(int M, int K1, int K2, int N, const void* A1, const void* A2, const void* dZ,
                                  float* dW, float* db, float* partial, int maxChunks, void* stream) {
    return gnnGuard([&] {
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        int chunks = maxChunks < 1 ? 1 : maxChunks;
        int rows = (M + chunks - 1) / chunks;
        rows = (rows + 15) / 16 * 16;
        chunks = (M + rows - 1) / rows;
        auto a1 = static_cast<const __nv_bfloat16*>(A1);
        auto a2 = static_cast<const __nv_bfloat16*>(A2);
        auto dz = static_cast<const __nv_bfloat16*>(dZ);
        if ((reinterpret_cast<uintptr_t>(A1) | reinterpret_cast<uintptr_t>(A2) | reinterpret_cast<uintptr_t>(dZ)) & 15)
            throw std::runtime_error("weight-gradient operands must be 16-byte aligned");
#define OLF_DW(a, b2, c) gemmDwKernel<a, b2, c><<<chunks, 128, 0, st>>>(M, rows, a1, a2, dz, partial)
        if (K1 == 16 && K2 == 0 && N == 64) OLF_DW(16, 0, 64);
        else if (K1 == 64 && K2 == 0 && N == 128) OLF_DW(64, 0, 128);
        else if (K1 == 64 && K2 == 64 && N == 64) OLF_DW(64, 64, 64);
        else if (K1 == 64 && K2 == 0 && N == 16) OLF_DW(64, 0, 16);
        else throw std::runtime_error("unsupported weight-gradient shape");
#undef OLF_DW
        const int KN = (K1 + K2) * N;
        reducePartialsKernel<<<(KN + N + 255) / 256, 256, 0, st>>>(chunks, KN, N, partial, dW, db);
    });
}

extern "C" int olfgpu_gnn_message_forward(int B, int nb, const int* inPtr, const int* inEdge, const int* edgeSrc,
                                          const int* edgeBranch, const int* outage, const void* PQ, const float* C,
                                          const float* bmsg, void* agg, void* stream) {
    return gnnGuard([&] {
        const long long warps = (long long)B * nb;
        messageForwardKernel<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
            B, nb, inPtr, inEdge, edgeSrc, edgeBranch, outage, static_cast<const __nv_bfloat16*>(PQ), C, bmsg,
            static_cast<__nv_bfloat16*>(agg));
    });
}

extern "C" int olfgpu_gnn_message_backward(int B, int nb, int nEdges, const int* inPtr, const int* inEdge,
                                           const int* outPtr, const int* outEdge, const int* edgeSrc,
                                           const int* edgeDst, const int* edgeBranch, const int* outage,
                                           const void* PQ, const float* C, const float* bmsg, const float* dAgg,
                                           float* dPQ, float* dC, void* stream) {
    return gnnGuard([&] {
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const long long warps = (long long)B * nb;
        auto pq = static_cast<const __nv_bfloat16*>(PQ);
        messageBackwardNodesKernel<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, st>>>(
            B, nb, inPtr, inEdge, outPtr, outEdge, edgeSrc, edgeDst, edgeBranch, outage, pq, C, bmsg, dAgg, dPQ);
        messageBackwardEdgesKernel<<<(unsigned)(((long long)nEdges * 32 + 255) / 256), 256, 0, st>>>(
            B, nb, nEdges, edgeSrc, edgeDst, edgeBranch, outage, pq, C, bmsg, dAgg, dC);
    });
}

extern "C" int olfgpu_gnn_edge_project(int nEdges, const float* Es, const float* We, float* C, void* stream) {
    return gnnGuard([&] {
        edgeProjectKernel<<<(nEdges * 64 + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(nEdges, Es, We, C);
    });
}

extern "C" int olfgpu_gnn_edge_project_backward(int nEdges, const float* Es, const float* dC, float* dWe,
                                                float* dbmsg, void* stream) {
    return gnnGuard([&] {
        if ((reinterpret_cast<uintptr_t>(Es) | reinterpret_cast<uintptr_t>(dC)) & 15)
            throw std::runtime_error("edge features and their gradients must be 16-byte aligned");
        edgeProjectBackwardKernel<<<64 / 8, EPB_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(nEdges, Es, dC, dWe,
                                                                                                 dbmsg);
    });
}

extern "C" int olfgpu_gnn_relu_grad(long long count, int N, int ldd, const float* dOut, const void* z, void* dz,
                                    float* dzF32, void* stream) {
    return gnnGuard([&] {
        reluGradKernel<<<(unsigned)((count + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
            (size_t)count, N, ldd, dOut, static_cast<const __nv_bfloat16*>(z), static_cast<__nv_bfloat16*>(dz), dzF32);
    });
}

extern "C" int olfgpu_gnn_adam(int count, int K, int N, float* w, const float* grad, float* m, float* v, float lr,
                               float beta1, float beta2, float eps, int step, void* wBf16, void* wTBf16, void* stream) {
    return gnnGuard([&] {
        const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
        adamKernel<<<(count + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
            count, K, N, w, grad, m, v, lr, beta1, beta2, eps, c1, c2, static_cast<__nv_bfloat16*>(wBf16),
            static_cast<__nv_bfloat16*>(wTBf16));
    });
}

extern "C" int olfgpu_gnn_mse(int M, int ldo, const float* out, const float* target, float* dOut, float* partial,
                              void* stream) {
    return gnnGuard([&] {
        mseKernel<<<(M + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(M, ldo, out, target, dOut, partial,
                                                                                  1.f / (2.f * (float)M));
    });
}

extern "C" int olfgpu_gnn_copy_cols(int M, int ncols, const float* src, int lds, int srcCol0, float* dst, int ldd,
                                    int dstCol0, int accumulate, void* stream) {
    return gnnGuard([&] {
        const long long count = (long long)M * ncols;
        copyColsKernel<<<(unsigned)((count + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
            count, ncols, src, lds, srcCol0, dst, ldd, dstCol0, accumulate);
    });
}

extern "C" int olfgpu_gnn_compose_start(int nScenarios, int nb, const float* pred, int ldPred, double stdVm,
                                        double stdVa, const double* xBase, const unsigned char* identity,
                                        const double* target, double* x0, void* stream) {
    return gnnGuard([&] {
        const long long count = (long long)nScenarios * 2 * nb;
        composeStartKernel<<<(unsigned)((count + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
            nScenarios, nb, pred, ldPred, (long long)nb * ldPred, stdVm, stdVa, xBase, identity, target, x0);
    });
}

extern "C" int olfgpu_gnn_message_forward_compact(int R, int nb, const int* rowNode, const int* rowSample,
                                                  const int* rowOf, const int* inPtr, const int* inEdge,
                                                  const int* edgeSrc, const int* edgeBranch, const int* outage,
                                                  const void* PQ, const void* PQbase, const float* C,
                                                  const float* bmsg, void* agg, void* stream) {
    return gnnGuard([&] {
        if (R <= 0) return;
        messageForwardCompactKernel<<<(unsigned)(((long long)R * 32 + 255) / 256), 256, 0,
                                      static_cast<cudaStream_t>(stream)>>>(
            R, nb, rowNode, rowSample, rowOf, inPtr, inEdge, edgeSrc, edgeBranch, outage,
            static_cast<const __nv_bfloat16*>(PQ), static_cast<const __nv_bfloat16*>(PQbase), C, bmsg,
            static_cast<__nv_bfloat16*>(agg));
    });
}

extern "C" int olfgpu_gnn_compact_inputs(int R, int nb, int nFeat, const int* rowNode, const int* rowSample,
                                         const int* outage, const int* branchFrom, const int* branchTo,
                                         const void* xBase, const float* flows, void* x, int* rowOf, void* stream) {
    return gnnGuard([&] {
        if (R <= 0) return;
        if (nFeat < 0 || nFeat + 3 > 16) throw std::invalid_argument("outage columns outside the 16 input columns");
        compactInputsKernel<<<(R + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
            R, nb, nFeat, rowNode, rowSample, outage, branchFrom, branchTo, static_cast<const __nv_bfloat16*>(xBase),
            flows, static_cast<__nv_bfloat16*>(x), rowOf);
    });
}

extern "C" int olfgpu_gnn_compose_start_compact(int nScenarios, int nb, const float* predBase, const float* predRows,
                                                int ldPred, int R, const int* rowNode, const int* rowSample,
                                                double stdVm, double stdVa, const double* xBase,
                                                const unsigned char* identity, const double* target, double* x0,
                                                void* stream) {
    return gnnGuard([&] {
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const long long count = (long long)nScenarios * 2 * nb;
        // every scenario first takes the outage-free prediction, then its own rows
        composeStartKernel<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(nScenarios, nb, predBase, ldPred, 0,
                                                                            stdVm, stdVa, xBase, identity, target, x0);
        if (R > 0) {
            scatterStartKernel<<<(R + 255) / 256, 256, 0, st>>>(R, nb, rowNode, rowSample, predRows, ldPred, stdVm,
                                                                stdVa, xBase, identity, x0);
        }
    });
}
