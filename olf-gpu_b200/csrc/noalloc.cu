// A batched linear solve that allocates nothing: its scratch (the Jacobian blocks, the block-LU factors, the solve
// work vectors and the lane flags) lives in one file-scope device array of fixed size, and the caller hands in device
// buffers for the inputs and the output.  Declared in include/olfgpu_b200.h (olfgpu_linear_solve_noalloc).
//
// Shared-scratch rules: every call on a device uses the same array, which keeps the previous call's contents (this
// file clears what must start at zero on every call), and two calls whose work overlaps on the GPU -- on different
// streams, or from different host threads -- race on it.  Calls must be ordered (one stream, or synchronised).
#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/olfgpu_b200.h"
#include "engine.hpp"

namespace olfb200 {

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(64) << 20;   // 64 MiB, held by every GPU that loads the library

__device__ __align__(256) unsigned char gNoAllocScratch[NOALLOC_SCRATCH_BYTES];

// The array's device address, looked up with the device current (the symbol's host-side name is a stand-in, not a
// device address: it is never handed to a kernel).  The lookup is cached per device and per CUDA context: after the
// device's context is destroyed and re-created (cudaDeviceReset), the module is loaded again and the array may sit
// elsewhere, so a new context means a new lookup.  The current context comes from the driver's cuCtxGetCurrent,
// reached through the runtime's entry-point query (the library does not link the driver library itself).
std::mutex gScratchMutex;
struct ScratchSlot {
    void* context = nullptr;
    void* address = nullptr;
};
ScratchSlot gScratch[128];

void* currentContext() {
    using CtxGetCurrent = int (*)(void**);
    static CtxGetCurrent fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            f = nullptr;
        }
        return reinterpret_cast<CtxGetCurrent>(f);
    }();
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0 || !ctx) throw std::runtime_error("no current CUDA context for the no-allocation solve");
    return ctx;
}

void* scratchAddress(int device) {
    if (device < 0 || device >= 128) throw std::runtime_error("device ordinal out of range");
    void* ctx = currentContext();
    std::lock_guard<std::mutex> lock(gScratchMutex);
    ScratchSlot& slot = gScratch[device];
    if (slot.context != ctx || !slot.address) {
        void* p = nullptr;
        const cudaError_t err = cudaGetSymbolAddress(&p, gNoAllocScratch);
        if (err != cudaSuccess || p == nullptr) {
            throw std::runtime_error(std::string("cudaGetSymbolAddress of the no-allocation scratch failed: ") +
                                     cudaGetErrorString(err));
        }
        slot.context = ctx;
        slot.address = p;
    }
    return slot.address;
}

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

// Byte offsets of the scratch regions for S lanes.
struct ScratchLayout {
    size_t J, lu, w, dx, F, active, pending, trouble, total;
};

ScratchLayout layoutFor(const DevNet& net, size_t S, bool fp32) {
    ScratchLayout l{};
    size_t o = 0;
    l.J = o;
    o = align256(o + static_cast<size_t>(net.nA) * 4 * S * 8);
    l.lu = o;
    o = align256(o + static_cast<size_t>(net.nLu) * 4 * S * (fp32 ? 4 : 8));
    l.w = o;
    o = align256(o + static_cast<size_t>(net.nb) * 2 * S * (fp32 ? 4 : 8));
    l.dx = o;
    o = align256(o + static_cast<size_t>(net.n) * S * 8);
    l.F = o;
    o = align256(o + static_cast<size_t>(net.n) * S * 8);
    l.active = o;
    o = align256(o + S);
    l.pending = o;
    o = align256(o + S);
    l.trouble = o;
    o = align256(o + S * 4);
    l.total = o;
    return l;
}

// CSR values [nS][nnz] (scenario-major) -> Jacobian blocks [nA][4][S]; rhs [nS][n] -> F = -rhs [n][S]; lane flags.
__global__ void noallocInstallKernel(const int* csrToA, const double* csrVals, const double* rhs, int nnz, int n,
                                     int nS, int S, double* J, double* F, int8_t* active, int8_t* pending, int* trouble) {
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t cells = (size_t)nnz * nS;
    if (tid < cells) {
        const int s = (int)(tid % nS), k = (int)(tid / nS);
        J[(size_t)csrToA[k] * S + s] = csrVals[(size_t)s * nnz + k];
    }
    if (tid < (size_t)n * nS) {
        const int s = (int)(tid % nS), r = (int)(tid / nS);
        F[(size_t)r * S + s] = -rhs[(size_t)s * n + r];
    }
    if (tid < (size_t)S) {
        active[tid] = tid < (size_t)nS ? 1 : 0;
        pending[tid] = 0;
        trouble[tid] = 0;
    }
}

// Solution [n][S] -> out [nS][n]; a scenario whose factorization met a (near-)singular 2x2 pivot gets NaN throughout,
// so a failed solve never passes for an answer.
__global__ void noallocGatherKernel(const double* dx, const int* trouble, double* out, int n, int nS, int S) {
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (size_t)n * nS) return;
    const int r = (int)(tid % n), s = (int)(tid / n);
    out[(size_t)s * n + r] = trouble[s] ? __longlong_as_double(0x7ff8000000000000LL) : dx[(size_t)r * S + s];
}

}  // namespace

void linearSolveNoAlloc(const std::shared_ptr<NetStructure>& net, int nScenarios, const double* csrVals,
                        const double* rhs, double* out, int precision, cudaStream_t st) {
    if (nScenarios <= 0) throw std::runtime_error("nScenarios must be positive");
    if (!csrVals || !rhs || !out) throw std::runtime_error("null device buffer");
    if (precision != 0 && precision != 1) throw std::runtime_error("precision must be 0 (FP64) or 1 (FP32)");
    int device = 0;
    OLF_CUDA(cudaGetDevice(&device));
    const std::shared_ptr<DeviceNet> dnp = net->find(device);
    if (!dnp) {
        throw std::runtime_error("the structure is not resident on the current device: create a batch context on it "
                                 "first (that call uploads the structure)");
    }
    const DeviceNet& dn = *dnp;
    const DevNet& v = dn.view;
    const bool fp32 = precision == 1;
    const size_t S = static_cast<size_t>((nScenarios + 31) / 32 * 32);
    const ScratchLayout lay = layoutFor(v, S, fp32);
    if (lay.total > NOALLOC_SCRATCH_BYTES) {
        size_t fit = 0;
        for (size_t s2 = 32; layoutFor(v, s2, fp32).total <= NOALLOC_SCRATCH_BYTES; s2 += 32) fit = s2;
        throw std::runtime_error("batch of " + std::to_string(nScenarios) + " scenarios needs " +
                                 std::to_string(lay.total) + " bytes of scratch; the no-allocation solve holds " +
                                 std::to_string(NOALLOC_SCRATCH_BYTES) + " bytes (at most " + std::to_string(fit) +
                                 " scenarios of this structure)");
    }
    unsigned char* base = static_cast<unsigned char*>(scratchAddress(device));
    DevBatch b{};
    b.S = static_cast<int>(S);
    b.nS = nScenarios;
    b.J = reinterpret_cast<double*>(base + lay.J);
    b.lu64 = fp32 ? nullptr : reinterpret_cast<double*>(base + lay.lu);
    b.lu32 = fp32 ? reinterpret_cast<float*>(base + lay.lu) : nullptr;
    b.w64 = fp32 ? nullptr : reinterpret_cast<double*>(base + lay.w);
    b.w32 = fp32 ? reinterpret_cast<float*>(base + lay.w) : nullptr;
    b.dx = reinterpret_cast<double*>(base + lay.dx);
    b.F = reinterpret_cast<double*>(base + lay.F);
    b.active = reinterpret_cast<int8_t*>(base + lay.active);
    b.pending = reinterpret_cast<int8_t*>(base + lay.pending);
    b.trouble = reinterpret_cast<int*>(base + lay.trouble);
    // the Jacobian blocks keep the previous call's values: blocks entries outside the CSR pattern must read zero
    OLF_CUDA(cudaMemsetAsync(b.J, 0, static_cast<size_t>(v.nA) * 4 * S * 8, st));
    const size_t cells = std::max<size_t>(std::max<size_t>(static_cast<size_t>(net->host.nnz) * nScenarios,
                                                           static_cast<size_t>(v.n) * nScenarios), S);
    noallocInstallKernel<<<(unsigned)((cells + 255) / 256), 256, 0, st>>>(
        dn.csrToAD.as<int>(), csrVals, rhs, net->host.nnz, v.n, nScenarios, static_cast<int>(S), b.J, b.F, b.active,
        b.pending, b.trouble);
    launchFactor(v, b, dn.levelPtr.data(), dn.levelSplit.data(), static_cast<int>(dn.levelPtr.size()) - 1, fp32,
                 nullptr, st);
    launchSolve(v, b, dn.fwd(), dn.bwd(), fp32, false, nullptr, st);
    const size_t outCells = static_cast<size_t>(v.n) * nScenarios;
    noallocGatherKernel<<<(unsigned)((outCells + 255) / 256), 256, 0, st>>>(b.dx, b.trouble, out, v.n, nScenarios,
                                                                           static_cast<int>(S));
    OLF_CUDA(cudaGetLastError());
}

}  // namespace olfb200
