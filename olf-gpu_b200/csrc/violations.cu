// Post-contingency limit-violation screening on the device (sa/olf_gpu_violations.cu:160-361): after a batched solve,
// every limited branch and bus of every scenario is compared with its limits on the states the context holds, and
// the candidates are handed to the host.  Like the reference's screen it does not decide: a limit is a candidate as
// soon as the value exceeds its threshold relaxed by `band` (relative), and a group's later limits stop being
// candidates once one is exceeded beyond the band (the host reports the first confirmed limit of a group); so the
// host's exact re-test on its own values sees every violation.
//
// Layout: branch limits as groups (side 1 / 2; quantity I = hypot(p, q) / v, P = |p|, S = sqrt(p^2 + q^2)) per
// limited element (a closed branch, or an open-ended branch evaluated with its connected side's terms), thresholds per
// group in the caller's order; bus limits as (V row, high, low); the realistic-voltage band over the same buses.  One
// thread per (element, lane) or (bus, lane), lanes coalesced.  A scenario's candidates are record ids appended through
// an atomic counter and sorted by the host, so the result does not depend on scheduling: branch limit l is l, bus i's
// high limit nLimits + 2i, its low limit nLimits + 2i + 1, its realistic-band exit nLimits + 2 nBus + i.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "engine.hpp"

namespace olfb200 {

namespace {

struct ViolationDev {
    int nElem, nLimits, nBus, capacity, realistic;
    double band, minV, maxV;
    const int *elemId, *elemCols, *groupPtr, *groupSide, *groupQty, *limPtr;
    const double* limThreshold;
    const int* busVRow;
    const double *busHigh, *busLow;
    int* records;
    int* counts;
};

enum { QTY_I = 0, QTY_P = 1, QTY_S = 2 };

__device__ __forceinline__ void emit(const ViolationDev& v, int s, int id) {
    const int k = atomicAdd(&v.counts[s], 1);
    if (k < v.capacity) v.records[(size_t)s * v.capacity + k] = id;
}

__device__ __forceinline__ bool live(const DevBatch& b, int s) { return s < b.nS && (!b.laneLive || b.laneLive[s]); }

// 32 lanes x 8 limited elements per CTA
__global__ void screenBranchesKernel(DevNet net, DevBatch b, ViolationDev v) {
    const int s = blockIdx.y * 32 + threadIdx.x;
    const int r = blockIdx.x * 8 + threadIdx.y;
    if (r >= v.nElem || !live(b, s)) return;
    const size_t S = b.S;
    const int e = v.elemId[r];
    const int words = b.S >> 5;
    if ((b.disabled[(size_t)e * words + (s >> 5)] >> (s & 31)) & 1u) return;   // out of service in this scenario
    const int* c = v.elemCols + 4 * (size_t)r;   // closed: ph1 v1 ph2 v2 columns; open: -1 v1 -1 v2 (-1: open side)
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    double p1 = nan, q1 = nan, p2 = nan, q2 = nan, v1 = nan, v2 = nan;
    if (e < net.ncb) {
        // closed_branch.cuh:161-229, the fill's terms
        const double* p = net.cbPar + (size_t)e * 8;
        const double y = p[0], g1 = p[1], g2 = p[2], b1 = p[3], b2 = p[4], ksi = p[5], r1 = p[6], a1 = p[7];
        const double2 tr = net.cbTrig[e];
        const double sk = tr.x, ck = tr.y;
        const double ph1 = b.x[(size_t)c[0] * S + s], ph2 = b.x[(size_t)c[2] * S + s];
        v1 = b.x[(size_t)c[1] * S + s];
        v2 = b.x[(size_t)c[3] * S + s];
        double s1, c1, s2, c2;
        sincos(ksi - a1 - ph1 + ph2, &s1, &c1);
        sincos(ksi + a1 + ph1 - ph2, &s2, &c2);
        p1 = r1 * v1 * (g1 * r1 * v1 + y * r1 * v1 * sk - y * v2 * s1);
        q1 = r1 * v1 * (-b1 * r1 * v1 + y * r1 * v1 * ck - y * v2 * c1);
        p2 = v2 * (g2 * v2 - y * r1 * v1 * s2 + y * v2 * sk);
        q2 = v2 * (-b2 * v2 - y * r1 * v1 * c2 + y * v2 * ck);
    } else {
        // open_branch.cuh:65-87: the connected side's flow
        const double* p = net.obPar + (size_t)(e - net.ncb) * 7;
        const double y = p[0], ksi = p[1], g1 = p[2], b1 = p[3], g2 = p[4], b2 = p[5], r1 = p[6];
        double sk, ck;
        sincos(ksi, &sk, &ck);
        if (c[1] >= 0) {   // side 2 open
            v1 = b.x[(size_t)c[1] * S + s];
            const double d2 = (g2 + y * sk) * (g2 + y * sk) + (-b2 + y * ck) * (-b2 + y * ck);
            const double gp1 = g1 + y * y * g2 / d2 + (b2 * b2 + g2 * g2) * y * sk / d2;
            const double bq1 = b1 + y * y * b2 / d2 - (b2 * b2 + g2 * g2) * y * ck / d2;
            p1 = r1 * r1 * v1 * v1 * gp1;
            q1 = -r1 * r1 * v1 * v1 * bq1;
        }
        if (c[3] >= 0) {   // side 1 open
            v2 = b.x[(size_t)c[3] * S + s];
            const double d1 = (g1 + y * sk) * (g1 + y * sk) + (-b1 + y * ck) * (-b1 + y * ck);
            const double gp2 = g2 + y * y * g1 / d1 + (b1 * b1 + g1 * g1) * y * sk / d1;
            const double bq2 = b2 + y * y * b1 / d1 - (b1 * b1 + g1 * g1) * y * ck / d1;
            p2 = v2 * v2 * gp2;
            q2 = -v2 * v2 * bq2;
        }
    }
    for (int g = v.groupPtr[r]; g < v.groupPtr[r + 1]; g++) {
        const bool one = v.groupSide[g] == 1;
        const double p = one ? p1 : p2, q = one ? q1 : q2, vv = one ? v1 : v2;
        double value;
        switch (v.groupQty[g]) {
            case QTY_I: value = hypot(p, q) / vv; break;
            case QTY_P: value = fabs(p); break;
            default: value = sqrt(p * p + q * q); break;
        }
        if (isnan(value)) continue;
        for (int l = v.limPtr[g]; l < v.limPtr[g + 1]; l++) {
            const double t = v.limThreshold[l];
            if (value > t - fabs(t) * v.band) {
                emit(v, s, l);
                if (value > t + fabs(t) * v.band) break;   // certainly reported here: the group's later limits never are
            }
        }
    }
}

// 32 lanes x 8 buses per CTA: high / low voltage limits (a NaN limit compares false) and the realistic band
__global__ void screenBusesKernel(DevBatch b, ViolationDev v) {
    const int s = blockIdx.y * 32 + threadIdx.x;
    const int i = blockIdx.x * 8 + threadIdx.y;
    if (i >= v.nBus || !live(b, s)) return;
    const int row = v.busVRow[i];
    if (row < 0) return;
    const double x = b.x[(size_t)row * b.S + s];
    const double hi = v.busHigh[i], lo = v.busLow[i];
    if (x > hi - fabs(hi) * v.band) emit(v, s, v.nLimits + 2 * i);
    if (x < lo + fabs(lo) * v.band) emit(v, s, v.nLimits + 2 * i + 1);
    if (v.realistic && (x < v.minV || x > v.maxV)) emit(v, s, v.nLimits + 2 * v.nBus + i);
}

}  // namespace

void screenViolations(BatchContext& ctx, const ViolationTables& t, int capacity, int* records, int* counts) {
    OLF_CUDA(cudaSetDevice(ctx.device));
    const Structure& s = ctx.net->host;
    if (capacity <= 0) throw std::runtime_error("capacity must be positive");
    if (t.nElem < 0 || t.nBus < 0) throw std::runtime_error("negative table size");
    const int nGroups = t.nElem > 0 ? t.groupPtr[t.nElem] : 0;
    const int nLimits = nGroups > 0 ? t.limPtr[nGroups] : 0;
    if (t.nElem > 0 && t.groupPtr[0] != 0) throw std::runtime_error("groupPtr must start at 0");
    if (nGroups > 0 && t.limPtr[0] != 0) throw std::runtime_error("limPtr must start at 0");
    // the limited elements' bus columns (closed: ph1 v1 ph2 v2; open: -1 v1 -1 v2 with -1 at the open side)
    std::vector<int> cols(static_cast<size_t>(std::max(t.nElem, 1)) * 4, -1);
    for (int r = 0; r < t.nElem; r++) {
        const int e = t.elemId[r];
        if (e < 0 || e >= s.ncb + s.nob) throw std::runtime_error("limited element " + std::to_string(e) + " is no branch");
        if (t.groupPtr[r + 1] < t.groupPtr[r]) throw std::runtime_error("groupPtr not ascending");
        if (e < s.ncb) {
            const int* ix = &s.cbIx[static_cast<size_t>(e) * CB_INDICES];
            for (int k = 0; k < 4; k++) cols[4 * r + k] = ix[4 + k];
            if (cols[4 * r] < 0 || cols[4 * r + 1] < 0 || cols[4 * r + 2] < 0 || cols[4 * r + 3] < 0) {
                throw std::runtime_error("closed branch " + std::to_string(e) + " lacks a state column");
            }
        } else {
            const int* ix = &s.obIx[static_cast<size_t>(e - s.ncb) * OB_INDICES];
            cols[4 * r + 1] = ix[4];
            cols[4 * r + 3] = ix[5];
        }
    }
    for (int g = 0; g < nGroups; g++) {
        if (t.groupSide[g] != 1 && t.groupSide[g] != 2) throw std::runtime_error("group side must be 1 or 2");
        if (t.groupQty[g] < QTY_I || t.groupQty[g] > QTY_S) throw std::runtime_error("group quantity must be 0, 1 or 2");
        if (t.limPtr[g + 1] < t.limPtr[g]) throw std::runtime_error("limPtr not ascending");
    }
    for (int i = 0; i < t.nBus; i++)
        if (t.busVRow[i] >= s.n) throw std::runtime_error("bus voltage row out of range");
    // one device block of every table (freed with the call)
    std::vector<char> blob;
    auto place = [&](const void* src, size_t bytes) {
        const size_t off = (blob.size() + 255) / 256 * 256;
        blob.resize(off + std::max<size_t>(bytes, 8));
        if (bytes && src) std::memcpy(blob.data() + off, src, bytes);
        return off;
    };
    const size_t oId = place(t.elemId, sizeof(int) * t.nElem), oCols = place(cols.data(), sizeof(int) * cols.size()),
                 oGp = place(t.groupPtr, sizeof(int) * (t.nElem > 0 ? t.nElem + 1 : 0)),
                 oGs = place(t.groupSide, sizeof(int) * nGroups), oGq = place(t.groupQty, sizeof(int) * nGroups),
                 oLp = place(t.limPtr, sizeof(int) * (nGroups > 0 ? nGroups + 1 : 0)),
                 oLt = place(t.limThreshold, sizeof(double) * nLimits), oBr = place(t.busVRow, sizeof(int) * t.nBus),
                 oBh = place(t.busHigh, sizeof(double) * t.nBus), oBl = place(t.busLow, sizeof(double) * t.nBus);
    const size_t oRec = place(nullptr, sizeof(int) * static_cast<size_t>(ctx.nS) * capacity);
    const size_t oCnt = place(nullptr, sizeof(int) * ctx.nS);
    DeviceBuffer dev;
    dev.alloc(blob.size());
    cudaStream_t st = ctx.stream;
    OLF_CUDA(cudaMemcpyAsync(dev.p, blob.data(), oRec, cudaMemcpyHostToDevice, st));
    OLF_CUDA(cudaMemsetAsync(static_cast<char*>(dev.p) + oCnt, 0, sizeof(int) * ctx.nS, st));
    char* base = static_cast<char*>(dev.p);
    ViolationDev v{};
    v.nElem = t.nElem;
    v.nLimits = nLimits;
    v.nBus = t.nBus;
    v.capacity = capacity;
    v.realistic = t.realistic;
    v.band = t.band;
    v.minV = t.minV;
    v.maxV = t.maxV;
    v.elemId = reinterpret_cast<const int*>(base + oId);
    v.elemCols = reinterpret_cast<const int*>(base + oCols);
    v.groupPtr = reinterpret_cast<const int*>(base + oGp);
    v.groupSide = reinterpret_cast<const int*>(base + oGs);
    v.groupQty = reinterpret_cast<const int*>(base + oGq);
    v.limPtr = reinterpret_cast<const int*>(base + oLp);
    v.limThreshold = reinterpret_cast<const double*>(base + oLt);
    v.busVRow = reinterpret_cast<const int*>(base + oBr);
    v.busHigh = reinterpret_cast<const double*>(base + oBh);
    v.busLow = reinterpret_cast<const double*>(base + oBl);
    v.records = reinterpret_cast<int*>(base + oRec);
    v.counts = reinterpret_cast<int*>(base + oCnt);
    const DevBatch b = ctx.batch();
    const DevNet& net = ctx.dn->view;
    if (t.nElem > 0) screenBranchesKernel<<<dim3((t.nElem + 7) / 8, ctx.S / 32), dim3(32, 8), 0, st>>>(net, b, v);
    if (t.nBus > 0) screenBusesKernel<<<dim3((t.nBus + 7) / 8, ctx.S / 32), dim3(32, 8), 0, st>>>(b, v);
    OLF_CUDA(cudaGetLastError());
    std::vector<int> rec(static_cast<size_t>(ctx.nS) * capacity), cnt(ctx.nS);
    OLF_CUDA(cudaMemcpyAsync(rec.data(), v.records, rec.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    OLF_CUDA(cudaMemcpyAsync(cnt.data(), v.counts, cnt.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    OLF_CUDA(cudaStreamSynchronize(st));
    for (int sc = 0; sc < ctx.nS; sc++) {
        int* row = rec.data() + static_cast<size_t>(sc) * capacity;
        std::sort(row, row + std::min(cnt[sc], capacity));
    }
    if (records) std::memcpy(records, rec.data(), rec.size() * sizeof(int));
    if (counts) std::memcpy(counts, cnt.data(), cnt.size() * sizeof(int));
}

}  // namespace olfb200
