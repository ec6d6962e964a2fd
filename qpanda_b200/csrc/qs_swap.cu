// qs_swap.cu - the half-slice swap of sharded states (qs_sharded.cpp) as one
// kernel that reads and writes both sides in place.
//
// A swap of rank bit j with local position p exchanges, between the two
// shards that differ in rank bit j, the rows of 2^p amplitudes (2^(p+1)
// apart) that the shard with rank bit 0 holds at local bit p = 1 with the
// rows the other holds at local bit p = 0.  Element (row r, unit c) of one
// half trades places with the same element of the other: each element pair is
// read once and written once, by one thread, so the two halves need no
// staging buffer and no third copy.  The other side may be a peer GPU's
// memory (peer access enabled, or an IPC mapping of another process's shard):
// the loads and stores then cross NVLink inside this kernel, and the two
// shards' processes split the rows (or, for a single row, its units) so that
// each element pair is still touched by exactly one thread.
#include "qs_common.cuh"
#include "qs_swap.h"

namespace {

constexpr int kSwapThreads = 256;
constexpr int kInFlight = 4;

// Rows [r0, r0 + nr) x units [c0, c0 + 2^lcu) of two halves with the same
// pitch (bytes).  U: the 16- or 8-byte unit.
template <typename U>
__global__ void __launch_bounds__(kSwapThreads) k_swap_halves(char *a, char *b, uint64_t pitch, uint64_t r0,
                                                              uint64_t nr, uint64_t c0, int lcu)
{
    const uint64_t total = nr << lcu, mask = (1ull << lcu) - 1;
    const uint64_t stride = (uint64_t)gridDim.x * kSwapThreads;
    uint64_t i = (uint64_t)blockIdx.x * kSwapThreads + threadIdx.x;
    for (; i + (kInFlight - 1) * stride < total; i += kInFlight * stride) {
        U *pa[kInFlight], *pb[kInFlight];
        U x[kInFlight], y[kInFlight];
#pragma unroll
        for (int k = 0; k < kInFlight; ++k) {
            const uint64_t e = i + k * stride, off = (r0 + (e >> lcu)) * pitch + (c0 + (e & mask)) * sizeof(U);
            pa[k] = reinterpret_cast<U *>(a + off);
            pb[k] = reinterpret_cast<U *>(b + off);
            x[k] = *pa[k];
            y[k] = *pb[k];
        }
#pragma unroll
        for (int k = 0; k < kInFlight; ++k) {
            *pa[k] = y[k];
            *pb[k] = x[k];
        }
    }
    for (; i < total; i += stride) {
        const uint64_t off = (r0 + (i >> lcu)) * pitch + (c0 + (i & mask)) * sizeof(U);
        U *pa = reinterpret_cast<U *>(a + off), *pb = reinterpret_cast<U *>(b + off);
        const U x = *pa, y = *pb;
        *pa = y;
        *pb = x;
    }
}

int ilog2(uint64_t v)
{
    int l = 0;
    while ((1ull << l) < v) ++l;
    return l;
}

}  // namespace

int qs_launch_swap_halves(void *a, void *b, size_t width, size_t pitch, size_t r0, size_t nr, size_t c0,
                          size_t w, cudaStream_t stream)
{
    if (!a || !b || a == b) return qs_fail(QS_ERR_ARG, "swap: two distinct halves needed");
    if (!nr || !w) return QS_OK;
    const size_t unit = (width % 16 == 0 && c0 % 16 == 0 && w % 16 == 0 && pitch % 16 == 0 &&
                         (uintptr_t)a % 16 == 0 && (uintptr_t)b % 16 == 0) ? 16 : 8;
    const uint64_t ncu = w / unit;
    if (w % unit || c0 % unit || c0 + w > width || (ncu & (ncu - 1)) || (uintptr_t)a % 8 || (uintptr_t)b % 8)
        return qs_fail(QS_ERR_ARG, "swap: row part [%zu, +%zu) of %zu bytes is not a power-of-two count of units",
                       c0, w, width);
    const uint64_t total = (uint64_t)nr * ncu;
    const uint64_t want = (total + kSwapThreads - 1) / kSwapThreads;
    const unsigned grid = (unsigned)(want < (uint64_t)QS_SM_COUNT * 8 ? want : (uint64_t)QS_SM_COUNT * 8);
    char *pa = static_cast<char *>(a), *pb = static_cast<char *>(b);
    if (unit == 16)
        k_swap_halves<uint4><<<grid, kSwapThreads, 0, stream>>>(pa, pb, pitch, r0, nr, c0 / 16, ilog2(ncu));
    else
        k_swap_halves<uint2><<<grid, kSwapThreads, 0, stream>>>(pa, pb, pitch, r0, nr, c0 / 8, ilog2(ncu));
    QS_LAUNCH_CHECK("k_swap_halves");
    return QS_OK;
}
