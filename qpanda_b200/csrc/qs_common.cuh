// qs_common.cuh - shared definitions of the B200 state-vector backend.
//
// State layout in HBM: one contiguous array of 2^n interleaved complex
// amplitudes (float2 for complex64, double2 for complex128), amplitude index
// bit q = qubit q (the little-endian order of
// QPandaSDK/QuantumInstructionHandle/CPUQuantumGates.cpp).  A 16-byte vector
// holds two complex64 amplitudes or one complex128 amplitude.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/qpanda_b200.h"

#define QS_MAX_HOLES 40          // bit positions a kernel can hold fixed (>= max qubits)
#define QS_MAX_QUBITS 38
#define QS_SM_COUNT 148          // B200

// ------------------------------------------------------------------ errors
int qs_fail(int code, const char *fmt, ...);     // records the message, returns code
int qs_cuda_fail(cudaError_t e, const char *where);
void qs_clear_error();

#define QS_CUDA_TRY(expr)                                                  \
    do {                                                                   \
        cudaError_t _e = (expr);                                           \
        if (_e != cudaSuccess) return qs_cuda_fail(_e, #expr);             \
    } while (0)

// After a launch: catch configuration errors immediately.
#define QS_LAUNCH_CHECK(name)                                              \
    do {                                                                   \
        cudaError_t _e = cudaGetLastError();                               \
        if (_e != cudaSuccess) return qs_cuda_fail(_e, name);              \
    } while (0)

// ------------------------------------------------------------------ state
struct qs_state {
    int n = 0;
    int dtype = QS_C64;
    uint64_t N = 0;
    void *amp = nullptr;                 // device amplitudes
    cudaStream_t stream = nullptr;
    int device = 0;
    // Device scratch for reductions (partial sums, trees); grown on demand
    // and kept until qs_destroy.
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    // Small pinned host buffer for scalar results.
    void *pinned = nullptr;
    // Norm partials of fused passes (3 x fused grid doubles), on first use.
    double *fused_norm = nullptr;
    // Second state-size buffer of remapping plans (qs_plan_opts.remap), on first use.
    void *spare = nullptr;
    // Stream-ordered memory (qs_create_async): cudaMallocAsync / cudaFreeAsync
    // on `stream`, and an ordinary host buffer instead of pinned memory.
    bool stream_alloc = false;
    size_t amp_bytes() const { return N * (dtype == QS_C64 ? 8ull : 16ull); }
};

int qs_ensure_scratch(qs_state *s, size_t bytes);
int qs_dev_alloc(qs_state *s, size_t bytes, void **p);
void qs_dev_free(qs_state *s, void *p);
int qs_check_state(const qs_state *s);

// ------------------------------------------------------------------ index math
// Zero-bit insertion at an ascending list of positions: maps a compact index
// of the free bits to a full amplitude index whose listed bits are 0.
struct Holes {
    int k;
    uint64_t low[QS_MAX_HOLES];          // (1 << pos) - 1, ascending positions
};

__host__ __device__ inline uint64_t insert_holes(uint64_t x, const Holes &h)
{
#ifdef __CUDACC__
#pragma unroll 4
#endif
    for (int j = 0; j < h.k; ++j) {
        uint64_t lo = x & h.low[j];
        x = ((x & ~h.low[j]) << 1) | lo;
    }
    return x;
}

// Build Holes from a bit mask (positions = set bits, ascending).
inline Holes holes_from_mask(uint64_t mask)
{
    Holes h;
    h.k = 0;
    for (int b = 0; b < 64 && mask; ++b) {
        if (mask & (1ull << b)) {
            h.low[h.k++] = (1ull << b) - 1;
            mask &= ~(1ull << b);
        }
    }
    return h;
}

template <typename T> struct vec2;
template <> struct vec2<float> { typedef float2 type; };
template <> struct vec2<double> { typedef double2 type; };

// Grid size for a streaming kernel over `items` work items of `threads` each.
inline unsigned grid_for(uint64_t items, int threads, int blocks_per_sm = 16)
{
    uint64_t b = (items + threads - 1) / threads;
    uint64_t cap = (uint64_t)QS_SM_COUNT * blocks_per_sm;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (unsigned)b;
}

// ------------------------------------------------------------------ kernels API
// (qs_gates.cu)
int launch_pair(qs_state *s, uint64_t holes_mask, uint64_t cmask, uint64_t off0,
                uint64_t off1, const double m[8]);
int launch_quad(qs_state *s, int q0, int q1, uint64_t cmask, const double m[32]);
int launch_phase(qs_state *s, uint64_t mask, double re, double im);
int launch_fill_zero_state(qs_state *s);
