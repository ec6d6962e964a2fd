// qs_noalloc.cu - qubit measurement that allocates no memory.
//
// qs_measure (qs_measure.cu) keeps its reduction partials in the state's
// scratch buffer, which qs_create allocates with cudaMalloc.  Some callers
// cannot allocate at the point where they want to measure: a serving engine
// that reserves all HBM up front and forbids allocation on its hot path, a
// framework whose caching allocator owns the device memory and must not see
// cudaMalloc/cudaFree behind its back, or code that holds a state vector in a
// buffer it allocated itself and has no qs_state at all.  qs_measure_noalloc
// serves them: the caller passes the amplitudes and two device output words,
// and the partial sums live in a fixed array compiled into this library.
//
// The array (g_noalloc_scratch, 512 KB + 256 B) exists on every GPU that
// loads the library, from module load until process exit.  It holds one
// partial sum per 2^16 amplitudes, which caps the state at 32 qubits.  All
// calls on a device share it and it keeps the last call's contents: every
// partial a call reads was written by that same call, so nothing needs
// clearing, but calls that overlap on the GPU (different streams without an
// ordering between them) race on the array.
#include <mutex>

#include "qs_common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kChunkBits = 16;                     // amplitudes per partial: 2^16
constexpr int kMaxPartials = 1 << 16;              // => states up to 2^32 amplitudes
constexpr int kMaxQubits = kChunkBits + 16;        // 32

struct NaResult {
    double p0;
    double scale;
    int outcome;
    int status;
};

// partials, then the result record
static __device__ __align__(256) double g_noalloc_scratch[kMaxPartials + 32];

__device__ __forceinline__ double na_warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ double na_block_sum(double v)
{
    __shared__ double red[kThreads / 32];
    v = na_warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double r = 0;
    if (wid == 0) {
        r = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
        r = na_warp_sum(r);
    }
    __syncthreads();
    return r;
}

// CTA b sums |a_i|^2 over the amplitudes of chunk b (2^16 consecutive
// indices, or the whole state if smaller) whose bit q is 0, in a fixed order.
// When bit q lies above the chunk, the chunk is all in or all out (a chunk
// all out writes 0 at once).  Loads are 16 bytes: two complex64 amplitudes
// (the pair 2k, 2k+1 shares bit q for q >= 1; for q = 0 the first of each
// pair counts) when the buffer is 16-byte aligned (vec), else one amplitude.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_na_chunk_sum(const T *__restrict__ a, uint64_t N, int q, int vec, double *partials)
{
    typedef typename vec2<T>::type V;
    const uint64_t chunk = N < (1ull << kChunkBits) ? N : (1ull << kChunkBits);
    const uint64_t base = (uint64_t)blockIdx.x * chunk;
    double acc = 0;
    const bool whole = (1ull << q) >= chunk;             // bit q is constant on the chunk
    if (!(whole && ((base >> q) & 1ull))) {
        if (sizeof(T) == 4 && vec) {
            const float4 *p4 = reinterpret_cast<const float4 *>(a + 2 * base);
            const uint64_t pairs = chunk >> 1;
            if (whole || q == 0) {
#pragma unroll 4
                for (uint64_t w = threadIdx.x; w < pairs; w += kThreads) {
                    const float4 x = p4[w];
                    acc += fma((double)x.x, (double)x.x, (double)x.y * (double)x.y);
                    if (q) acc += fma((double)x.z, (double)x.z, (double)x.w * (double)x.w);
                }
            } else {
                // pairs with bit q - 1 of the pair index clear
                const uint64_t lo = (1ull << (q - 1)) - 1;
#pragma unroll 4
                for (uint64_t w = threadIdx.x; w < (pairs >> 1); w += kThreads) {
                    const float4 x = p4[((w & ~lo) << 1) | (w & lo)];
                    acc += fma((double)x.x, (double)x.x, (double)x.y * (double)x.y);
                    acc += fma((double)x.z, (double)x.z, (double)x.w * (double)x.w);
                }
            }
        } else {
            const V *pa = reinterpret_cast<const V *>(a) + base;
            const uint64_t lo = (1ull << q) - 1, items = whole ? chunk : chunk >> 1;
#pragma unroll 4
            for (uint64_t w = threadIdx.x; w < items; w += kThreads) {
                const V x = pa[whole ? w : (((w & ~lo) << 1) | (w & lo))];
                acc += fma((double)x.x, (double)x.x, (double)x.y * (double)x.y);
            }
        }
    }
    double s = na_block_sum(acc);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// Fixed-order total, then qubitMeasure's rule: outcome = ((float)u > p0),
// scale = 1/sqrt(p of the outcome) (CPUQuantumGates.cpp:1071-1126).
__global__ void k_na_decide(const double *partials, int count, NaResult *res, double u, int *outcome_out,
                            double *p0_out)
{
    double acc = 0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) acc += partials[i];
    double tot = na_block_sum(acc);
    if (threadIdx.x == 0) {
        const float fi = (float)u;
        const int out = ((double)fi > tot) ? 1 : 0;
        const double psel = out ? 1.0 - tot : tot;
        res->p0 = tot;
        res->outcome = out;
        res->status = psel > 0.0 ? 0 : 1;
        res->scale = psel > 0.0 ? 1.0 / sqrt(psel) : 1.0;
        *outcome_out = res->status ? -1 : out;
        *p0_out = tot;
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
k_na_collapse(T *__restrict__ a, uint64_t pairs, int q, const NaResult *res)
{
    if (res->status) return;
    typedef typename vec2<T>::type V;
    V *pa = reinterpret_cast<V *>(a);
    const int out = res->outcome;
    const T sc = (T)res->scale;
    const uint64_t st = 1ull << q;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < pairs; w += stride) {
        const uint64_t i0 = ((w >> q) << (q + 1)) | (w & (st - 1));
        const uint64_t ik = out ? i0 + st : i0, iz = out ? i0 : i0 + st;
        V x = pa[ik];
        pa[ik] = V{x.x * sc, x.y * sc};
        pa[iz] = V{(T)0, (T)0};
    }
}

// Device address of g_noalloc_scratch, looked up once per device (the first
// call on it) and kept: a cudaDeviceReset between calls would leave it stale,
// and is not supported.
constexpr int kMaxDevices = 64;
std::mutex g_na_mutex;
double *g_na_addr[kMaxDevices] = {nullptr};

int noalloc_scratch(double **out)
{
    int dev = 0;
    QS_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return qs_fail(QS_ERR_UNSUPPORTED, "qs_measure_noalloc: device %d", dev);
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return qs_cuda_fail(e, "qs_measure_noalloc: cudaGetSymbolAddress");
        g_na_addr[dev] = static_cast<double *>(p);
    }
    *out = g_na_addr[dev];
    return QS_OK;
}

template <typename T>
int measure_noalloc_t(void *amp, int n, int q, double u, int *outcome_dev, double *p0_dev, cudaStream_t st)
{
    double *scratch = nullptr;
    int r = noalloc_scratch(&scratch);
    if (r) return r;
    const uint64_t N = 1ull << n;
    const uint64_t chunks = N >> kChunkBits ? N >> kChunkBits : 1;
    double *partials = scratch;
    NaResult *res = reinterpret_cast<NaResult *>(scratch + kMaxPartials);
    const int vec = ((uintptr_t)amp & 15u) == 0;
    k_na_chunk_sum<T><<<(unsigned)chunks, kThreads, 0, st>>>(static_cast<const T *>(amp), N, q, vec, partials);
    QS_LAUNCH_CHECK("k_na_chunk_sum");
    k_na_decide<<<1, kThreads, 0, st>>>(partials, (int)chunks, res, u, outcome_dev, p0_dev);
    QS_LAUNCH_CHECK("k_na_decide");
    const uint64_t pairs = N >> 1;
    k_na_collapse<T><<<grid_for(pairs, kThreads), kThreads, 0, st>>>(static_cast<T *>(amp), pairs, q, res);
    QS_LAUNCH_CHECK("k_na_collapse");
    return QS_OK;
}

}  // namespace

extern "C" int qs_measure_noalloc(void *amp, int n_qubits, int dtype, int q, double u, int *outcome_dev,
                                  double *p0_dev, void *stream)
{
    if (!amp || !outcome_dev || !p0_dev) return qs_fail(QS_ERR_ARG, "qs_measure_noalloc: null pointer");
    if (dtype != QS_C64 && dtype != QS_C128) return qs_fail(QS_ERR_ARG, "qs_measure_noalloc: bad dtype %d", dtype);
    if (n_qubits < 1 || n_qubits > kMaxQubits)
        return qs_fail(QS_ERR_ARG,
                       "qs_measure_noalloc: %d qubits; its fixed scratch holds %d partial sums of 2^%d "
                       "amplitudes, so states of 1..%d qubits only (use qs_measure for larger ones)",
                       n_qubits, kMaxPartials, kChunkBits, kMaxQubits);
    if (q < 0 || q >= n_qubits) return qs_fail(QS_ERR_ARG, "qs_measure_noalloc: qubit %d out of range", q);
    const uintptr_t align = dtype == QS_C64 ? 8 : 16;
    if ((uintptr_t)amp % align)
        return qs_fail(QS_ERR_ARG, "qs_measure_noalloc: amplitudes must be %u-byte aligned", (unsigned)align);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return dtype == QS_C64 ? measure_noalloc_t<float>(amp, n_qubits, q, u, outcome_dev, p0_dev, st)
                           : measure_noalloc_t<double>(amp, n_qubits, q, u, outcome_dev, p0_dev, st);
}
