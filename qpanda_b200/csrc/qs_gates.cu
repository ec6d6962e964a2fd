// qs_gates.cu - the plain per-gate path: HBM-streaming kernels for every
// gate of QPandaSDK/QuantumInstructionHandle/CPUQuantumGates.cpp.
//
// All gates lower to three kernels:
//   k_pair   - a 2x2 complex matrix on amplitude pairs (base|off0, base|off1)
//              where base has zeros at the "hole" bits and ones at the control
//              bits.  1-qubit gates (off0 = 0, off1 = 2^t), controlled gates,
//              CNOT/Toffoli (X with controls) and the exchange family
//              (iSWAP, sqiSWAP, SWAP, controlSwap: off0 = 2^a, off1 = 2^b).
//   k_quad   - a dense 4x4 on (q0, q1) with controls.
//   k_phase  - multiply the amplitudes that have every bit of a mask set (CR).
//
// Each thread owns whole pairs, found by inserting zero bits at the hole
// positions ("pair-index remapping"): both halves of every pair are read and
// written by the same thread, so no gate needs a second pass or a barrier,
// and for any target the warp's addresses cover whole 32-byte sectors.
// When bit 0 is not a hole, a thread owns two neighbouring pairs and moves
// them as 16-byte vectors (float4 for complex64, 2 x double2 for complex128).
// For complex64 with the target on qubit 0 the pair is the two halves of one
// float4.  Arithmetic: FP32 for complex64 states, FP64 for complex128.
#include "qs_common.cuh"

namespace {

enum { PAIR_SCALAR = 0, PAIR_VEC2 = 1, PAIR_INVEC = 2 };

template <typename T> struct Mat2 { T m[8]; };
template <typename T> struct Mat4 { T m[32]; };

template <typename T>
__device__ __forceinline__ void cmul_add2(T &xr, T &xi, T ar, T ai, T br, T bi,
                                          const T *r0, const T *r1)
{
    // (xr, xi) = r0 * a + r1 * b, r0 = (r0[0], r0[1]), r1 = (r1[0], r1[1])
    T re = r0[0] * ar - r0[1] * ai;
    T im = r0[0] * ai + r0[1] * ar;
    re = fma(r1[0], br, re); re = fma(-r1[1], bi, re);
    im = fma(r1[0], bi, im); im = fma(r1[1], br, im);
    xr = re; xi = im;
}

template <typename T>
__device__ __forceinline__ void apply2(T &ar, T &ai, T &br, T &bi, const Mat2<T> &M)
{
    T xr, xi, yr, yi;
    cmul_add2(xr, xi, ar, ai, br, bi, &M.m[0], &M.m[2]);
    cmul_add2(yr, yi, ar, ai, br, bi, &M.m[4], &M.m[6]);
    ar = xr; ai = xi; br = yr; bi = yi;
}

template <typename T, int MODE>
__global__ void __launch_bounds__(256)
k_pair(T *__restrict__ a, uint64_t items, Holes h, uint64_t cmask, uint64_t off0,
       uint64_t off1, Mat2<T> M)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < items; w += stride) {
        if constexpr (MODE == PAIR_SCALAR) {
            uint64_t base = insert_holes(w, h) | cmask;
            typedef typename vec2<T>::type V;
            V *pa = reinterpret_cast<V *>(a);
            V x = pa[base | off0], y = pa[base | off1];
            apply2(x.x, x.y, y.x, y.y, M);
            pa[base | off0] = x;
            pa[base | off1] = y;
        } else if constexpr (MODE == PAIR_VEC2) {
            uint64_t base = insert_holes(w << 1, h) | cmask;   // bit 0 free and 0
            if constexpr (sizeof(T) == 4) {
                float4 *p0 = reinterpret_cast<float4 *>(a + 2 * (base | off0));
                float4 *p1 = reinterpret_cast<float4 *>(a + 2 * (base | off1));
                float4 x = *p0, y = *p1;
                apply2(x.x, x.y, y.x, y.y, M);
                apply2(x.z, x.w, y.z, y.w, M);
                *p0 = x;
                *p1 = y;
            } else {
                double2 *p0 = reinterpret_cast<double2 *>(a) + (base | off0);
                double2 *p1 = reinterpret_cast<double2 *>(a) + (base | off1);
                double2 x0 = p0[0], x1 = p0[1], y0 = p1[0], y1 = p1[1];
                apply2(x0.x, x0.y, y0.x, y0.y, M);
                apply2(x1.x, x1.y, y1.x, y1.y, M);
                p0[0] = x0; p0[1] = x1;
                p1[0] = y0; p1[1] = y1;
            }
        } else {   // PAIR_INVEC: complex64, target qubit 0, pair inside one float4
            uint64_t base = insert_holes(w, h) | cmask;
            float4 *p = reinterpret_cast<float4 *>(a + 2 * base);
            float4 v = *p;
            apply2(v.x, v.y, v.z, v.w, *reinterpret_cast<const Mat2<float> *>(&M));
            *p = v;
        }
    }
}

template <typename T>
__device__ __forceinline__ void apply4(T (&v)[8], const Mat4<T> &M)
{
    T o[8];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        T re = 0, im = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            T mr = M.m[8 * r + 2 * c], mi = M.m[8 * r + 2 * c + 1];
            re = fma(mr, v[2 * c], re); re = fma(-mi, v[2 * c + 1], re);
            im = fma(mr, v[2 * c + 1], im); im = fma(mi, v[2 * c], im);
        }
        o[2 * r] = re; o[2 * r + 1] = im;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = o[j];
}

template <typename T, bool VEC>
__global__ void __launch_bounds__(256)
k_quad(T *__restrict__ a, uint64_t items, Holes h, uint64_t cmask, uint64_t o0, uint64_t o1,
       Mat4<T> M)
{
    typedef typename vec2<T>::type V;
    V *pa = reinterpret_cast<V *>(a);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < items; w += stride) {
        uint64_t base = insert_holes(VEC ? (w << 1) : w, h) | cmask;
        uint64_t idx[4] = {base, base | o0, base | o1, base | o0 | o1};
        if constexpr (!VEC) {
            T v[8];
#pragma unroll
            for (int j = 0; j < 4; ++j) { V t = pa[idx[j]]; v[2 * j] = t.x; v[2 * j + 1] = t.y; }
            apply4(v, M);
#pragma unroll
            for (int j = 0; j < 4; ++j) pa[idx[j]] = V{v[2 * j], v[2 * j + 1]};
        } else if constexpr (sizeof(T) == 4) {
            // base has bit 0 clear: each member pair (idx, idx + 1) is one float4
            float4 *p4 = reinterpret_cast<float4 *>(a);
            float4 t[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) t[j] = p4[idx[j] >> 1];
            T v0[8], v1[8];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                v0[2 * j] = t[j].x; v0[2 * j + 1] = t[j].y;
                v1[2 * j] = t[j].z; v1[2 * j + 1] = t[j].w;
            }
            apply4(v0, M);
            apply4(v1, M);
#pragma unroll
            for (int j = 0; j < 4; ++j) p4[idx[j] >> 1] = make_float4(v0[2 * j], v0[2 * j + 1], v1[2 * j], v1[2 * j + 1]);
        } else {
            T v0[8], v1[8];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                V t0 = pa[idx[j]], t1 = pa[idx[j] + 1];
                v0[2 * j] = t0.x; v0[2 * j + 1] = t0.y;
                v1[2 * j] = t1.x; v1[2 * j + 1] = t1.y;
            }
            apply4(v0, M);
            apply4(v1, M);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                pa[idx[j]] = V{v0[2 * j], v0[2 * j + 1]};
                pa[idx[j] + 1] = V{v1[2 * j], v1[2 * j + 1]};
            }
        }
    }
}

template <typename T, bool VEC>
__global__ void __launch_bounds__(256)
k_phase(T *__restrict__ a, uint64_t items, Holes h, uint64_t mask, T pr, T pi)
{
    typedef typename vec2<T>::type V;
    V *pa = reinterpret_cast<V *>(a);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < items; w += stride) {
        uint64_t i = insert_holes(VEC ? (w << 1) : w, h) | mask;
        if constexpr (VEC && sizeof(T) == 4) {
            // i has bit 0 clear: amplitudes i, i + 1 are one float4
            float4 *p4 = reinterpret_cast<float4 *>(a) + (i >> 1);
            const float4 t = *p4;
            *p4 = make_float4(t.x * pr - t.y * pi, t.x * pi + t.y * pr, t.z * pr - t.w * pi, t.z * pi + t.w * pr);
        } else {
#pragma unroll
            for (int j = 0; j < (VEC ? 2 : 1); ++j) {
                V t = pa[i + j];
                pa[i + j] = V{t.x * pr - t.y * pi, t.x * pi + t.y * pr};
            }
        }
    }
}

template <typename T>
__global__ void k_zero_state(T *__restrict__ a, uint64_t n_vec4)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    float4 *p = reinterpret_cast<float4 *>(a);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_vec4; i += stride) {
        float4 v = z;
        if (i == 0) {   // amplitude 0 = 1 + 0i
            if (sizeof(T) == 4) v.x = 1.f;
            else reinterpret_cast<double *>(&v)[0] = 1.0;
        }
        p[i] = v;
    }
}

template <typename T>
int do_pair(qs_state *s, uint64_t holes_mask, uint64_t cmask, uint64_t off0, uint64_t off1,
            const double m[8])
{
    Mat2<T> M;
    for (int j = 0; j < 8; ++j) M.m[j] = (T)m[j];
    Holes h = holes_from_mask(holes_mask);
    uint64_t pairs = s->N >> h.k;
    T *a = static_cast<T *>(s->amp);
    const int thr = 256;
    if (!(holes_mask & 1ull)) {
        uint64_t items = pairs >> 1;
        k_pair<T, PAIR_VEC2><<<grid_for(items, thr), thr, 0, s->stream>>>(a, items, h, cmask, off0, off1, M);
    } else if (sizeof(T) == 4 && off0 == 0 && off1 == 1) {
        k_pair<T, PAIR_INVEC><<<grid_for(pairs, thr), thr, 0, s->stream>>>(a, pairs, h, cmask, off0, off1, M);
    } else {
        k_pair<T, PAIR_SCALAR><<<grid_for(pairs, thr), thr, 0, s->stream>>>(a, pairs, h, cmask, off0, off1, M);
    }
    QS_LAUNCH_CHECK("k_pair");
    return QS_OK;
}

template <typename T>
int do_quad(qs_state *s, int q0, int q1, uint64_t cmask, const double m[32])
{
    Mat4<T> M;
    for (int j = 0; j < 32; ++j) M.m[j] = (T)m[j];
    uint64_t hm = cmask | (1ull << q0) | (1ull << q1);
    Holes h = holes_from_mask(hm);
    uint64_t quads = s->N >> h.k;
    T *a = static_cast<T *>(s->amp);
    const int thr = 256;
    if (!(hm & 1ull) && quads >= 2) {
        uint64_t items = quads >> 1;
        k_quad<T, true><<<grid_for(items, thr), thr, 0, s->stream>>>(a, items, h, cmask, 1ull << q0, 1ull << q1, M);
    } else {
        k_quad<T, false><<<grid_for(quads, thr), thr, 0, s->stream>>>(a, quads, h, cmask, 1ull << q0, 1ull << q1, M);
    }
    QS_LAUNCH_CHECK("k_quad");
    return QS_OK;
}

template <typename T>
int do_phase(qs_state *s, uint64_t mask, double re, double im)
{
    Holes h = holes_from_mask(mask);
    uint64_t items = s->N >> h.k;
    T *a = static_cast<T *>(s->amp);
    const int thr = 256;
    if (!(mask & 1ull) && items >= 2) {
        k_phase<T, true><<<grid_for(items >> 1, thr), thr, 0, s->stream>>>(a, items >> 1, h, mask, (T)re, (T)im);
    } else {
        k_phase<T, false><<<grid_for(items, thr), thr, 0, s->stream>>>(a, items, h, mask, (T)re, (T)im);
    }
    QS_LAUNCH_CHECK("k_phase");
    return QS_OK;
}

}  // namespace

int launch_pair(qs_state *s, uint64_t holes_mask, uint64_t cmask, uint64_t off0, uint64_t off1,
                const double m[8])
{
    return s->dtype == QS_C64 ? do_pair<float>(s, holes_mask, cmask, off0, off1, m)
                              : do_pair<double>(s, holes_mask, cmask, off0, off1, m);
}

int launch_quad(qs_state *s, int q0, int q1, uint64_t cmask, const double m[32])
{
    return s->dtype == QS_C64 ? do_quad<float>(s, q0, q1, cmask, m)
                              : do_quad<double>(s, q0, q1, cmask, m);
}

int launch_phase(qs_state *s, uint64_t mask, double re, double im)
{
    return s->dtype == QS_C64 ? do_phase<float>(s, mask, re, im)
                              : do_phase<double>(s, mask, re, im);
}

int launch_fill_zero_state(qs_state *s)
{
    uint64_t nvec = s->amp_bytes() / 16;
    if (s->dtype == QS_C64)
        k_zero_state<float><<<grid_for(nvec, 256), 256, 0, s->stream>>>(static_cast<float *>(s->amp), nvec);
    else
        k_zero_state<double><<<grid_for(nvec, 256), 256, 0, s->stream>>>(static_cast<double *>(s->amp), nvec);
    QS_LAUNCH_CHECK("k_zero_state");
    return QS_OK;
}
