// ek_fft32.cuh -- FP32 complex transforms of 2^K points held by 2^(K-4)
// threads (16 points a thread), for the row passes of the FP32 Poisson form.
//
// Forward: decimation in frequency, radix-16 passes from the top index bit
// down (bits [b, b+4), b = K-4, K-8, ...), then one radix-2^(K mod 4) pass on
// the lowest bits when K is not a multiple of 4.  A radix-16 pass is a
// 16-point DFT in registers (4 x 4 split, constant internal twiddles)
// followed by the 15 twiddles exp(-2 pi i kb f / 2^(b+4)); output digit f is
// stored at digit brev4(f), so the transform ends in bit-reversed order.
// Inverse: the adjoint passes in reverse order (conjugate twiddles before the
// inverse DFT), bit-reversed input to natural order.
//
// Shared memory holds transform p of a block at index
// i ^ (((i >> 4) ^ (i >> 8) ^ p) & 15), free of bank conflicts for the
// passes, natural-order and bit-reversed accesses.  The map is linear over
// XOR, so an element's address is its group base's address XOR a
// compile-time constant.  Every pass writes back onto the slots its group
// read, so one barrier per pass suffices.
// The pass twiddles come from per-pass tables laid out f-major, kb-minor:
// the 32 lanes of a warp read consecutive entries.
#pragma once
#include <cuda_runtime.h>

namespace ek {
namespace fft32 {

__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

constexpr float C1 = 0.92387953251128674f;  // cos(pi/8)
constexpr float S1 = 0.38268343236508977f;  // sin(pi/8)
constexpr float R2 = 0.70710678118654752f;  // cos(pi/4)

__host__ __device__ constexpr int brev4(int f) { return ((f & 1) << 3) | ((f & 2) << 1) | ((f & 4) >> 1) | ((f & 8) >> 3); }
__host__ __device__ constexpr int brevq(int f, int q) { return brev4(f) >> (4 - q); }
// XOR-linear part of the shared-memory swizzle (without the transform term)
__host__ __device__ constexpr int lin(int v) { return v ^ (((v >> 4) ^ (v >> 8)) & 15); }

__device__ __forceinline__ int swz_base(int i, int p) { return i ^ (((i >> 4) ^ (i >> 8) ^ p) & 15); }

// z * exp(-/+ 2 pi i m/16) (forward: minus), m a compile-time constant
template <bool INV, int M>
__device__ __forceinline__ float2 w16(float2 z) {
    constexpr int m = M & 15;
    if constexpr (m == 0) {
        return z;
    } else if constexpr (m == 8) {
        return make_float2(-z.x, -z.y);
    } else if constexpr (m == 4 || m == 12) {
        // forward m = 4: -i z; m = 12: +i z; inverse the other way round
        constexpr bool minus_i = (m == 4) != INV;
        return minus_i ? make_float2(z.y, -z.x) : make_float2(-z.y, z.x);
    } else if constexpr ((m & 1) == 0) {
        // (c + i s) with |c| = |s| = cos(pi/4)
        constexpr float c = (m == 2 || m == 14) ? R2 : -R2;
        constexpr float s0 = (m == 2 || m == 6) ? -R2 : R2;  // forward imaginary part
        constexpr float s = INV ? -s0 : s0;
        constexpr bool same = (c > 0) == (s > 0);
        // z (c + i s) = (c z.x - s z.y, s z.x + c z.y)
        if constexpr (same) return make_float2(c * (z.x - z.y), c * (z.x + z.y));
        else return make_float2(c * (z.x + z.y), c * (z.y - z.x));
    } else {
        constexpr float cs[8] = {1.0f, C1, R2, S1, 0.0f, -S1, -R2, -C1};   // cos(pi j/8), j < 8
        constexpr float sn[8] = {0.0f, S1, R2, C1, 1.0f, C1, R2, S1};      // sin(pi j/8), j < 8
        constexpr float c = m < 8 ? cs[m] : -cs[m - 8];
        constexpr float s0 = m < 8 ? -sn[m] : sn[m - 8];  // forward: -sin(pi m/8)
        constexpr float s = INV ? -s0 : s0;
        return make_float2(z.x * c - z.y * s, z.x * s + z.y * c);
    }
}

// 4-point DFT in place: (a, b, c, d) -> (X0, X1, X2, X3)
template <bool INV>
__device__ __forceinline__ void dft4(float2 &a, float2 &b, float2 &c, float2 &d) {
    const float2 s0 = a + c, d0 = a - c, s1 = b + d, d1 = b - d;
    const float2 id1 = make_float2(-d1.y, d1.x);  // i d1
    a = s0 + s1;
    c = s0 - s1;
    if (INV) {
        b = d0 + id1;
        d = d0 - id1;
    } else {
        b = d0 - id1;
        d = d0 + id1;
    }
}

// 16-point DFT in place; output f sits at x[out16(f)]
__host__ __device__ constexpr int out16(int f) { return 4 * (f & 3) + (f >> 2); }
template <bool INV>
__device__ __forceinline__ void dft16(float2 (&x)[16]) {
    // n = n1 + 4 n2, f = 4 f1 + f2: 4-point DFTs over n2, twiddles W16^(n1 f2),
    // 4-point DFTs over n1
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) dft4<INV>(x[n1], x[n1 + 4], x[n1 + 8], x[n1 + 12]);
    x[5] = w16<INV, 1>(x[5]);
    x[6] = w16<INV, 2>(x[6]);
    x[7] = w16<INV, 3>(x[7]);
    x[9] = w16<INV, 2>(x[9]);
    x[10] = w16<INV, 4>(x[10]);
    x[11] = w16<INV, 6>(x[11]);
    x[13] = w16<INV, 3>(x[13]);
    x[14] = w16<INV, 6>(x[14]);
    x[15] = w16<INV, 9>(x[15]);
#pragma unroll
    for (int f2 = 0; f2 < 4; ++f2) dft4<INV>(x[4 * f2], x[4 * f2 + 1], x[4 * f2 + 2], x[4 * f2 + 3]);
}

// 2^Q-point DFT (Q = 1..3) in place on x[o .. o + 2^Q); output f at x[o + outq<Q>(f)]
template <int Q> __host__ __device__ constexpr int outq(int f) { return Q == 3 ? 2 * (f & 3) + (f >> 2) : f; }
template <bool INV, int Q>
__device__ __forceinline__ void dftq(float2 *x) {
    if constexpr (Q == 1) {
        const float2 a = x[0], b = x[1];
        x[0] = a + b;
        x[1] = a - b;
    } else if constexpr (Q == 2) {
        dft4<INV>(x[0], x[1], x[2], x[3]);
    } else {
        // n = n1 + 2 n2, f = 4 f1 + f2: 4-point DFTs over n2, twiddles W8^(n1 f2),
        // 2-point DFTs over n1
        dft4<INV>(x[0], x[2], x[4], x[6]);
        dft4<INV>(x[1], x[3], x[5], x[7]);
        x[3] = w16<INV, 2>(x[3]);
        x[5] = w16<INV, 4>(x[5]);
        x[7] = w16<INV, 6>(x[7]);
#pragma unroll
        for (int f2 = 0; f2 < 4; ++f2) {
            const float2 a = x[2 * f2], b = x[2 * f2 + 1];
            x[2 * f2] = a + b;
            x[2 * f2 + 1] = a - b;
        }
    }
}

template <int K>
struct Shape {
    static constexpr int N = 1 << K, T = N >> 4, NF = K >> 2, Q = K & 3;
    // full pass i = 1..NF works on bits [K - 4i, K - 4i + 4)
    __host__ __device__ static constexpr int bit(int i) { return K - 4 * i; }
    // offset of pass i's twiddle table (passes with bit >= 1 have one)
    __host__ __device__ static constexpr int off(int i) {
        int o = 0;
        for (int j = 1; j < i; ++j) o += 15 << (K - 4 * j);
        return o;
    }
};

// Entries of the twiddle tables of a 2^K-point transform (< 2^K).
__host__ __device__ constexpr int table_size(int K) {
    int o = 0;
    for (int b = K - 4; b >= 1; b -= 4) o += 15 << b;
    return o;
}

// Pass twiddle of the table, loaded with an L2 evict_last policy: the tables
// (32 KB at nx = 4096) are read by every block of every solve, and between
// two solves the LBM step streams ~0.9 GB through L2; kept there, the
// inverse pass ran 19.8 us against 20.9 us at 4096 x 1024 (B200).
__device__ __forceinline__ float2 ldtw(const float2 *p) {
    float2 v;
    unsigned long long pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    asm volatile("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ float2 mulw(float2 a, float2 w) {
    return make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}
__device__ __forceinline__ float2 mulw_conj(float2 a, float2 w) {
    return make_float2(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y);
}

// Thread t's group of full pass I: first element and in-group offset kb.
template <int K, int I>
__device__ __forceinline__ void group(int t, int &base, int &kb) {
    constexpr int b = Shape<K>::bit(I);
    kb = t & ((1 << b) - 1);
    base = kb | ((t >> b) << (b + 4));
}

// Forward full pass I on x (its group's elements, v = 0..15), result into s.
template <int K, int I>
__device__ __forceinline__ void fwd_pass_store(float2 (&x)[16], float2 *s, int t, int p,
                                               const float2 *__restrict__ twp) {
    constexpr int b = Shape<K>::bit(I);
    int base, kb;
    group<K, I>(t, base, kb);
    dft16<false>(x);
    const int sb = swz_base(base, p);
    if constexpr (b > 0) {
        const float2 *tp = twp + Shape<K>::off(I) + kb;
#pragma unroll
        for (int f = 1; f < 16; ++f) x[out16(f)] = mulw(x[out16(f)], ldtw(tp + ((f - 1) << b)));
    }
#pragma unroll
    for (int f = 0; f < 16; ++f) s[sb ^ lin(brev4(f) << b)] = x[out16(f)];
}

template <int K, int I>
__device__ __forceinline__ void fwd_pass_load(float2 (&x)[16], const float2 *s, int t, int p) {
    constexpr int b = Shape<K>::bit(I);
    int base, kb;
    group<K, I>(t, base, kb);
    const int sb = swz_base(base, p);
#pragma unroll
    for (int v = 0; v < 16; ++v) x[v] = s[sb ^ lin(v << b)];
}

// Forward passes 2..NF and the partial pass, after pass 1 stored into s.
template <int K, int I>
__device__ __forceinline__ void fwd_rest(float2 *s, int t, int p, const float2 *__restrict__ twp) {
    if constexpr (I <= Shape<K>::NF) {
        float2 x[16];
        fwd_pass_load<K, I>(x, s, t, p);  // a pass writes back onto its group's own slots
        fwd_pass_store<K, I>(x, s, t, p, twp);
        __syncthreads();
        fwd_rest<K, I + 1>(s, t, p, twp);
    } else if constexpr (Shape<K>::Q > 0) {
        constexpr int Q = Shape<K>::Q, R = 1 << Q;
        const int sb = swz_base(t << 4, p);
        float2 x[16];
#pragma unroll
        for (int v = 0; v < 16; ++v) x[v] = s[sb ^ v];
#pragma unroll
        for (int j = 0; j < 16; j += R) dftq<false, Q>(x + j);
#pragma unroll
        for (int j = 0; j < 16; j += R)
#pragma unroll
            for (int f = 0; f < R; ++f) s[sb ^ (j + brevq(f, Q))] = x[j + outq<Q>(f)];
        __syncthreads();
    }
}

// Inverse full pass I: conjugate twiddles, inverse DFT; x ends in natural
// order of v (element base | v << b).
template <int K, int I>
__device__ __forceinline__ void inv_pass_load(float2 (&x)[16], const float2 *s, int t, int p,
                                              const float2 *__restrict__ twp) {
    constexpr int b = Shape<K>::bit(I);
    int base, kb;
    group<K, I>(t, base, kb);
    const int sb = swz_base(base, p);
    float2 z[16];
#pragma unroll
    for (int f = 0; f < 16; ++f) z[f] = s[sb ^ lin(brev4(f) << b)];
    if constexpr (b > 0) {
        const float2 *tp = twp + Shape<K>::off(I) + kb;
#pragma unroll
        for (int f = 1; f < 16; ++f) z[f] = mulw_conj(z[f], ldtw(tp + ((f - 1) << b)));
    }
    dft16<true>(z);
#pragma unroll
    for (int v = 0; v < 16; ++v) x[v] = z[out16(v)];
}

template <int K, int I>
__device__ __forceinline__ void inv_pass_store(const float2 (&x)[16], float2 *s, int t, int p) {
    constexpr int b = Shape<K>::bit(I);
    int base, kb;
    group<K, I>(t, base, kb);
    const int sb = swz_base(base, p);
#pragma unroll
    for (int v = 0; v < 16; ++v) s[sb ^ lin(v << b)] = x[v];
}

// Inverse passes NF..2 (after the partial pass); pass 1 is left to the caller,
// which takes its output from registers.
template <int K, int I>
__device__ __forceinline__ void inv_full(float2 *s, int t, int p, const float2 *__restrict__ twp) {
    if constexpr (I >= 2) {
        float2 x[16];
        inv_pass_load<K, I>(x, s, t, p, twp);
        inv_pass_store<K, I>(x, s, t, p);
        __syncthreads();
        inv_full<K, I - 1>(s, t, p, twp);
    }
}

template <int K>
__device__ __forceinline__ void inv_partial(float2 *s, int t, int p) {
    if constexpr (Shape<K>::Q > 0) {
        constexpr int Q = Shape<K>::Q, R = 1 << Q;
        const int sb = swz_base(t << 4, p);
        float2 x[16];
#pragma unroll
        for (int j = 0; j < 16; j += R)
#pragma unroll
            for (int f = 0; f < R; ++f) x[j + f] = s[sb ^ (j + brevq(f, Q))];
#pragma unroll
        for (int j = 0; j < 16; j += R) {
            dftq<true, Q>(x + j);
            float2 y[R];
#pragma unroll
            for (int v = 0; v < R; ++v) y[v] = x[j + outq<Q>(v)];
#pragma unroll
            for (int v = 0; v < R; ++v) s[sb ^ (j + v)] = y[v];
        }
        __syncthreads();
    }
}

}  // namespace fft32
}  // namespace ek
