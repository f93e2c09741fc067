// Shared-memory Stockham FFT building blocks for sm_100a.
//
// A "tile" is a batch of B independent 1-D transforms of length n held in
// shared memory; element j of transform b lives at tile[j*js + b*bs].  Each
// stage is a radix-R Stockham step (autosorting, no bit reversal):
//
//   for butterfly (i, b), i < n/R, k = i mod span:
//     u_t = x[i + t*n/R] * w^(t*k*n/(R*span)),   w = exp(S*2*pi*i/n)
//     y[(i-k)*R + k + t*span] = DFT_R(u)_t,       span *= R after the stage
//
// Stages run in place: every thread first stages the R inputs of each of its
// butterflies in registers, the block synchronises, then the outputs are
// written.  Twiddles come from a table w_n^j = exp(-2*pi*i*j/n) held in
// shared memory (computed on the host in long double), conjugated for S = +1.
// Radices 2, 3, 4, 5 and 8 are compiled; the per-size factorisation is a
// runtime plan (FftPlan1) so one kernel serves every 2/3/5-smooth length.
//
// Conventions follow cuFFT's: S = -1 forward, S = +1 inverse, unnormalised.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ftsp {

template <typename T> struct CplxOf;
template <> struct CplxOf<float> { using type = float2; };
template <> struct CplxOf<double> { using type = double2; };
template <typename T> using cplx = typename CplxOf<T>::type;

template <typename V> struct RealOf;
template <> struct RealOf<float2> { using type = float; };
template <> struct RealOf<double2> { using type = double; };

template <typename V>
__device__ __forceinline__ V mkc(typename RealOf<V>::type x, typename RealOf<V>::type y)
{
    V z;
    z.x = x;
    z.y = y;
    return z;
}
template <typename V> __device__ __forceinline__ V cadd(V a, V b) { return mkc<V>(a.x + b.x, a.y + b.y); }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { return mkc<V>(a.x - b.x, a.y - b.y); }
template <typename V> __device__ __forceinline__ V cmul(V a, V b)
{
    return mkc<V>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename V> __device__ __forceinline__ V cscale(V a, typename RealOf<V>::type s) { return mkc<V>(s * a.x, s * a.y); }
// multiply by S*i
template <int S, typename V> __device__ __forceinline__ V mul_si(V z)
{
    return S < 0 ? mkc<V>(z.y, -z.x) : mkc<V>(-z.y, z.x);
}

// ---- radix butterflies (in place on u[0..R-1]) ----
template <int S, typename V> __device__ __forceinline__ void dft2(V* u)
{
    const V a = u[0], b = u[1];
    u[0] = cadd(a, b);
    u[1] = csub(a, b);
}

template <int S, typename V> __device__ __forceinline__ void dft3(V* u)
{
    using R = typename RealOf<V>::type;
    const R h = R(0.86602540378443864676372317075293618);   // sin(2 pi / 3)
    const V a = cadd(u[1], u[2]);
    const V b = csub(u[1], u[2]);
    const V c = mkc<V>(u[0].x - R(0.5) * a.x, u[0].y - R(0.5) * a.y);
    const V sb = mul_si<S>(cscale(b, h));
    u[0] = cadd(u[0], a);
    u[1] = cadd(c, sb);
    u[2] = csub(c, sb);
}

template <int S, typename V> __device__ __forceinline__ void dft4(V* u)
{
    const V a0 = cadd(u[0], u[2]), a1 = csub(u[0], u[2]);
    const V b0 = cadd(u[1], u[3]), b1 = mul_si<S>(csub(u[1], u[3]));
    u[0] = cadd(a0, b0);
    u[2] = csub(a0, b0);
    u[1] = cadd(a1, b1);
    u[3] = csub(a1, b1);
}

template <int S, typename V> __device__ __forceinline__ void dft5(V* u)
{
    using R = typename RealOf<V>::type;
    const R c1 = R(0.30901699437494742410229341718281906);  // cos(2 pi/5)
    const R c2 = R(-0.80901699437494742410229341718281906); // cos(4 pi/5)
    const R s1 = R(0.95105651629515357211643933337938214);  // sin(2 pi/5)
    const R s2 = R(0.58778525229247312916870595463907277);  // sin(4 pi/5)
    const V a1 = cadd(u[1], u[4]), b1 = csub(u[1], u[4]);
    const V a2 = cadd(u[2], u[3]), b2 = csub(u[2], u[3]);
    const V r1 = mkc<V>(u[0].x + c1 * a1.x + c2 * a2.x, u[0].y + c1 * a1.y + c2 * a2.y);
    const V r2 = mkc<V>(u[0].x + c2 * a1.x + c1 * a2.x, u[0].y + c2 * a1.y + c1 * a2.y);
    const V i1 = mul_si<S>(mkc<V>(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y));
    const V i2 = mul_si<S>(mkc<V>(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y));
    u[0] = cadd(u[0], cadd(a1, a2));
    u[1] = cadd(r1, i1);
    u[4] = csub(r1, i1);
    u[2] = cadd(r2, i2);
    u[3] = csub(r2, i2);
}

template <int S, typename V> __device__ __forceinline__ void dft8(V* u)
{
    using R = typename RealOf<V>::type;
    const R r = R(0.70710678118654752440084436210484904);   // 1/sqrt(2)
    V e[4] = {u[0], u[2], u[4], u[6]};
    V o[4] = {u[1], u[3], u[5], u[7]};
    dft4<S>(e);
    dft4<S>(o);
    // o[t] *= exp(S*2*pi*i*t/8)
    const V o1 = o[1], o3 = o[3];
    o[1] = mkc<V>(r * (o1.x - S * o1.y), r * (o1.y + S * o1.x));   // (1 + S i)/sqrt2
    o[2] = mul_si<S>(o[2]);
    o[3] = mkc<V>(r * (-o3.x - S * o3.y), r * (-o3.y + S * o3.x)); // (-1 + S i)/sqrt2
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        u[t] = cadd(e[t], o[t]);
        u[t + 4] = csub(e[t], o[t]);
    }
}

template <int S, int R, typename V> __device__ __forceinline__ void dftR(V* u)
{
    if constexpr (R == 2) dft2<S>(u);
    else if constexpr (R == 3) dft3<S>(u);
    else if constexpr (R == 4) dft4<S>(u);
    else if constexpr (R == 5) dft5<S>(u);
    else if constexpr (R == 8) dft8<S>(u);
}

// Runtime factorisation of one transform length.
struct FftPlan1 {
    int n;
    int nst;
    int rad[12];
};

template <int S, typename V> __device__ __forceinline__ V twiddle(const V* tw, int idx)
{
    V w = tw[idx];
    if (S > 0) w.y = -w.y;
    return w;
}

// One radix-R stage over a tile.  E bounds the elements any thread touches:
// the caller guarantees B*n <= E*blockDim.x.
template <typename V, int S, int R, int E>
__device__ __forceinline__ void fft_stage(V* tile, const V* __restrict__ tw, int n, int B, int js, int bs, int span)
{
    constexpr int NB = (E + R - 1) / R;
    const int m = n / R;
    const int total = B * m;
    const int tstep = n / (R * span);
    V u[NB][R];
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int idx = threadIdx.x + q * blockDim.x;
        if (idx < total) {
            const int b = idx % B, i = idx / B;
            const V* src = tile + i * js + b * bs;
#pragma unroll
            for (int t = 0; t < R; ++t) u[q][t] = src[t * m * js];
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int idx = threadIdx.x + q * blockDim.x;
        if (idx < total) {
            const int b = idx % B, i = idx / B;
            const int k = i % span;
            if (k) {
                const int step = k * tstep;
#pragma unroll
                for (int t = 1; t < R; ++t) u[q][t] = cmul(u[q][t], twiddle<S>(tw, t * step));
            }
            dftR<S, R>(u[q]);
            V* dst = tile + ((i - k) * R + k) * js + b * bs;
#pragma unroll
            for (int t = 0; t < R; ++t) dst[t * span * js] = u[q][t];
        }
    }
    __syncthreads();
}

// Full transform of a tile (caller has synchronised after filling it).
template <typename V, int S, int E>
__device__ __forceinline__ void fft_tile(V* tile, const V* __restrict__ tw, const FftPlan1& p, int B, int js, int bs)
{
    int span = 1;
    for (int st = 0; st < p.nst; ++st) {
        const int R = p.rad[st];
        switch (R) {
        case 8: fft_stage<V, S, 8, E>(tile, tw, p.n, B, js, bs, span); break;
        case 4: fft_stage<V, S, 4, E>(tile, tw, p.n, B, js, bs, span); break;
        case 2: fft_stage<V, S, 2, E>(tile, tw, p.n, B, js, bs, span); break;
        case 3: fft_stage<V, S, 3, E>(tile, tw, p.n, B, js, bs, span); break;
        case 5: fft_stage<V, S, 5, E>(tile, tw, p.n, B, js, bs, span); break;
        default: break;
        }
        span *= R;
    }
}

template <typename V>
__device__ __forceinline__ void load_twiddles(V* dst, const V* __restrict__ src, int n)
{
    for (int j = threadIdx.x; j < n; j += blockDim.x) dst[j] = src[j];
}

}  // namespace ftsp
