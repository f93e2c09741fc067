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
// Radices 2, 3, 4, 5, 8 and 16 are compiled; the per-size factorisation is
// a runtime plan (FftPlan1) so one kernel serves every 2/3/5-smooth length.
// Index arithmetic uses precomputed magic-number division (FastDiv) instead
// of hardware-emulated integer division, and a thread recomputes its
// butterfly indices after the barrier instead of keeping them live.
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

// 16 = 4 x 4: DFT4 over the stride-4 sub-sequences, twiddles W16^(j*k),
// DFT4 across them; outputs in natural order.
template <int S, typename V> __device__ __forceinline__ void dft16(V* u)
{
    using R = typename RealOf<V>::type;
    const R c1 = R(0.92387953251128675612818318939678829);   // cos(pi/8)
    const R s1 = R(0.38268343236508977172845998403039887);   // sin(pi/8)
    const R r2 = R(0.70710678118654752440084436210484904);   // 1/sqrt(2)
    V a[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        a[j][0] = u[j];
        a[j][1] = u[j + 4];
        a[j][2] = u[j + 8];
        a[j][3] = u[j + 12];
        dft4<S>(a[j]);
    }
    // a[j][k] *= exp(S*2*pi*i*j*k/16) for j, k in 1..3
    auto rot = [](V z, R c, R sn) { return mkc<V>(z.x * c - S * z.y * sn, z.y * c + S * z.x * sn); };
    a[1][1] = rot(a[1][1], c1, s1);
    a[1][2] = rot(a[1][2], r2, r2);
    a[1][3] = rot(a[1][3], s1, c1);
    a[2][1] = rot(a[2][1], r2, r2);
    a[2][2] = mul_si<S>(a[2][2]);
    a[2][3] = rot(a[2][3], -r2, r2);
    a[3][1] = rot(a[3][1], s1, c1);
    a[3][2] = rot(a[3][2], -r2, r2);
    a[3][3] = rot(a[3][3], -c1, -s1);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        V b[4] = {a[0][k], a[1][k], a[2][k], a[3][k]};
        dft4<S>(b);
        u[k] = b[0];
        u[k + 4] = b[1];
        u[k + 8] = b[2];
        u[k + 12] = b[3];
    }
}

template <int S, int R, typename V> __device__ __forceinline__ void dftR(V* u)
{
    if constexpr (R == 2) dft2<S>(u);
    else if constexpr (R == 3) dft3<S>(u);
    else if constexpr (R == 4) dft4<S>(u);
    else if constexpr (R == 5) dft5<S>(u);
    else if constexpr (R == 8) dft8<S>(u);
    else if constexpr (R == 16) dft16<S>(u);
}

// Magic-number division for 0 <= n < 2^31 (Granlund & Montgomery, PLDI'94):
// q = (umulhi(n, m) + n) >> s with s = ceil(log2 d), m = 2^32 (2^s - d)/d + 1.
struct FastDiv {
    unsigned d, m, s;
};
__device__ __forceinline__ unsigned fdiv(unsigned n, const FastDiv& f) { return (__umulhi(n, f.m) + n) >> f.s; }
inline FastDiv make_fastdiv(unsigned d)
{
    FastDiv f{d, 0u, 0u};
    if (d <= 1) return f;
    unsigned l = 0;
    while ((1u << l) < d) ++l;
    f.m = (unsigned)(((1ull << 32) * ((1ull << l) - d)) / d + 1ull);
    f.s = l;
    return f;
}

// Runtime factorisation of one transform length: radices, the span (product
// of the earlier radices) before each stage with its FastDiv, and the twiddle
// index step n / (R * span).
struct FftPlan1 {
    int n;
    int nst;
    int rad[8];
    int span[8];
    int tstep[8];
    FastDiv fspan[8];
};

template <int S, typename V> __device__ __forceinline__ V twiddle(const V* tw, int idx)
{
    V w = tw[idx];
    if (S > 0) w.y = -w.y;
    return w;
}

// One radix-R stage over a tile.  E bounds the elements any thread touches:
// the caller guarantees B*n <= E*blockDim.x.  Butterfly idx maps to line
// b = idx mod B and butterfly i = idx div B of that line.
template <typename V, int S, int R, int E>
__device__ __noinline__ void fft_stage(V* tile, const V* __restrict__ tw, unsigned n, unsigned B, const FastDiv& fB,
                                          int js, int bs, unsigned span, const FastDiv& fspan, unsigned tstep)
{
    constexpr int NB = (E + R - 1) / R;
    const unsigned m = n / R;
    const unsigned total = B * m;
    V u[NB][R];
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const unsigned idx = threadIdx.x + q * blockDim.x;
        if (idx < total) {
            const unsigned i = fdiv(idx, fB), b = idx - i * B;
            const V* src = tile + (int)i * js + (int)b * bs;
#pragma unroll
            for (int t = 0; t < R; ++t) u[q][t] = src[t * (int)m * js];
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const unsigned idx = threadIdx.x + q * blockDim.x;
        if (idx < total) {
            const unsigned i = fdiv(idx, fB), b = idx - i * B;
            const unsigned kq = fdiv(i, fspan), k = i - kq * span;
            if (k) {
                const unsigned step = k * tstep;
#pragma unroll
                for (int t = 1; t < R; ++t) u[q][t] = cmul(u[q][t], twiddle<S>(tw, t * step));
            }
            dftR<S, R>(u[q]);
            V* dst = tile + (int)(kq * span * R + k) * js + (int)b * bs;
#pragma unroll
            for (int t = 0; t < R; ++t) dst[t * (int)span * js] = u[q][t];
        }
    }
    __syncthreads();
}

// Full transform of a tile (caller has synchronised after filling it).  The
// plan lives in device memory (uniform loads): indexing a plan held in the
// kernel's parameter block by stage would force a local-memory copy of it.
template <typename V, int S, int E>
__device__ __forceinline__ void fft_tile(V* tile, const V* __restrict__ tw, const FftPlan1* __restrict__ p, unsigned B,
                                         const FastDiv& fB, int js, int bs)
{
    const int nst = p->nst;
    const unsigned n = p->n;
    for (int st = 0; st < nst; ++st) {
        const unsigned span = p->span[st], tstep = p->tstep[st];
        const FastDiv fs = p->fspan[st];
        switch (p->rad[st]) {
        case 16: fft_stage<V, S, 16, E>(tile, tw, n, B, fB, js, bs, span, fs, tstep); break;
        case 8: fft_stage<V, S, 8, E>(tile, tw, n, B, fB, js, bs, span, fs, tstep); break;
        case 4: fft_stage<V, S, 4, E>(tile, tw, n, B, fB, js, bs, span, fs, tstep); break;
        case 2: fft_stage<V, S, 2, E>(tile, tw, n, B, fB, js, bs, span, fs, tstep); break;
        case 3: fft_stage<V, S, 3, E>(tile, tw, n, B, fB, js, bs, span, fs, tstep); break;
        case 5: fft_stage<V, S, 5, E>(tile, tw, n, B, fB, js, bs, span, fs, tstep); break;
        default: break;
        }
    }
}

template <typename V>
__device__ __forceinline__ void load_twiddles(V* dst, const V* __restrict__ src, int n)
{
    for (int j = threadIdx.x; j < n; j += blockDim.x) dst[j] = src[j];
}

}  // namespace ftsp

namespace ftsp {

// ---------------------------------------------------------------------------
// Compile-time transforms for the production lengths.  Length, batch,
// strides, thread count and the radix plan are constants, the stages are
// unrolled, and every index is computed with constant divisors.  The plan is
// the runtime planner's: the power-of-two part in the fewest stages of radix
// <= RMAX spread evenly, then 3s and 5s.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int ct_p2(int n)
{
    int p = 0;
    while (n % 2 == 0) {
        n /= 2;
        ++p;
    }
    return p;
}
__host__ __device__ constexpr int ct_lg(int r)
{
    int l = 0;
    while ((1 << l) < r) ++l;
    return l;
}
__host__ __device__ constexpr int ct_nst(int n, int rmax)
{
    const int p2 = ct_p2(n), bits = ct_lg(rmax);
    int r = n >> p2, nst = (p2 + bits - 1) / bits;
    while (r % 3 == 0) { r /= 3; ++nst; }
    while (r % 5 == 0) { r /= 5; ++nst; }
    return nst;
}
__host__ __device__ constexpr int ct_rad(int n, int rmax, int st)
{
    const int p2 = ct_p2(n), bits = ct_lg(rmax);
    const int nst2 = (p2 + bits - 1) / bits;
    int left = p2;
    for (int s = 0; s < nst2; ++s) {
        const int b = (left + (nst2 - s) - 1) / (nst2 - s);
        if (s == st) return 1 << b;
        left -= b;
    }
    int r = n >> p2, s = nst2;
    while (r % 3 == 0) {
        if (s == st) return 3;
        r /= 3;
        ++s;
    }
    while (r % 5 == 0) {
        if (s == st) return 5;
        r /= 5;
        ++s;
    }
    return 1;
}
__host__ __device__ constexpr int ct_span(int n, int rmax, int st)
{
    int s = 1;
    for (int k = 0; k < st; ++k) s *= ct_rad(n, rmax, k);
    return s;
}

// One stage: B lines of length N, element (j, b) at tile[j*JS + b*BS],
// NT threads, E elements per thread at most (B*N <= E*NT).
template <typename V, int S, int N, int RMAX, int B, int JS, int BS, int NT, int E, int ST>
__device__ __forceinline__ void ct_stage(V* tile, const V* __restrict__ tw)
{
    constexpr int R = ct_rad(N, RMAX, ST);
    constexpr int SPAN = ct_span(N, RMAX, ST);
    constexpr int M = N / R;
    constexpr int TOTAL = B * M;
    constexpr int TSTEP = N / (R * SPAN);
    constexpr int NB = (TOTAL + NT - 1) / NT;
    static_assert(NB * R <= E + R, "too many elements per thread");
    V u[NB][R];
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const unsigned idx = threadIdx.x + q * NT;
        if (TOTAL % NT == 0 || idx < (unsigned)TOTAL) {
            const unsigned i = idx / B, b = idx % B;
            const V* src = tile + i * JS + b * BS;
#pragma unroll
            for (int t = 0; t < R; ++t) u[q][t] = src[t * M * JS];
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const unsigned idx = threadIdx.x + q * NT;
        if (TOTAL % NT == 0 || idx < (unsigned)TOTAL) {
            const unsigned i = idx / B, b = idx % B;
            const unsigned k = i % SPAN, kq = i / SPAN;
            if (SPAN > 1 && k) {
                const unsigned step = k * TSTEP;
#pragma unroll
                for (int t = 1; t < R; ++t) u[q][t] = cmul(u[q][t], twiddle<S>(tw, t * step));
            }
            dftR<S, R>(u[q]);
            V* dst = tile + (kq * SPAN * R + k) * JS + b * BS;
#pragma unroll
            for (int t = 0; t < R; ++t) dst[t * SPAN * JS] = u[q][t];
        }
    }
    __syncthreads();
}

template <typename V, int S, int N, int RMAX, int B, int JS, int BS, int NT, int E, int ST = 0>
__device__ __forceinline__ void ct_fft(V* tile, const V* __restrict__ tw)
{
    if constexpr (ST < ct_nst(N, RMAX)) {
        ct_stage<V, S, N, RMAX, B, JS, BS, NT, E, ST>(tile, tw);
        ct_fft<V, S, N, RMAX, B, JS, BS, NT, E, ST + 1>(tile, tw);
    }
}

// ---------------------------------------------------------------------------
// Stages as separate gather / butterfly / scatter steps, for kernels that keep
// a stage's values in registers across a pointwise step.  REV selects the
// reversed radix order: a transform in reversed order starts with the radix
// that the forward order ends with, and the Stockham last stage leaves each
// thread holding positions i + t*SPAN (SPAN = N/R) of its line, which are
// exactly the inputs i + t*M (M = N/R) of the first stage of the reversed
// order.  So "last stage, pointwise, first stage of the next transform" runs
// without a shared-memory round trip.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int ct_rad_o(int n, int rmax, int st, bool rev)
{
    return ct_rad(n, rmax, rev ? ct_nst(n, rmax) - 1 - st : st);
}
__host__ __device__ constexpr int ct_span_o(int n, int rmax, int st, bool rev)
{
    int s = 1;
    for (int k = 0; k < st; ++k) s *= ct_rad_o(n, rmax, k, rev);
    return s;
}

// Stage ST of B lines of length N with NT threads: butterfly idx = tid + q*NT
// (q < NB) works on line b = idx % B, butterfly i = idx / B of the line.
template <int N, int RMAX, int B, int NT, int ST, bool REV>
struct CtSt {
    static constexpr int R = ct_rad_o(N, RMAX, ST, REV);
    static constexpr int SPAN = ct_span_o(N, RMAX, ST, REV);
    static constexpr int M = N / R;
    static constexpr int TOTAL = B * M;
    static constexpr int TSTEP = N / (R * SPAN);
    static constexpr int NB = (TOTAL + NT - 1) / NT;
    __device__ static bool valid(int q) { return TOTAL % NT == 0 || threadIdx.x + q * NT < (unsigned)TOTAL; }
    __device__ static int butterfly(int q) { return (int)((threadIdx.x + q * NT) / B); }
    __device__ static int line(int q) { return (int)((threadIdx.x + q * NT) % B); }
    // position along the line of output t of butterfly q
    __device__ static int out_pos(int q, int t)
    {
        const int i = butterfly(q), k = i % SPAN, kq = i / SPAN;
        return kq * SPAN * R + k + t * SPAN;
    }
};

template <class St, int JS, int BS, typename V>
__device__ __forceinline__ void st_gather(const V* tile, V (&u)[St::NB][St::R])
{
#pragma unroll
    for (int q = 0; q < St::NB; ++q)
        if (St::valid(q)) {
            const V* src = tile + St::butterfly(q) * JS + St::line(q) * BS;
#pragma unroll
            for (int t = 0; t < St::R; ++t) u[q][t] = src[t * St::M * JS];
        }
}

template <int S, class St, typename V>
__device__ __forceinline__ void st_butterfly(V (&u)[St::NB][St::R], const V* __restrict__ tw)
{
#pragma unroll
    for (int q = 0; q < St::NB; ++q)
        if (St::valid(q)) {
            const unsigned k = (unsigned)St::butterfly(q) % St::SPAN;
            if (St::SPAN > 1 && k) {
                const unsigned step = k * St::TSTEP;
#pragma unroll
                for (int t = 1; t < St::R; ++t) u[q][t] = cmul(u[q][t], twiddle<S>(tw, t * step));
            }
            dftR<S, St::R>(u[q]);
        }
}

template <class St, int JS, int BS, typename V>
__device__ __forceinline__ void st_scatter(V* tile, const V (&u)[St::NB][St::R])
{
#pragma unroll
    for (int q = 0; q < St::NB; ++q)
        if (St::valid(q)) {
            V* dst = tile + St::out_pos(q, 0) * JS + St::line(q) * BS;
#pragma unroll
            for (int t = 0; t < St::R; ++t) dst[t * St::SPAN * JS] = u[q][t];
        }
}

// Stages [ST, END) of one transform through shared memory.
template <typename V, int S, int N, int RMAX, int B, int JS, int BS, int NT, bool REV, int ST, int END>
__device__ __forceinline__ void st_range(V* tile, const V* __restrict__ tw)
{
    if constexpr (ST < END) {
        using St = CtSt<N, RMAX, B, NT, ST, REV>;
        V u[St::NB][St::R];
        st_gather<St, JS, BS>(tile, u);
        __syncthreads();
        st_butterfly<S, St>(u, tw);
        st_scatter<St, JS, BS>(tile, u);
        __syncthreads();
        st_range<V, S, N, RMAX, B, JS, BS, NT, REV, ST + 1, END>(tile, tw);
    }
}

}  // namespace ftsp
