// FFT pass kernels with fused pointwise work.
//
// A 3-D transform of an m1 x m2 x m3 row-major grid (z fastest) is split
// into passes that each read and write HBM once:
//   * plane pass   : one x-plane (m2 x m3) per CTA, z- and y-transforms in
//                    shared memory (used when the plane fits: complex64 up
//                    to 128^2, complex128 up to 96^2);
//   * z-line pass  : B contiguous z-rows per CTA;
//   * strided pass : an n x W tile of lines along y or x, W contiguous
//                    z-columns wide, so every load and store is a W-element
//                    contiguous run.
// Each kernel is  [load -> transform(S1)] -> pointwise Op -> [transform(S2)
// -> store] -> Op::end (block reductions, reusing the tile as scratch);
// S = 0 skips that transform, -1/+1 select its sign.  The Op sees
// the element's coordinates (in k-space after a transform) and its global
// offset, so propagator, density, stress and smoothing work rides in the same
// pass as the FFT instead of costing extra HBM round trips.
#pragma once

#include "fft_core.cuh"

#include <type_traits>

namespace ftsp {

// Programmatic dependent launch: a pass launched with the programmatic
// stream-serialisation attribute starts while the previous kernel drains;
// griddepcontrol.wait holds it until that kernel has completed and its
// writes are visible, so only the prologue (constant twiddles into shared
// memory, index set-up) overlaps.  launch_dependents lets the next pass be
// scheduled once this CTA has issued its last global reads.  Both are no-ops
// for launches without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }


struct PlaneGeom {
    int m1, m2, m3;
    int P;                 // shared-memory pitch of a plane row (m3 + 1)
    const FftPlan1* py;    // device-memory plans of the y and z transforms
    const FftPlan1* pz;
    FastDiv fm2, fm3;
};

struct LineGeom {
    int m1, m2, m3;
    int n;                 // transform length (m1 for x, m2 for y, m3 for z)
    int W;                 // z-columns per tile (strided passes)
    int B;                 // rows per tile (z-line pass)
    int P;                 // shared-memory pitch
    const FftPlan1* p;     // device-memory plan of the transform
    FastDiv fW, fB, fm2, fm3;
};

// ---- block reductions (deterministic: fixed shuffle/smem order) ----
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* scratch)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int c = 0; c < K; ++c) {
        double x = v[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        v[c] = x;
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int c = 0; c < K; ++c) scratch[warp * K + c] = v[c];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int c = 0; c < K; ++c) {
            double s = 0.0;
            for (int w = 0; w < nw; ++w) s += scratch[w * K + c];
            v[c] = s;
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Plane pass: grid (m1, nfields), one x-plane per CTA.
// Shared memory: tile[m2][P] + twiddles(m2) + twiddles(m3).
// ---------------------------------------------------------------------------
template <typename T, int E, int S1, int S2, class Op>
__global__ void __launch_bounds__(1024, 1) k_plane(PlaneGeom g, const cplx<T>* src, cplx<T>* dst,
                                                size_t fstride, const cplx<T>* __restrict__ twy,
                                                const cplx<T>* __restrict__ twz, Op op)
{
    using V = cplx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    V* sty = tile + (size_t)g.m2 * g.P;
    V* stz = sty + g.m2;
    const int x = blockIdx.x;
    const int f = blockIdx.y;
    const int ne = g.m2 * g.m3;
    const size_t base = (size_t)f * fstride + (size_t)x * ne;
    if (S1 != 0 || S2 != 0) {
        load_twiddles(sty, twy, g.m2);
        load_twiddles(stz, twz, g.m3);
    }
    if (S1 != 0) {
        for (int e0 = threadIdx.x; e0 < ne; e0 += 4 * blockDim.x) {
            V v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = e0 + u * blockDim.x;
                if (e < ne) v[u] = src[base + e];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = e0 + u * blockDim.x;
                if (e < ne) {
                    const int y = fdiv(e, g.fm3), z = e - y * g.m3;
                    tile[y * g.P + z] = v[u];
                }
            }
        }
        __syncthreads();
        fft_tile<V, S1, E>(tile, stz, g.pz, g.m2, g.fm2, 1, g.P);
        fft_tile<V, S1, E>(tile, sty, g.py, g.m3, g.fm3, g.P, 1);
    } else {
        __syncthreads();
    }
    op.begin();
    constexpr int PB = sizeof(T) == 4 ? 8 : 4;
    for (int e0 = threadIdx.x; e0 < ne; e0 += PB * blockDim.x) {
        typename Op::Pre pre[PB];
#pragma unroll
        for (int k = 0; k < PB; ++k) {
            const int e = e0 + k * blockDim.x;
            if (e < ne) pre[k] = op.load(f, base + e);
        }
#pragma unroll
        for (int k = 0; k < PB; ++k) {
            const int e = e0 + k * blockDim.x;
            if (e < ne) {
                const int y = fdiv(e, g.fm3), z = e - y * g.m3;
                V v = S1 != 0 ? tile[y * g.P + z] : mkc<V>(T(0), T(0));
                v = op.apply(f, x, y, z, base + e, v, pre[k]);
                if (S2 != 0) tile[y * g.P + z] = v;
            }
        }
    }
    if (S2 != 0) {
        __syncthreads();
        fft_tile<V, S2, E>(tile, stz, g.pz, g.m2, g.fm2, 1, g.P);
        fft_tile<V, S2, E>(tile, sty, g.py, g.m3, g.fm3, g.P, 1);
        for (int e = threadIdx.x; e < ne; e += blockDim.x) {
            const int y = fdiv(e, g.fm3), z = e - y * g.m3;
            dst[base + e] = tile[y * g.P + z];
        }
    }
    op.end(reinterpret_cast<double*>(tile), blockIdx.x + (size_t)blockIdx.y * gridDim.x);
}

// ---------------------------------------------------------------------------
// z-line pass: grid (m1*m2/B, nfields); B rows of m3 per CTA.
// Shared memory: tile[B][P] (P = m3 + 1) + twiddles(m3).
// ---------------------------------------------------------------------------
template <typename T, int E, int S1, int S2, class Op>
__global__ void __launch_bounds__(256, 2) k_zline(LineGeom g, const cplx<T>* src, cplx<T>* dst,
                                                size_t fstride, const cplx<T>* __restrict__ twz, Op op)
{
    using V = cplx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    V* st = tile + (size_t)g.B * g.P;
    const int f = blockIdx.y;
    const int ne = g.B * g.m3;
    const int row0 = blockIdx.x * g.B;
    const size_t base = (size_t)f * fstride + (size_t)row0 * g.m3;
    if (S1 != 0 || S2 != 0) load_twiddles(st, twz, g.m3);
    if (S1 != 0) {
        for (int e = threadIdx.x; e < ne; e += blockDim.x) {
            const int b = fdiv(e, g.fm3), z = e - b * g.m3;
            tile[b * g.P + z] = src[base + e];
        }
        __syncthreads();
        fft_tile<V, S1, E>(tile, st, g.p, g.B, g.fB, 1, g.P);
    } else {
        __syncthreads();
    }
    op.begin();
    constexpr int PB = sizeof(T) == 4 ? 8 : 4;
    for (int e0 = threadIdx.x; e0 < ne; e0 += PB * blockDim.x) {
        typename Op::Pre pre[PB];
#pragma unroll
        for (int k = 0; k < PB; ++k) {
            const int e = e0 + k * blockDim.x;
            if (e < ne) pre[k] = op.load(f, base + e);
        }
#pragma unroll
        for (int k = 0; k < PB; ++k) {
            const int e = e0 + k * blockDim.x;
            if (e < ne) {
                const int b = fdiv(e, g.fm3), z = e - b * g.m3;
                const int row = row0 + b;
                const int x = fdiv(row, g.fm2), y = row - x * g.m2;
                V v = S1 != 0 ? tile[b * g.P + z] : mkc<V>(T(0), T(0));
                v = op.apply(f, x, y, z, base + e, v, pre[k]);
                if (S2 != 0) tile[b * g.P + z] = v;
            }
        }
    }
    if (S2 != 0) {
        __syncthreads();
        fft_tile<V, S2, E>(tile, st, g.p, g.B, g.fB, 1, g.P);
        for (int e = threadIdx.x; e < ne; e += blockDim.x) {
            const int b = fdiv(e, g.fm3), z = e - b * g.m3;
            dst[base + e] = tile[b * g.P + z];
        }
    }
    op.end(reinterpret_cast<double*>(tile), blockIdx.x + (size_t)blockIdx.y * gridDim.x);
}

// ---------------------------------------------------------------------------
// Strided pass along y (DIM = 1) or x (DIM = 0): grid (outer * m3/W, nf).
// Tile[n][W] (pitch W) of lines; the outer index is x for DIM 1, y for DIM 0.
// ---------------------------------------------------------------------------
template <typename T, int E, int DIM, int S1, int S2, class Op>
__global__ void __launch_bounds__(256, 2) k_strided(LineGeom g, const cplx<T>* src, cplx<T>* dst,
                                                  size_t fstride, const cplx<T>* __restrict__ tw, Op op)
{
    using V = cplx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    V* st = tile + (size_t)g.n * g.W;
    const int nzb = g.m3 / g.W;
    const int outer = blockIdx.x / nzb;
    const int z0 = (blockIdx.x - outer * nzb) * g.W;
    const int f = blockIdx.y;
    const size_t plane = (size_t)g.m2 * g.m3;
    const size_t lstride = DIM == 1 ? (size_t)g.m3 : plane;
    const size_t base = (size_t)f * fstride + (DIM == 1 ? (size_t)outer * plane : (size_t)outer * g.m3) + z0;
    const int ne = g.n * g.W;
    if (S1 != 0 || S2 != 0) load_twiddles(st, tw, g.n);
    if (S1 != 0) {
        for (int e0 = threadIdx.x; e0 < ne; e0 += 4 * blockDim.x) {
            V v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = e0 + u * blockDim.x;
                if (e < ne) {
                    const int j = fdiv(e, g.fW), w = e - j * g.W;
                    v[u] = src[base + j * lstride + w];
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = e0 + u * blockDim.x;
                if (e < ne) tile[e] = v[u];
            }
        }
        __syncthreads();
        fft_tile<V, S1, E>(tile, st, g.p, g.W, g.fW, g.W, 1);
    } else {
        __syncthreads();
    }
    op.begin();
    constexpr int PB = sizeof(T) == 4 ? 8 : 4;
    for (int e0 = threadIdx.x; e0 < ne; e0 += PB * blockDim.x) {
        typename Op::Pre pre[PB];
#pragma unroll
        for (int k = 0; k < PB; ++k) {
            const int e = e0 + k * blockDim.x;
            if (e < ne) {
                const int j = fdiv(e, g.fW), w = e - j * g.W;
                pre[k] = op.load(f, base + j * lstride + w);
            }
        }
#pragma unroll
        for (int k = 0; k < PB; ++k) {
            const int e = e0 + k * blockDim.x;
            if (e < ne) {
                const int j = fdiv(e, g.fW), w = e - j * g.W;
                const int x = DIM == 1 ? outer : j;
                const int y = DIM == 1 ? j : outer;
                const size_t off = base + j * lstride + w;
                V v = S1 != 0 ? tile[e] : mkc<V>(T(0), T(0));
                v = op.apply(f, x, y, z0 + w, off, v, pre[k]);
                if (S2 != 0) tile[e] = v;
            }
        }
    }
    pdl_trigger();
    if (S2 != 0) {
        __syncthreads();
        fft_tile<V, S2, E>(tile, st, g.p, g.W, g.fW, g.W, 1);
        for (int e = threadIdx.x; e < ne; e += blockDim.x) {
            const int j = fdiv(e, g.fW), w = e - j * g.W;
            dst[base + j * lstride + w] = tile[e];
        }
    }
    op.end(reinterpret_cast<double*>(tile), blockIdx.x + (size_t)blockIdx.y * gridDim.x);
}

// ---------------------------------------------------------------------------
// Pointwise ops
// ---------------------------------------------------------------------------
// Op interface: begin() once per thread; load(f, g) issues the global loads
// an element needs and returns them (the kernels batch PB elements so that
// many loads are in flight); apply(f, x, y, z, g, v, pre) does the element's
// arithmetic and stores and returns the value for the second transform;
// end(scratch, cta) closes per-block reductions.
template <typename T>
struct OpIdentity {
    struct Pre {};
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ Pre load(int, size_t) const { return Pre{}; }
    __device__ __forceinline__ cplx<T> apply(int, int, int, int, size_t, cplx<T> v, const Pre&) const { return v; }
    __device__ __forceinline__ void end(double*, size_t) {}
};

// Power-of-two renormalisation of the propagators (all optional: a null eF
// turns it off).  Each real-space segment pass records, per CTA, the largest
// component magnitude of the propagator it wrote (pmax_cur); the next pass of
// the same sweep reduces those maxima, scales its output by 2^-d with
// d = floor(log2 max), and accumulates d into a per-segment exponent:
//   qF[s] is stored as qF_true[s] 2^-aF[s],  qB[s] as qB_true[s] 2^-aB[s].
// Scaling by powers of two is exact in binary floating point, so complex128
// results are unchanged while complex64 propagators stay in range.  A density
// or stress contribution of segment s then carries 2^(aF[s] + aB[s+1] - aF[N-1])
// (the partition function is Q_true = mean(qF[N-1]) 2^aF[N-1]).
struct Renorm {
    int* eF;                 // forward exponents aF[0..N) (null: no renormalisation)
    int* eB;                 // backward exponents aB[0..N)
    const float* pmax_prev;  // per-CTA maxima written by the previous pass of this sweep
    float* pmax_cur;         // per-CTA maxima of this pass
    int nparts;              // number of entries of pmax_prev
    int s;                   // segment index of this pass
    int N;                   // segments of the species
};

// the exponent floor(log2 max) of the previous pass's per-CTA maxima; m is
// this thread's share of them (its strided elements), loaded beforehand
__device__ __forceinline__ int reduce_exponent_local(float m)
{
    __shared__ float s_red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float r = 0.0f;
        for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) r = fmaxf(r, s_red[w]);
        s_red[0] = r;
    }
    __syncthreads();
    const float M = s_red[0];
    __syncthreads();
    return (M > 0.0f && isfinite(M)) ? ilogbf(M) : 0;
}

__device__ __forceinline__ float local_max(const float* pm, int n)
{
    float m = 0.0f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmaxf(m, pm[i]);
    return m;
}

__device__ __forceinline__ int reduce_exponent(const float* pm, int n) { return reduce_exponent_local(local_max(pm, n)); }

// Chain-propagator pointwise work in the real-space pass of one segment.
// KIND selects the sweep position:
//   forward : q = u * E (u = IFFT of the previous bond, or 1 at s = 0);
//             q is stored as qF[s]; the last segment also sums q for Q.
//   backward: u = exp(+W_s) qB[s] (the previous transform's output, or 1 at
//             s = N-1); phi = qF[s] * u is accumulated into the per-type
//             and charge densities with the species factor (n/V)/Q; the
//             propagation continues with qB[s] = u * E.
enum PropKind { FWD_START = 0, FWD_MID = 1, FWD_LAST = 2, FWD_SINGLE = 3, BWD_START = 4, BWD_MID = 5, BWD_LAST = 6, BWD_SINGLE = 7 };

// Bulk prefetch of a contiguous global range into L2 (the TMA unit's
// non-blocking prefetch: no shared memory, no barrier, nothing to wait on).
// Address 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void l2_prefetch_bulk(const void* p, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

template <typename T, int KIND>
struct OpProp {
    using V = cplx<T>;
    const V* E;              // exp(-W) of the segment's class
    V* qstore;               // forward: qF[s]
    const V* qread;          // backward: qF[s]
    V* rho_type;             // backward: density accumulator of the segment's type
    V* rho_charge;           // backward: charge accumulator (null when z == 0)
    T z;                     // segment valence
    const double2* factor;   // backward: species factor (n/V)/Q (Q of the stored, scaled qF)
    double2* partial;        // forward last: per-CTA sums of q
    Renorm rn;               // renormalisation (rn.eF null: off)
    bool store_u;            // forward: store u = q / E (renormalised) instead of q
    double acc[2];
    float amax;
    float pm_local;          // this thread's share of the previous maxima (preload)
    bool preloaded;
    T fr, fi;                // density factor (with the segment's exponent folded in)
    T oscale;                // output scale 2^-d

    static constexpr bool FWD = KIND <= FWD_SINGLE;
    static constexpr bool NEED_E = KIND == FWD_START || KIND == FWD_MID || KIND == FWD_LAST || KIND == FWD_SINGLE ||
                                   KIND == BWD_START || KIND == BWD_MID;
    // global loads per point (the forward passes read only the class table)
    static constexpr int LOADS = FWD ? 1 : 4;
    static constexpr bool MAX_OUT = KIND == FWD_START || KIND == FWD_MID || KIND == BWD_START || KIND == BWD_MID;
    struct Pre {
        V e, q, r, c;
    };

    // loads the previous pass's per-CTA maxima early (kernels that call it
    // right after the dependency wait hide the latency behind their first
    // transform stages; begin() reduces them)
    __device__ __forceinline__ void preload()
    {
        preloaded = false;
        if ((KIND == FWD_MID || KIND == FWD_LAST || KIND == BWD_MID) && rn.eF) {
            pm_local = local_max(rn.pmax_prev, rn.nparts);
            preloaded = true;
        }
    }
    __device__ __forceinline__ void begin()
    {
        acc[0] = acc[1] = 0.0;
        amax = 0.0f;
        oscale = T(1);
        int dens_exp = 0;
        if (rn.eF) {
            const bool first = blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0;
            if (KIND == FWD_START || KIND == FWD_SINGLE) {
                if (first) rn.eF[0] = 0;
            } else if (KIND == FWD_MID || KIND == FWD_LAST) {
                const int d = preloaded ? reduce_exponent_local(pm_local) : reduce_exponent(rn.pmax_prev, rn.nparts);
                oscale = (T)ldexp(1.0, -d);
                if (first) rn.eF[rn.s] = rn.eF[rn.s - 1] + d;
            } else if (KIND == BWD_START || KIND == BWD_SINGLE) {
                if (first) rn.eB[rn.s] = 0;
            } else if (KIND == BWD_MID) {
                const int d = preloaded ? reduce_exponent_local(pm_local) : reduce_exponent(rn.pmax_prev, rn.nparts);
                oscale = (T)ldexp(1.0, -d);
                if (first) rn.eB[rn.s] = rn.eB[rn.s + 1] + d;
                dens_exp = rn.eF[rn.s] + rn.eB[rn.s + 1] - rn.eF[rn.N - 1];
            } else {   // BWD_LAST (s = 0)
                dens_exp = rn.eF[0] + rn.eB[1] - rn.eF[rn.N - 1];
            }
        }
        if (!FWD) {
            const double2 fc = *factor;
            fr = T(ldexp(fc.x, dens_exp));
            fi = T(ldexp(fc.y, dens_exp));
        }
    }
    __device__ __forceinline__ Pre load(int, size_t g) const
    {
        Pre p;
        if (NEED_E) p.e = E[g];
        if (!FWD) {
            p.q = qread[g];
            p.r = rho_type[g];
            if (rho_charge) p.c = rho_charge[g];
        }
        return p;
    }
    // the operands of the pointwise step of one plane (elements g0 .. g0+n),
    // requested at kernel start so that the loads after the inverse transform
    // find them in L2
    __device__ __forceinline__ void prefetch(size_t g0, unsigned n) const
    {
        const unsigned bytes = n * (unsigned)sizeof(V);
        if (NEED_E) l2_prefetch_bulk(E + g0, bytes);
        if (!FWD) {
            l2_prefetch_bulk(qread + g0, bytes);
            l2_prefetch_bulk(rho_type + g0, bytes);
            if (rho_charge) l2_prefetch_bulk(rho_charge + g0, bytes);
        }
    }
    __device__ __forceinline__ void track(V q)
    {
        if (MAX_OUT) amax = fmaxf(amax, fmaxf(fabsf((float)q.x), fabsf((float)q.y)));
    }
    __device__ __forceinline__ V apply(int, int, int, int, size_t g, V u, const Pre& p)
    {
        if (FWD) {
            V q = (KIND == FWD_START || KIND == FWD_SINGLE) ? p.e : cmul(u, p.e);
            if (KIND == FWD_MID || KIND == FWD_LAST) q = cscale(q, oscale);
            if (store_u) {
                if (KIND == FWD_MID || KIND == FWD_LAST) qstore[g] = cscale(u, oscale);
            } else {
                qstore[g] = q;
            }
            track(q);
            if (KIND == FWD_LAST || KIND == FWD_SINGLE) {
                acc[0] += (double)q.x;
                acc[1] += (double)q.y;
            }
            return q;
        } else {
            const V phi = (KIND == BWD_START || KIND == BWD_SINGLE) ? p.q : cmul(p.q, u);
            const V w = cmul(phi, mkc<V>(fr, fi));
            rho_type[g] = cadd(p.r, w);
            if (rho_charge) rho_charge[g] = cadd(p.c, cscale(w, z));
            if (KIND == BWD_START) {
                track(p.e);
                return p.e;
            }
            if (KIND == BWD_MID) {
                const V q = cscale(cmul(u, p.e), oscale);
                track(q);
                return q;
            }
            return u;
        }
    }
    __device__ __forceinline__ void end(double* scratch, size_t cta)
    {
        if (KIND == FWD_LAST || KIND == FWD_SINGLE) {
            __syncthreads();
            block_sum<2>(acc, scratch);
            if (threadIdx.x == 0) partial[cta] = make_double2(acc[0], acc[1]);
        }
        if (MAX_OUT && rn.eF) {
            __syncthreads();
            float* sm = reinterpret_cast<float*>(scratch);
            float m = amax;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
            __syncthreads();
            if (threadIdx.x == 0) {
                float r = 0.0f;
                for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) r = fmaxf(r, sm[w]);
                rn.pmax_cur[cta] = r;
            }
        }
    }
};

// Bond pointwise work in the k-space (x) pass of one bond s -> s+1.
//   forward : F = DFT(qF[s]) (sign -1); optionally stored for the stress;
//             output F * Phi_s / V.
//   backward: B' = DFT_{+}(qB[s+1]) (sign +1, i.e. B(-k)); optionally the
//             connectivity stress sums  sum_k k_a k_b Phi_s F_s B'  (weighted
//             by b_s^2 and the species factor) are accumulated; output
//             B' * Phi_s / V.
// Phi_s(k) = exp(-b^2 k^2/6) is separable: phix[kx] phiy[ky] phiz[kz].
template <typename T, bool FWD, bool STRESS>
struct OpBond {
    using V = cplx<T>;
    V* Fstore;
    const V* Fread;
    const T* phix;
    const T* phiy;
    const T* phiz;
    const double* kx;
    const double* ky;
    const double* kz;
    T invV;
    double b2;
    const double2* factor;
    double2* partial;        // [cta][6] accumulated across bonds
    const int* eF;           // renormalisation exponents (null: off)
    const int* eB;
    int s, N;                // bond s -> s+1 of a species with N segments
    double acc[12];
    // resident CTAs per SM asked of the fused bond pass: without the stress
    // sums it fits 64 registers, so a 128^3 pass (1024 CTAs of 128 threads)
    // runs in one wave; with them, fewer registers would spill
    static constexpr int FUSED_MIN_BLOCKS = STRESS ? 2 : 8;
    struct Pre {
        V F;
    };

    __device__ __forceinline__ void begin()
    {
        if (STRESS) {
#pragma unroll
            for (int c = 0; c < 12; ++c) acc[c] = 0.0;
        }
    }
    __device__ __forceinline__ Pre load(int, size_t g) const
    {
        Pre p;
        if (!FWD && STRESS) p.F = Fread[g];
        return p;
    }
    __device__ __forceinline__ V apply(int, int x, int y, int z, size_t g, V v, const Pre& pre)
    {
        // read-only loads: they do not alias the Fstore writes, so the y and z
        // factors (fixed for a thread's column) are loaded once
        const T phi = __ldg(phix + x) * __ldg(phiy + y) * __ldg(phiz + z);
        if (FWD) {
            if (Fstore) Fstore[g] = v;
        } else if (STRESS) {
            const V F = pre.F;
            const V p = cmul(F, v);
            const double pr = (double)p.x * (double)phi, pi = (double)p.y * (double)phi;
            const double ax = kx[x], ay = ky[y], az = kz[z];
            const double kk[6] = {ax * ax, ay * ay, az * az, ax * ay, ax * az, ay * az};
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                acc[2 * c] += kk[c] * pr;
                acc[2 * c + 1] += kk[c] * pi;
            }
        }
        return cscale(v, phi * invV);
    }
    __device__ __forceinline__ void end(double* scratch, size_t cta)
    {
        if (STRESS) {
            __syncthreads();
            block_sum<12>(acc, scratch);
            if (threadIdx.x == 0) {
                const double2 fc = *factor;
                const double w = eF ? ldexp(b2, eF[s] + eB[s + 1] - eF[N - 1]) : b2;
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    const double sr = w * acc[2 * c], si = w * acc[2 * c + 1];
                    double2 o = partial[cta * 6 + c];
                    o.x += sr * fc.x - si * fc.y;
                    o.y += sr * fc.y + si * fc.x;
                    partial[cta * 6 + c] = o;
                }
            }
        }
    }
};

}  // namespace ftsp

namespace ftsp {


// ---------------------------------------------------------------------------
// Compile-time specialisations of the three passes for production grids.
// Same structure and Op interface as the runtime-plan kernels above; all
// sizes are template constants.
// ---------------------------------------------------------------------------

// Plane pass for an m2 = m3 = N plane, NT threads, E elements per thread.
template <typename T, int N, int RMAX, int NT, int E, int S1, int S2, class Op>
__global__ void __launch_bounds__(NT, 1) k_plane_ct(const cplx<T>* src, cplx<T>* dst, size_t fstride,
                                                    const cplx<T>* __restrict__ twn, Op op)
{
    using V = cplx<T>;
    constexpr int P = N + 1, NE = N * N;
    static_assert(NE <= NT * E, "plane does not fit the thread block");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    V* stw = tile + N * P;
    const int x = blockIdx.x;
    const int f = blockIdx.y;
    const size_t base = (size_t)f * fstride + (size_t)x * NE;
    if (S1 != 0 || S2 != 0)
        for (int j = threadIdx.x; j < N; j += NT) stw[j] = twn[j];
    pdl_wait();
    constexpr int EPT = (NE + NT - 1) / NT;   // elements per thread
    if (S1 != 0) {
        V v[EPT];   // every load of the thread in flight before the first smem store
#pragma unroll
        for (int u = 0; u < EPT; ++u) {
            const int e = threadIdx.x + u * NT;
            if (NE % NT == 0 || e < NE) v[u] = src[base + e];
        }
#pragma unroll
        for (int u = 0; u < EPT; ++u) {
            const int e = threadIdx.x + u * NT;
            if (NE % NT == 0 || e < NE) tile[(e / N) * P + e % N] = v[u];
        }
        __syncthreads();
        ct_fft<V, S1, N, RMAX, N, 1, P, NT, E>(tile, stw);   // z-lines
        ct_fft<V, S1, N, RMAX, N, P, 1, NT, E>(tile, stw);   // y-lines
    } else {
        __syncthreads();
    }
    op.begin();
    constexpr int PB = (sizeof(T) == 4 && NT < 1024) ? 8 : 4;
#pragma unroll 1
    for (int u0 = 0; u0 < EPT; u0 += PB) {
        typename Op::Pre pre[PB];
#pragma unroll
        for (int k = 0; k < PB; ++k) {
            const int e = threadIdx.x + (u0 + k) * NT;
            if (u0 + k < EPT && (NE % NT == 0 || e < NE)) pre[k] = op.load(f, base + e);
        }
#pragma unroll
        for (int k = 0; k < PB; ++k) {
            const int e = threadIdx.x + (u0 + k) * NT;
            if (u0 + k < EPT && (NE % NT == 0 || e < NE)) {
                const int y = e / N, z = e % N;
                V v = S1 != 0 ? tile[y * P + z] : mkc<V>(T(0), T(0));
                v = op.apply(f, x, y, z, base + e, v, pre[k]);
                if (S2 != 0) tile[y * P + z] = v;
            }
        }
    }
    pdl_trigger();
    if (S2 != 0) {
        __syncthreads();
        ct_fft<V, S2, N, RMAX, N, 1, P, NT, E>(tile, stw);
        ct_fft<V, S2, N, RMAX, N, P, 1, NT, E>(tile, stw);
        for (int e = threadIdx.x; e < NE; e += NT) dst[base + e] = tile[(e / N) * P + e % N];
    }
    op.end(reinterpret_cast<double*>(tile), blockIdx.x + (size_t)blockIdx.y * gridDim.x);
}

// Plane pass with both transforms (the mid segment passes), two
// shared-memory round trips fewer than k_plane_ct: the inverse transform
// runs along y first, and the coalesced load of thread tid (rows
// tid/N + u*NT/N of column tid%N) is the input set of its first radix stage
// along y, so that stage runs on the loaded registers; the forward
// transform ends along y, and its last stage stores its outputs (rows
// i + t*SPAN of the column) straight to global memory.  Same grid, Op
// interface and results (up to the rounding of the axis order) as
// k_plane_ct.
template <int N, int RMAX, int NT, int E>
__host__ __device__ constexpr bool plane_fused_ok()
{
    constexpr int NST = ct_nst(N, RMAX);
    if (NST < 2 || NT % N != 0) return false;
    using A0 = CtSt<N, RMAX, N, NT, 0, false>;
    using AL = CtSt<N, RMAX, N, NT, NST - 1, false>;
    return A0::NB * A0::R == E && (A0::M * N) % NT == 0 && A0::TOTAL % NT == 0 && AL::NB * AL::R == E &&
           AL::TOTAL % NT == 0 && N * N == NT * E;
}

template <typename T, int N, int RMAX, int NT, int E, int S1, int S2, class Op>
__global__ void __launch_bounds__(NT, 1) k_plane_fused(const cplx<T>* src, cplx<T>* dst, size_t fstride,
                                                       const cplx<T>* __restrict__ twn, Op op)
{
    using V = cplx<T>;
    constexpr int P = N + 1, NE = N * N;
    constexpr int NST = ct_nst(N, RMAX);
    static_assert(S1 != 0 && S2 != 0, "the fused plane pass runs both transforms");
    static_assert(plane_fused_ok<N, RMAX, NT, E>(), "plane shape not supported by the fused pass");
    using A0 = CtSt<N, RMAX, N, NT, 0, false>;          // first y stage (line = z column)
    using AL = CtSt<N, RMAX, N, NT, NST - 1, false>;    // last y stage
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    V* stw = tile + N * P;
    const int x = blockIdx.x;
    const int f = blockIdx.y;
    const size_t base = (size_t)f * fstride + (size_t)x * NE;
    for (int j = threadIdx.x; j < N; j += NT) stw[j] = twn[j];
    // the L2 prefetch of the pointwise operands goes out before the wait for
    // the previous pass: a prefetch only moves lines into L2, the device's
    // point of coherence, so it cannot observe a stale value, and the class
    // table (the bulk of it) is not written during a sweep
    if (threadIdx.x == 0) op.prefetch(base, (unsigned)NE);
    pdl_wait();
    op.preload();
    V v[E];   // value u: row tid/N + u*NT/N, column tid%N
#pragma unroll
    for (int u = 0; u < E; ++u) v[u] = src[base + threadIdx.x + u * NT];
    __syncthreads();   // twiddles in shared memory
    {
        V a[A0::NB][A0::R];
#pragma unroll
        for (int q = 0; q < A0::NB; ++q)
#pragma unroll
            for (int t = 0; t < A0::R; ++t) a[q][t] = v[q + t * (A0::M * N / NT)];
        st_butterfly<S1, A0>(a, stw);
        st_scatter<A0, P, 1>(tile, a);
        __syncthreads();
    }
    st_range<V, S1, N, RMAX, N, P, 1, NT, false, 1, NST>(tile, stw);   // rest of y
    ct_fft<V, S1, N, RMAX, N, 1, P, NT, E>(tile, stw);                  // z-lines
    op.begin();
    constexpr int EPT = NE / NT;
    // loads in flight per batch: every FFT value is in shared memory here,
    // so the registers hold the operands of PB points
    constexpr int PB = (sizeof(T) == 4 && Op::LOADS <= 1) ? 16 : 4;
#pragma unroll 1
    for (int u0 = 0; u0 < EPT; u0 += PB) {
        typename Op::Pre pre[PB];
#pragma unroll
        for (int k = 0; k < PB; ++k)
            if (u0 + k < EPT) pre[k] = op.load(f, base + threadIdx.x + (u0 + k) * NT);
#pragma unroll
        for (int k = 0; k < PB; ++k)
            if (u0 + k < EPT) {
                const int e = threadIdx.x + (u0 + k) * NT;
                const int y = e / N, z = e % N;
                tile[y * P + z] = op.apply(f, x, y, z, base + e, tile[y * P + z], pre[k]);
            }
    }
    pdl_trigger();
    __syncthreads();
    ct_fft<V, S2, N, RMAX, N, 1, P, NT, E>(tile, stw);                  // z-lines
    st_range<V, S2, N, RMAX, N, P, 1, NT, false, 0, NST - 1>(tile, stw);
    {
        V a[AL::NB][AL::R];
        st_gather<AL, P, 1>(tile, a);
        st_butterfly<S2, AL>(a, stw);
#pragma unroll
        for (int q = 0; q < AL::NB; ++q)
#pragma unroll
            for (int t = 0; t < AL::R; ++t) dst[base + (size_t)AL::out_pos(q, t) * N + AL::line(q)] = a[q][t];
    }
    op.end(reinterpret_cast<double*>(tile), blockIdx.x + (size_t)blockIdx.y * gridDim.x);
}

// Strided pass: lines of length N along y (DIM 1, outer index x) or x (DIM 0,
// outer index y), W contiguous z-columns per tile; grid (outer * M3/W, nf).
template <typename T, int N, int W, int DIM, int RMAX, int NT, int E, int S1, int S2, class Op>
__global__ void __launch_bounds__(NT, 2) k_strided_ct(int m2, int m3, const cplx<T>* src, cplx<T>* dst,
                                                      size_t fstride, const cplx<T>* __restrict__ twn, Op op)
{
    using V = cplx<T>;
    constexpr int NE = N * W;
    static_assert(NE <= NT * E, "tile does not fit the thread block");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    V* stw = tile + NE;
    const int nzb = m3 / W;
    const int outer = blockIdx.x / nzb;
    const int z0 = (blockIdx.x - outer * nzb) * W;
    const int f = blockIdx.y;
    const size_t plane = (size_t)m2 * m3;
    const size_t lstride = DIM == 1 ? (size_t)m3 : plane;
    const size_t base = (size_t)f * fstride + (DIM == 1 ? (size_t)outer * plane : (size_t)outer * m3) + z0;
    if (S1 != 0 || S2 != 0)
        for (int j = threadIdx.x; j < N; j += NT) stw[j] = twn[j];
    pdl_wait();
    constexpr int EPT = (NE + NT - 1) / NT;
    if (S1 != 0) {
        V v[EPT];
#pragma unroll
        for (int u = 0; u < EPT; ++u) {
            const int e = threadIdx.x + u * NT;
            if (NE % NT == 0 || e < NE) v[u] = src[base + (e / W) * lstride + e % W];
        }
#pragma unroll
        for (int u = 0; u < EPT; ++u) {
            const int e = threadIdx.x + u * NT;
            if (NE % NT == 0 || e < NE) tile[e] = v[u];
        }
        __syncthreads();
        ct_fft<V, S1, N, RMAX, W, W, 1, NT, E>(tile, stw);
    } else {
        __syncthreads();
    }
    op.begin();
    constexpr int PB = (sizeof(T) == 4 && NT < 1024) ? 8 : 4;
#pragma unroll 1
    for (int u0 = 0; u0 < EPT; u0 += PB) {
        typename Op::Pre pre[PB];
#pragma unroll
        for (int k = 0; k < PB; ++k) {
            const int e = threadIdx.x + (u0 + k) * NT;
            if (u0 + k < EPT && (NE % NT == 0 || e < NE)) pre[k] = op.load(f, base + (e / W) * lstride + e % W);
        }
#pragma unroll
        for (int k = 0; k < PB; ++k) {
            const int e = threadIdx.x + (u0 + k) * NT;
            if (u0 + k < EPT && (NE % NT == 0 || e < NE)) {
                const int j = e / W, w = e % W;
                const int x = DIM == 1 ? outer : j;
                const int y = DIM == 1 ? j : outer;
                const size_t off = base + j * lstride + w;
                V v = S1 != 0 ? tile[e] : mkc<V>(T(0), T(0));
                v = op.apply(f, x, y, z0 + w, off, v, pre[k]);
                if (S2 != 0) tile[e] = v;
            }
        }
    }
    pdl_trigger();
    if (S2 != 0) {
        __syncthreads();
        ct_fft<V, S2, N, RMAX, W, W, 1, NT, E>(tile, stw);
        for (int e = threadIdx.x; e < NE; e += NT) dst[base + (e / W) * lstride + e % W] = tile[e];
    }
    op.end(reinterpret_cast<double*>(tile), blockIdx.x + (size_t)blockIdx.y * gridDim.x);
}

// Strided pass with both transforms (the bond pass), shared-memory round
// trips cut to the stages that need them.  The coalesced load of thread
// tid (positions tid/W + u*NT/W of column tid%W) is the input set of its
// first-stage butterflies, so stage 0 runs on the loaded registers; the
// second transform runs in reversed radix order, so the last stage of the
// first transform, the pointwise op and the first stage of the second stay
// in registers; the last stage stores its outputs (positions i + t*SPAN of
// the column) straight to global memory.  For N = 128 (radix 16 x 8) that is
// two shared-memory round trips instead of six.  Same grid, Op interface and
// results (up to the rounding of the second transform's radix order) as
// k_strided_ct.
template <int N, int W, int RMAX, int NT, int E>
__host__ __device__ constexpr bool strided_fused_ok()
{
    constexpr int NST = ct_nst(N, RMAX);
    if (NST < 2 || NT % W != 0) return false;
    using A0 = CtSt<N, RMAX, W, NT, 0, false>;
    using AL = CtSt<N, RMAX, W, NT, NST - 1, false>;
    using BL = CtSt<N, RMAX, W, NT, NST - 1, true>;
    return A0::NB * A0::R == E && (A0::M * W) % NT == 0 && A0::TOTAL % NT == 0 && BL::NB * BL::R == E &&
           (BL::SPAN * W) % NT == 0 && BL::TOTAL % NT == 0 && AL::NB * AL::R == E && AL::TOTAL % NT == 0 &&
           N * W == NT * E;
}

// Source field of output field f of a pencil pass: Op::NSRC entries of
// Op::src where the op declares them (an output computed from another
// field's transform), else f.  The entries are read with constant indices.
template <class Op, class = void>
struct op_has_src : std::false_type {};
template <class Op>
struct op_has_src<Op, std::void_t<decltype(Op::NSRC)>> : std::true_type {};
template <class Op>
__device__ __forceinline__ int op_src_field(const Op& op, int f)
{
    if constexpr (op_has_src<Op>::value) {
        int s = f;
#pragma unroll
        for (int k = 0; k < Op::NSRC; ++k)
            if (k == f) s = op.src[k];
        return s;
    } else {
        return f;
    }
}

template <typename T, int N, int W, int DIM, int RMAX, int NT, int E, int S1, int S2, class Op>
__global__ void __launch_bounds__(NT, Op::FUSED_MIN_BLOCKS) k_strided_fused(int m2, int m3, const cplx<T>* src, cplx<T>* dst,
                                                         size_t fstride, const cplx<T>* __restrict__ twn, Op op)
{
    using V = cplx<T>;
    constexpr int NE = N * W;
    constexpr int NST = ct_nst(N, RMAX);
    static_assert(S1 != 0 && S2 != 0, "the fused pass runs both transforms");
    static_assert(strided_fused_ok<N, W, RMAX, NT, E>(), "tile shape not supported by the fused pass");
    using A0 = CtSt<N, RMAX, W, NT, 0, false>;          // first stage, first transform
    using AL = CtSt<N, RMAX, W, NT, NST - 1, false>;    // last stage, first transform
    using B0 = CtSt<N, RMAX, W, NT, 0, true>;           // first stage, second transform (radix of AL)
    using BL = CtSt<N, RMAX, W, NT, NST - 1, true>;     // last stage, second transform
    static_assert(B0::R == AL::R && B0::NB == AL::NB && B0::M == AL::SPAN, "stage mismatch");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    V* stw = tile + NE;
    const int nzb = m3 / W;
    const int outer = blockIdx.x / nzb;
    const int z0 = (blockIdx.x - outer * nzb) * W;
    const int f = blockIdx.y;
    const size_t plane = (size_t)m2 * m3;
    const size_t lstride = DIM == 1 ? (size_t)m3 : plane;
    const size_t inner = (DIM == 1 ? (size_t)outer * plane : (size_t)outer * m3) + z0;
    const size_t base = (size_t)f * fstride + inner;
    const size_t sbase = (size_t)op_src_field(op, f) * fstride + inner;
    for (int j = threadIdx.x; j < N; j += NT) stw[j] = twn[j];
    pdl_wait();
    // load: value u of the thread is position tid/W + u*NT/W of column tid%W
    V v[E];
#pragma unroll
    for (int u = 0; u < E; ++u) {
        const int e = threadIdx.x + u * NT;
        v[u] = src[sbase + (e / W) * lstride + e % W];
    }
    __syncthreads();   // twiddles in shared memory
    {
        V a[A0::NB][A0::R];
#pragma unroll
        for (int q = 0; q < A0::NB; ++q)
#pragma unroll
            for (int t = 0; t < A0::R; ++t) a[q][t] = v[q + t * (A0::M * W / NT)];
        st_butterfly<S1, A0>(a, stw);
        st_scatter<A0, W, 1>(tile, a);
        __syncthreads();
    }
    st_range<V, S1, N, RMAX, W, W, 1, NT, false, 1, NST - 1>(tile, stw);
    op.begin();
    {
        V a[AL::NB][AL::R];
        st_gather<AL, W, 1>(tile, a);
        typename Op::Pre pre[AL::NB][AL::R];
#pragma unroll
        for (int q = 0; q < AL::NB; ++q)
#pragma unroll
            for (int t = 0; t < AL::R; ++t)
                pre[q][t] = op.load(f, base + (size_t)AL::out_pos(q, t) * lstride + AL::line(q));
        __syncthreads();   // every gather done before the tile is rewritten
        st_butterfly<S1, AL>(a, stw);
#pragma unroll
        for (int q = 0; q < AL::NB; ++q)
#pragma unroll
            for (int t = 0; t < AL::R; ++t) {
                const int j = AL::out_pos(q, t), w = AL::line(q);
                const int x = DIM == 1 ? outer : j;
                const int y = DIM == 1 ? j : outer;
                a[q][t] = op.apply(f, x, y, z0 + w, base + (size_t)j * lstride + w, a[q][t], pre[q][t]);
            }
        pdl_trigger();
        st_butterfly<S2, B0>(a, stw);
        st_scatter<B0, W, 1>(tile, a);
        __syncthreads();
    }
    st_range<V, S2, N, RMAX, W, W, 1, NT, true, 1, NST - 1>(tile, stw);
    {
        V a[BL::NB][BL::R];
        st_gather<BL, W, 1>(tile, a);
        st_butterfly<S2, BL>(a, stw);
#pragma unroll
        for (int q = 0; q < BL::NB; ++q)
#pragma unroll
            for (int t = 0; t < BL::R; ++t)
                dst[base + (size_t)BL::out_pos(q, t) * lstride + BL::line(q)] = a[q][t];
    }
    op.end(reinterpret_cast<double*>(tile), blockIdx.x + (size_t)blockIdx.y * gridDim.x);
}

// Strided pass with one transform after the op (S1 = 0: the field loads of
// the batched 3-D transforms).  The op's values for the loaded positions
// (tid/W + u*NT/W of column tid%W) are the first-stage inputs, so stage 0
// runs on registers, and the last stage stores straight to global memory.
template <typename T, int N, int W, int DIM, int RMAX, int NT, int E, int S2, class Op>
__global__ void __launch_bounds__(NT, 2) k_strided_load_fused(int m2, int m3, cplx<T>* dst, size_t fstride,
                                                              const cplx<T>* __restrict__ twn, Op op)
{
    using V = cplx<T>;
    constexpr int NE = N * W;
    constexpr int NST = ct_nst(N, RMAX);
    static_assert(S2 != 0, "one transform");
    static_assert(strided_fused_ok<N, W, RMAX, NT, E>(), "tile shape not supported by the fused pass");
    using A0 = CtSt<N, RMAX, W, NT, 0, false>;
    using AL = CtSt<N, RMAX, W, NT, NST - 1, false>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    V* stw = tile + NE;
    const int nzb = m3 / W;
    const int outer = blockIdx.x / nzb;
    const int z0 = (blockIdx.x - outer * nzb) * W;
    const int f = blockIdx.y;
    const size_t plane = (size_t)m2 * m3;
    const size_t lstride = DIM == 1 ? (size_t)m3 : plane;
    const size_t base = (size_t)f * fstride + (DIM == 1 ? (size_t)outer * plane : (size_t)outer * m3) + z0;
    for (int j = threadIdx.x; j < N; j += NT) stw[j] = twn[j];
    pdl_wait();
    op.begin();
    V v[E];
    {
        typename Op::Pre pre[E];
#pragma unroll
        for (int u = 0; u < E; ++u) {
            const int e = threadIdx.x + u * NT;
            pre[u] = op.load(f, base + (e / W) * lstride + e % W);
        }
#pragma unroll
        for (int u = 0; u < E; ++u) {
            const int e = threadIdx.x + u * NT;
            const int j = e / W, w = e % W;
            const int x = DIM == 1 ? outer : j;
            const int y = DIM == 1 ? j : outer;
            v[u] = op.apply(f, x, y, z0 + w, base + j * lstride + w, mkc<V>(T(0), T(0)), pre[u]);
        }
    }
    pdl_trigger();
    __syncthreads();   // twiddles in shared memory
    {
        V a[A0::NB][A0::R];
#pragma unroll
        for (int q = 0; q < A0::NB; ++q)
#pragma unroll
            for (int t = 0; t < A0::R; ++t) a[q][t] = v[q + t * (A0::M * W / NT)];
        st_butterfly<S2, A0>(a, stw);
        st_scatter<A0, W, 1>(tile, a);
        __syncthreads();
    }
    st_range<V, S2, N, RMAX, W, W, 1, NT, false, 1, NST - 1>(tile, stw);
    {
        V a[AL::NB][AL::R];
        st_gather<AL, W, 1>(tile, a);
        st_butterfly<S2, AL>(a, stw);
#pragma unroll
        for (int q = 0; q < AL::NB; ++q)
#pragma unroll
            for (int t = 0; t < AL::R; ++t)
                dst[base + (size_t)AL::out_pos(q, t) * lstride + AL::line(q)] = a[q][t];
    }
    op.end(reinterpret_cast<double*>(tile), blockIdx.x + (size_t)blockIdx.y * gridDim.x);
}

// Plane pass with one transform after the op (S1 = 0): the op's values for
// the loaded positions (rows tid/N + u*NT/N of column tid%N) are the inputs
// of the first radix stage along y, which runs on registers; then the rest
// of y, then z, then the plane is stored from shared memory.
template <typename T, int N, int RMAX, int NT, int E, int S2, class Op>
__global__ void __launch_bounds__(NT, 1) k_plane_load_fused(cplx<T>* dst, size_t fstride,
                                                            const cplx<T>* __restrict__ twn, Op op)
{
    using V = cplx<T>;
    constexpr int P = N + 1, NE = N * N;
    constexpr int NST = ct_nst(N, RMAX);
    static_assert(S2 != 0, "one transform");
    static_assert(plane_fused_ok<N, RMAX, NT, E>(), "plane shape not supported by the fused pass");
    using A0 = CtSt<N, RMAX, N, NT, 0, false>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    V* stw = tile + N * P;
    const int x = blockIdx.x;
    const int f = blockIdx.y;
    const size_t base = (size_t)f * fstride + (size_t)x * NE;
    for (int j = threadIdx.x; j < N; j += NT) stw[j] = twn[j];
    pdl_wait();
    op.begin();
    V v[E];
    {
        typename Op::Pre pre[E];
#pragma unroll
        for (int u = 0; u < E; ++u) pre[u] = op.load(f, base + threadIdx.x + u * NT);
#pragma unroll
        for (int u = 0; u < E; ++u) {
            const int e = threadIdx.x + u * NT;
            v[u] = op.apply(f, x, e / N, e % N, base + e, mkc<V>(T(0), T(0)), pre[u]);
        }
    }
    pdl_trigger();
    __syncthreads();   // twiddles in shared memory
    {
        V a[A0::NB][A0::R];
#pragma unroll
        for (int q = 0; q < A0::NB; ++q)
#pragma unroll
            for (int t = 0; t < A0::R; ++t) a[q][t] = v[q + t * (A0::M * N / NT)];
        st_butterfly<S2, A0>(a, stw);
        st_scatter<A0, P, 1>(tile, a);
        __syncthreads();
    }
    st_range<V, S2, N, RMAX, N, P, 1, NT, false, 1, NST>(tile, stw);   // rest of y
    ct_fft<V, S2, N, RMAX, N, 1, P, NT, E>(tile, stw);                  // z-lines
    for (int e = threadIdx.x; e < NE; e += NT) dst[base + e] = tile[(e / N) * P + e % N];
    op.end(reinterpret_cast<double*>(tile), blockIdx.x + (size_t)blockIdx.y * gridDim.x);
}

// z-line pass: BR rows of length N per CTA; grid (m1*m2/BR, nf).
template <typename T, int N, int BR, int RMAX, int NT, int E, int S1, int S2, class Op>
__global__ void __launch_bounds__(NT, 2) k_zline_ct(int m2, const cplx<T>* src, cplx<T>* dst, size_t fstride,
                                                    const cplx<T>* __restrict__ twn, Op op)
{
    using V = cplx<T>;
    constexpr int P = N + 1, NE = BR * N;
    static_assert(NE <= NT * E, "tile does not fit the thread block");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    V* stw = tile + BR * P;
    const int f = blockIdx.y;
    const int row0 = blockIdx.x * BR;
    const size_t base = (size_t)f * fstride + (size_t)row0 * N;
    if (S1 != 0 || S2 != 0)
        for (int j = threadIdx.x; j < N; j += NT) stw[j] = twn[j];
    constexpr int EPT = (NE + NT - 1) / NT;
    if (S1 != 0) {
        V v[EPT];
#pragma unroll
        for (int u = 0; u < EPT; ++u) {
            const int e = threadIdx.x + u * NT;
            if (NE % NT == 0 || e < NE) v[u] = src[base + e];
        }
#pragma unroll
        for (int u = 0; u < EPT; ++u) {
            const int e = threadIdx.x + u * NT;
            if (NE % NT == 0 || e < NE) tile[(e / N) * P + e % N] = v[u];
        }
        __syncthreads();
        ct_fft<V, S1, N, RMAX, BR, 1, P, NT, E>(tile, stw);
    } else {
        __syncthreads();
    }
    op.begin();
    constexpr int PB = (sizeof(T) == 4 && NT < 1024) ? 8 : 4;
#pragma unroll 1
    for (int u0 = 0; u0 < EPT; u0 += PB) {
        typename Op::Pre pre[PB];
#pragma unroll
        for (int k = 0; k < PB; ++k) {
            const int e = threadIdx.x + (u0 + k) * NT;
            if (u0 + k < EPT && (NE % NT == 0 || e < NE)) pre[k] = op.load(f, base + e);
        }
#pragma unroll
        for (int k = 0; k < PB; ++k) {
            const int e = threadIdx.x + (u0 + k) * NT;
            if (u0 + k < EPT && (NE % NT == 0 || e < NE)) {
                const int b = e / N, z = e % N;
                const int row = row0 + b;
                const int x = row / m2, y = row - x * m2;
                V v = S1 != 0 ? tile[b * P + z] : mkc<V>(T(0), T(0));
                v = op.apply(f, x, y, z, base + e, v, pre[k]);
                if (S2 != 0) tile[b * P + z] = v;
            }
        }
    }
    if (S2 != 0) {
        __syncthreads();
        ct_fft<V, S2, N, RMAX, BR, 1, P, NT, E>(tile, stw);
        for (int e = threadIdx.x; e < NE; e += NT) dst[base + e] = tile[(e / N) * P + e % N];
    }
    op.end(reinterpret_cast<double*>(tile), blockIdx.x + (size_t)blockIdx.y * gridDim.x);
}


// ---------------------------------------------------------------------------
// Plane pass of a mid segment for 128^2 complex64 planes, with the z-transform
// pair around the pointwise step held in registers.
//
// The inverse transform runs y then z, the forward one z then y; both are
// radix 16 x 8 per axis (Stockham, autosorting).  The inverse z-transform ends
// with its radix-8 stage and the forward one starts with radix 8 (reversed
// radix order), so one thread holds the outputs i + 16t (t < 8) of butterfly i
// of a z-row, applies the pointwise op to them and runs the first forward
// butterfly on the same registers: no shared-memory round trip for the
// pointwise step, and none between the two z-transforms.  For those two
// stages the 16 butterflies of a row go to 16 consecutive threads, so a
// half-warp touches 16 consecutive z (128 bytes) of one row in global memory
// (the op's loads and stores are coalesced).  The forward stage writes
// positions 8i + t, a stride of 8 complex values; the tile's z index is
// swizzled, z ^ ((z >> 4) & 7), which keeps every half-warp access of every
// stage on 16 distinct 8-byte bank slots (rows are padded to ZREG_P values).
// Every z stage works on rows that one warp owns, so the z phase needs no
// block-wide barrier.
//
// Shared-memory round trips: 6 (y: 2, z: 2, z: 2 less the fused pair, y: 2
// less the register-resident first and last stages); block barriers: 7.
// Same grid, Op interface (forward ops: one load per point) and results, up
// to the rounding of the operation order, as k_plane_fused.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int plane_swz(int z) { return z ^ ((z >> 4) & 7); }

// Row pitch of the k_plane_zreg tile: 136 values (272 banks = 16 mod 32), so
// the two rows of a half-warp in the warp-owned z stages fall on opposite
// halves of the banks; accesses along y keep one row per half-warp.
constexpr int ZREG_P = 136;

// Global loads per point of a pointwise op (Op::LOADS where declared, else 4).
template <class Op, class = void>
struct op_loads {
    static constexpr int value = 4;
};
template <class Op>
struct op_loads<Op, std::void_t<decltype(Op::LOADS)>> {
    static constexpr int value = Op::LOADS;
};

// Twiddles of butterfly k of a stage with twiddle step 1 (N / (R * SPAN) = 1),
// then the radix-R DFT.
template <int S, int R, typename V>
__device__ __forceinline__ void bfly_k(V (&u)[R], int k, const V* __restrict__ tw)
{
    if (k) {
#pragma unroll
        for (int t = 1; t < R; ++t) u[t] = cmul(u[t], twiddle<S>(tw, t * k));
    }
    dftR<S, R>(u);
}

template <typename T, int S1, int S2, class Op>
__global__ void __launch_bounds__(1024, 1) k_plane_zreg(const cplx<T>* src, cplx<T>* dst, size_t fstride,
                                                        const cplx<T>* __restrict__ twn, Op op)
{
    using V = cplx<T>;
    constexpr int N = 128, P = ZREG_P, NE = N * N;
    static_assert(S1 != 0 && S2 != 0, "both transforms");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tile = reinterpret_cast<V*>(smem_raw);
    V* stw = tile + N * P;
    // twiddles w^(t i) of the register-resident z stage laid out [t][i]
    // (t < 8, i < 16): its 16 consecutive threads take 16 consecutive
    // entries, where the plain table would serve them with bank conflicts
    V* stz = stw + N;
    // twiddles w^(t b) of the warp-owned radix-16 z stage laid out [t][b]
    // (t < 16, b < 8): the 8 butterflies of a row read consecutive entries
    V* stb = stz + 128;
    const int tid = threadIdx.x;
    const int x = blockIdx.x;
    const int f = blockIdx.y;
    const size_t base = (size_t)f * fstride + (size_t)x * NE;
    for (int j = tid; j < N; j += 1024) stw[j] = twn[j];
    if (tid < 128) stz[tid] = twn[(tid >> 4) * (tid & 15)];
    else if (tid < 256) stb[tid - 128] = twn[((tid - 128) >> 3) * (tid & 7)];
    if (tid == 0) op.prefetch(base, (unsigned)NE);   // L2 prefetch: cannot observe a stale value
    pdl_wait();
    op.preload();
    const int zc = tid & 127;   // column of the y-stages
    const int hi = tid >> 7;    // 0..7
    // inverse y, stage 0 (radix 16, span 1): the coalesced load of column zc,
    // rows hi + 8t, is the input set of butterfly hi
    {
        V u[16];
#pragma unroll
        for (int t = 0; t < 16; ++t) u[t] = src[base + tid + t * 1024];
        __syncthreads();   // twiddles
        dftR<S1, 16>(u);
#pragma unroll
        for (int t = 0; t < 16; ++t) tile[(16 * hi + t) * P + plane_swz(zc)] = u[t];
        __syncthreads();
    }
    // inverse y, stage 1 (radix 8, span 16): butterflies hi and hi + 8 of column zc
    {
        V u[2][8];
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int t = 0; t < 8; ++t) u[q][t] = tile[(hi + 8 * q + 16 * t) * P + plane_swz(zc)];
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            bfly_k<S1, 8>(u[q], hi + 8 * q, stw);
#pragma unroll
            for (int t = 0; t < 8; ++t) tile[(hi + 8 * q + 16 * t) * P + plane_swz(zc)] = u[q][t];
        }
        __syncthreads();
    }
    // The z stages run on rows owned by one warp (rows 4w .. 4w+3 of warp
    // w), so they synchronise with __syncwarp only: the warps drift apart
    // there, and one warp's global loads of the pointwise step overlap the
    // transforms and shared-memory exchanges of the others.
    // inverse z, stage 0 (radix 16, span 1): row 4w + lane / 8, butterfly lane % 8
    {
        const int y = 4 * (threadIdx.x >> 5) + ((threadIdx.x & 31) >> 3), b = threadIdx.x & 7;
        V u[16];
#pragma unroll
        for (int t = 0; t < 16; ++t) u[t] = tile[y * P + plane_swz(b + 8 * t)];
        __syncwarp();
        dftR<S1, 16>(u);
#pragma unroll
        for (int t = 0; t < 16; ++t) tile[y * P + plane_swz(16 * b + t)] = u[t];
        __syncwarp();
    }
    // inverse z, stage 1 (radix 8, span 16) -> op -> forward z, stage 0
    // (radix 8, span 1): butterfly i = lane % 16 of rows 4w + (lane / 16) + 2q.
    // The op's loads depend on neither transform: those of row y0 are issued
    // before the block reduction of begin() and those of row y0 + 2 right after
    // the op of row y0, so their latency overlaps the barriers and the
    // transforms.  Each row is read, transformed, passed through the op and
    // written back in turn; per value the operations and their order are
    // those of the two-row form.
    const int i = threadIdx.x & 15;
    const int y0 = 4 * (threadIdx.x >> 5) + ((threadIdx.x >> 4) & 1);   // rows y0 and y0 + 2
    typename Op::Pre pre0[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) pre0[t] = op.load(f, base + (size_t)y0 * N + i + 16 * t);
    op.begin();
    {
        typename Op::Pre pre1[8];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int y = y0 + 2 * q;
            V u[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) u[t] = tile[y * P + plane_swz(i + 16 * t)];
            __syncwarp();   // the row's reads done before its positions are rewritten
            if (i) {
#pragma unroll
                for (int t = 1; t < 8; ++t) {
                    V w = stz[t * 16 + i];
                    if (S1 > 0) w.y = -w.y;
                    u[t] = cmul(u[t], w);
                }
            }
            dftR<S1, 8>(u);
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const int z = i + 16 * t;
                u[t] = op.apply(f, x, y, z, base + (size_t)y * N + z, u[t], q == 0 ? pre0[t] : pre1[t]);
            }
            if (q == 0) {
#pragma unroll
                for (int t = 0; t < 8; ++t) pre1[t] = op.load(f, base + (size_t)(y0 + 2) * N + i + 16 * t);
            }
            if (q == 1) pdl_trigger();
            dftR<S2, 8>(u);
#pragma unroll
            for (int t = 0; t < 8; ++t) tile[y * P + plane_swz(8 * i + t)] = u[t];
        }
        __syncwarp();
    }
    // forward z, stage 1 (radix 16, span 8): row 4w + lane / 8, butterfly lane % 8
    {
        const int y = 4 * (threadIdx.x >> 5) + ((threadIdx.x & 31) >> 3), b = threadIdx.x & 7;
        V u[16];
#pragma unroll
        for (int t = 0; t < 16; ++t) u[t] = tile[y * P + plane_swz(b + 8 * t)];
        __syncwarp();
        if (b) {
#pragma unroll
            for (int t = 1; t < 16; ++t) u[t] = cmul(u[t], twiddle<S2>(stb, t * 8 + b));
        }
        dftR<S2, 16>(u);
#pragma unroll
        for (int t = 0; t < 16; ++t) tile[y * P + plane_swz(b + 8 * t)] = u[t];
        __syncthreads();
    }
    // forward y, stage 0 (radix 16, span 1): column zc, butterfly hi
    {
        V u[16];
#pragma unroll
        for (int t = 0; t < 16; ++t) u[t] = tile[(hi + 8 * t) * P + plane_swz(zc)];
        __syncthreads();
        dftR<S2, 16>(u);
#pragma unroll
        for (int t = 0; t < 16; ++t) tile[(16 * hi + t) * P + plane_swz(zc)] = u[t];
        __syncthreads();
    }
    // forward y, stage 1 (radix 8, span 16): butterflies hi and hi + 8 of
    // column zc, stored straight to global memory (consecutive z per warp)
    {
        V u[2][8];
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int t = 0; t < 8; ++t) u[q][t] = tile[(hi + 8 * q + 16 * t) * P + plane_swz(zc)];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            bfly_k<S2, 8>(u[q], hi + 8 * q, stw);
#pragma unroll
            for (int t = 0; t < 8; ++t) dst[base + (size_t)(hi + 8 * q + 16 * t) * N + zc] = u[q][t];
        }
    }
    op.end(reinterpret_cast<double*>(tile), blockIdx.x + (size_t)blockIdx.y * gridDim.x);
}

}  // namespace ftsp
