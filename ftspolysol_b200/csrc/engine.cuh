// B200 complex-Langevin engine: device state, FFT executor, chain
// propagators, densities, Langevin update and observables.  Included by
// engine_f32.cu and engine_f64.cu (one instantiation each, compiled in
// parallel) and by abi.cu (the C ABI; no instantiation).
//
// One Engine<T> per system; T = double (FP64, reference-equivalent) or
// float (complex64 fields and propagators, FP64 reductions).  All device
// work of a handle is queued on one stream; a step needs no host
// synchronisation except the final status read in ftsp_step.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <stdexcept>
#include <string>
#include <vector>

#include "passes.cuh"
#include "chain_pairs.cuh"
#include "learned.cuh"
#include "ftsp.h"

namespace ftsp {

constexpr int MAXSP = 16;
constexpr int MAXION = 16;
constexpr int MAXM = 8;
constexpr int MAXMODE = 8;
constexpr int RED_BLOCKS = 1184;  // largest reduction grid (8 x 148 SMs); a kernel's grid is fixed per device => deterministic sums
constexpr int RED_THREADS = 256;
constexpr double PI = 3.141592653589793238462643383279502884;

struct CudaError : std::runtime_error {
    explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};

#define FTSP_CUDA(call)                                                                       \
    do {                                                                                      \
        cudaError_t err_ = (call);                                                            \
        if (err_ != cudaSuccess)                                                              \
            throw CudaError(std::string(#call) + ": " + cudaGetErrorString(err_));            \
    } while (0)

// ---- device scalars shared by the kernels of one step ----
struct DevScal {
    // every member is 16-byte aligned: several are read or written as double2
    alignas(16) double2 Q[MAXSP];
    alignas(16) double2 factor[MAXSP];
    alignas(16) double2 Qion[MAXION];
    alignas(16) double2 ion_factor[MAXION];
    alignas(16) double2 mean_dpsi;
    alignas(16) double2 mean_psi;
    alignas(16) double mean_eta;
    alignas(16) double corr[4];            // corrector: sum of psi (complex), non-finite cell count
    alignas(16) double fsq[2 * MAXMODE];   // sum over the grid of omega_a^2 (complex)
    alignas(16) double kobs[26];           // k-space observable sums
    alignas(16) double sconn[12];          // connectivity stress sums over the bond-pass CTAs
    alignas(16) double dmax[MAXMODE + 1];
    alignas(16) double rec[2 * 128];
    alignas(16) unsigned long long step;   // steps taken: keys the noise, schedules the checkpoints
    long long avg_seen;                    // time averaging: steps since ftsp_average_start
    long long avg_count;                   // of those, records accumulated (committed + pending)
    long long avg_committed;               // records in the blocks (past a checkpoint)
    alignas(16) double dt_scale;           // this step's dt / configured dt (1 unless the step is adaptive)
    double umax;                           // max |drift| at the start of this step (adaptive step)
    alignas(16) double lres[2];            // learned preconditioner: force residuals (learned, analytic) of the step
    alignas(16) double lres_sum[2];        // and their sums since the last statistics reset
    alignas(16) int nonfinite;
    int bad_last;                          // the last step produced a non-finite value
    int restarts;                          // checkpoint rollbacks so far
    int exhausted;                         // a non-finite step found max_restarts rollbacks taken: final
    int lr_use;                            // the next step preconditions with the learned G(k)
    int lr_checks;                         // steps judged by the residual test
    int lr_fallbacks;                      // of those, steps that fell back to the analytic G(k)
};
static_assert(offsetof(DevScal, rec) % 16 == 0 && offsetof(DevScal, corr) % 16 == 0, "DevScal alignment");

// ---- host configuration ----
struct Cls {
    int type;
    double z;
};

struct Species {
    double nc;
    int N;
    std::vector<int> type;
    std::vector<double> charge, bond;
    std::vector<int> cls;     // class of each segment
    std::vector<int> bcls;    // bond-length class of each bond
};

struct Ion {
    double z, count, smear;
};

struct HostCfg {
    int m1, m2, m3;
    size_t V;
    double L[3];
    double dV, a, lB, dt, lpsi, volume;
    bool elec;
    int M, nm;
    std::vector<double> coeff, lambda, O;
    std::vector<double2> gamma;
    std::vector<Species> sp;
    std::vector<Ion> ions;
    std::vector<Cls> cls;
    std::vector<double> bond_lengths;
    double self_pressure;
    int stress_mask, iso;
    bool noise;
    uint64_t seed;
    int precision, scheme, device;
    int restart_interval;   // device checkpoint every so many steps; rollback on a non-finite step (0: off)
    int max_restarts;       // rollbacks before a non-finite step is final (the reference's max_nan_restarts)
    int autotune;           // time the launch-geometry alternatives at creation
    int n_stress() const { return __builtin_popcount(stress_mask); }
    bool stress_on() const { return stress_mask != 0 || iso; }
    int record_len() const
    {
        const int S = (int)sp.size(), J = (int)ions.size();
        return 3 * (S + J) + 1 + n_stress() + (iso ? 1 : 0);
    }
};

// Radix plan: the power-of-two part in as few stages of radix <= 16 as
// possible, spread evenly (128 = 16 x 8, 64 = 8 x 8, 32 = 8 x 4), then the
// factors 3 and 5.
// max_bits: largest power-of-two radix as a bit count (4: radix 16 for
// complex64, 3: radix 8 for complex128, whose line passes hold 8 values per
// thread).
static FftPlan1 make_plan(int n, int max_bits)
{
    FftPlan1 p{};
    p.n = n;
    p.nst = 0;
    int r = n, p2 = 0;
    while (r % 2 == 0) {
        r /= 2;
        ++p2;
    }
    const int nst2 = (p2 + max_bits - 1) / max_bits;
    int left = p2;
    for (int st = 0; st < nst2; ++st) {
        const int bits = (left + (nst2 - st) - 1) / (nst2 - st);   // ceil(bits left / stages left)
        p.rad[p.nst++] = 1 << bits;
        left -= bits;
    }
    while (r % 3 == 0 && p.nst < 8) { p.rad[p.nst++] = 3; r /= 3; }
    while (r % 5 == 0 && p.nst < 8) { p.rad[p.nst++] = 5; r /= 5; }
    if (r != 1) throw std::runtime_error("grid size " + std::to_string(n) + " is not 2/3/5-smooth or needs more than 8 stages");
    int span = 1;
    for (int st = 0; st < p.nst; ++st) {
        p.span[st] = span;
        p.fspan[st] = make_fastdiv((unsigned)span);
        p.tstep[st] = n / (p.rad[st] * span);
        span *= p.rad[st];
    }
    return p;
}

static double wave_number(int i, int m, double L)
{
    const int mode = i > m / 2 ? i - m : i;
    return 2.0 * PI * mode / L;
}

// ---------------------------------------------------------------------------
// Generic kernels
// ---------------------------------------------------------------------------
template <class F>
__global__ void k_foreach(size_t n, F f)
{
    pdl_wait();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) f(i);
    pdl_trigger();
}

// Sum (MAX = false) or maximum (MAX = true) of K channels; partial[block*K + c].
template <int K, bool MAX, class F>
__global__ void __launch_bounds__(RED_THREADS) k_reduce(size_t n, F f, double* partial)
{
    __shared__ double scratch[(RED_THREADS / 32) * K];
    double acc[K];
#pragma unroll
    for (int c = 0; c < K; ++c) acc[c] = 0.0;
    pdl_wait();
    // items i, i + stride, ... in that order; U at a time, so that the loads
    // of U items are in flight together where f's loads cannot alias its
    // stores (read-only loads); the per-thread summation order is unchanged
    constexpr int U = K <= 6 ? 4 : 1;   // many channels: registers for occupancy instead
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + (U - 1) * stride < n; i += U * stride) {
#pragma unroll
        for (int u = 0; u < U; ++u) f(i + u * stride, acc);
    }
    for (; i < n; i += stride) f(i, acc);
    pdl_trigger();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < K; ++c) {
        double x = acc[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, x, o);
            x = MAX ? fmax(x, y) : x + y;
        }
        if (lane == 0) scratch[warp * K + c] = x;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int w = 0; w < RED_THREADS / 32; ++w) {
            const double y = scratch[w * K + threadIdx.x];
            s = MAX ? fmax(s, y) : s + y;
        }
        partial[blockIdx.x * K + threadIdx.x] = s;
    }
}

// Fixed-order combine of `count` partial rows of K channels: one warp per
// channel (grid K), lanes stride over the rows, then a shuffle tree.
// Time averaging of the observable record (complexLangevin.cu:424-441): a
// step's record is taken when more than `skip` steps have been seen since
// the averaging started, fewer than `samples` records have been taken and
// the step is finite; the real part of every entry, weighted by the step's
// dt scale (1 unless the step is adaptive).  Records first go to a pending
// accumulator (acc + nblk * (R + 2)); the pending records are committed to
// block avg_committed / per_block when the step is a checkpoint (every
// `every` steps, or every step without rollback) and discarded by a
// rollback, which restores the checkpoint (restore_if_bad), so the averages
// hold exactly the records of the trajectory that was kept, as the
// reference rewrites its observable file after a restart
// (complexLangevin.cu:638-656).  Per block: R weighted sums, the weight sum
// and the record count.  One CTA; the counters move after every thread has
// read them.
static __global__ void k_average(DevScal* d, double* acc, int R, int nblk, long long skip, long long samples,
                                 long long per_block, unsigned long long every)
{
    double* pend = acc + (size_t)nblk * (R + 2);
    const bool take = d->avg_seen + 1 > skip && d->avg_count < samples && !d->bad_last;
    if (take) {
        const double w = d->dt_scale;
        for (int i = threadIdx.x; i < R; i += blockDim.x) pend[i] += w * d->rec[2 * i];
        if (threadIdx.x == 0) {
            pend[R] += w;
            pend[R + 1] += 1.0;
        }
    }
    __syncthreads();
    const bool commit = !d->bad_last && (every == 0 || d->step % every == 0);
    const double pn = pend[R + 1];
    if (commit && pn > 0.0) {
        const long long b = d->avg_committed / per_block;
        double* a = acc + (size_t)(b < nblk ? b : nblk - 1) * (R + 2);
        for (int i = threadIdx.x; i < R + 2; i += blockDim.x) {
            a[i] += pend[i];
            pend[i] = 0.0;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        d->avg_seen += 1;
        if (take) d->avg_count += 1;
        if (commit && pn > 0.0) d->avg_committed += (long long)pn;
    }
}

// Any block size that is a multiple of 32 (up to 1024): threads stride over
// the rows, a shuffle tree per warp, then warp 0 combines the warps in order;
// the summation order depends only on count and the block size.
constexpr int COMBINE_THREADS = 256;
template <bool MAX>
__global__ void k_combine(const double* partial, int count, int K, double* out)
{
    __shared__ double ws[32];
    const int c = blockIdx.x;
    double s = 0.0;
    pdl_wait();
    for (int b = threadIdx.x; b < count; b += blockDim.x) {
        const double y = partial[(size_t)b * K + c];
        s = MAX ? fmax(s, y) : s + y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double y = __shfl_xor_sync(0xffffffffu, s, o);
        s = MAX ? fmax(s, y) : s + y;
    }
    const int nw = blockDim.x >> 5;
    if (nw == 1) {
        if (threadIdx.x == 0) out[c] = s;
        return;
    }
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < nw ? ws[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, s, o);
            s = MAX ? fmax(s, y) : s + y;
        }
        if (threadIdx.x == 0) out[c] = s;
    }
}

// ---- small complex helpers in double ----
__device__ __forceinline__ double2 dmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 dadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 dscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 dinv(double2 z)  // Smith's algorithm, as common.h:146-157
{
    const double ax = fabs(z.x), ay = fabs(z.y);
    if (ax >= ay) {
        const double r = z.y / z.x, den = z.x * (1.0 + r * r);
        return make_double2(1.0 / den, -r / den);
    }
    const double r = z.x / z.y, den = z.y * (1.0 + r * r);
    return make_double2(r / den, -1.0 / den);
}
__device__ __forceinline__ double2 dneglog(double2 z)
{
    return make_double2(-log(sqrt(z.x * z.x + z.y * z.y)), -atan2(z.y, z.x));
}
template <typename V> __device__ __forceinline__ double2 to_d(V v) { return make_double2((double)v.x, (double)v.y); }
template <typename V> __device__ __forceinline__ V from_d(double2 d)
{
    V v;
    v.x = (typename RealOf<V>::type)d.x;
    v.y = (typename RealOf<V>::type)d.y;
    return v;
}
// exp of a complex number as common.h:188-192: r = exp(x); (r cos y, r sin y)
__device__ __forceinline__ float2 cexpT(float x, float y)
{
    const float r = expf(x);
    float s, c;
    sincosf(y, &s, &c);
    return make_float2(r * c, r * s);
}
__device__ __forceinline__ double2 cexpT(double x, double y)
{
    const double r = exp(x);
    double s, c;
    sincos(y, &s, &c);
    return make_double2(r * c, r * s);
}

// ---- Philox4x32-10 counter-based generator (Salmon et al., SC'11) ----
struct U4 {
    uint32_t x, y, z, w;
};
__device__ __forceinline__ U4 philox(U4 c, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    }
    return c;
}
// Two independent standard normals per (element, field pair, step): the
// Box-Muller transform of two 53-bit uniforms in (0, 1), both of its outputs
// (r cos 2 pi u2 for field 2p, r sin 2 pi u2 for field 2p + 1).
__device__ __forceinline__ void normal_pair_at(uint64_t seed, uint64_t step, uint32_t pair, uint64_t i, double& n0,
                                               double& n1)
{
    const U4 r = philox(U4{(uint32_t)i, (uint32_t)(i >> 32), (uint32_t)step, pair}, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double u1 = ((double)(((uint64_t)r.x << 21) ^ (r.y >> 11)) + 0.5) * (1.0 / 9007199254740992.0);
    const double u2 = ((double)(((uint64_t)r.z << 21) ^ (r.w >> 11)) + 0.5) * (1.0 / 9007199254740992.0);
    const double rad = sqrt(-2.0 * log(u1));
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    n0 = rad * cs;
    n1 = rad * sn;
}

// ---- plain-data tables captured by the kernels' lambdas ----
struct GCoef {
    double2 g[MAXMODE * MAXM];   // gamma_a O_{a alpha}
};
struct ModeTab {
    double c[MAXMODE];
    double s[MAXMODE];
    double2 g[MAXMODE * MAXM];
};
struct SigTab {
    double s[MAXMODE + 1];
};

// a[i] for a run-time i < K with constant indices only: an array in a
// kernel's parameter block indexed at run time is copied to local memory
// by every thread
template <typename U, int K>
__device__ __forceinline__ U pick(const U (&a)[K], int i)
{
    U v = a[0];
#pragma unroll
    for (int k = 1; k < K; ++k)
        if (i == k) v = a[k];
    return v;
}
struct SiOTab {
    double O[MAXMODE * MAXM];
};
struct ClsTab {
    int type[64];
    double z[64];
};
struct IonTab {
    double z[MAXION];
    double nd[MAXION];
    double a2[MAXION];
};
struct ObsConst {
    double2 g[MAXMODE * MAXM];
    double z[MAXION];
    double a2ion[MAXION];
};
struct RecConst {
    double nv[MAXSP];
    double self_poly[MAXSP];
    double ideal_poly[MAXSP];
    double nvion[MAXION];
    double self_ion[MAXION];
    double ideal_ion[MAXION];
    double coeff[MAXMODE];
    double ideal_stress[6];   // (ideal + self) delta + mode term
    double ideal_iso;
    int active[6];
};

// Loaders used by the plain transforms: field f of a batch reads src[f].
template <typename T>
struct OpLoadN {
    const cplx<T>* s[16];
    size_t fs;
    struct Pre {
        cplx<T> v;
    };
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ Pre load(int f, size_t g) const { return Pre{s[f][g - f * fs]}; }
    __device__ __forceinline__ cplx<T> apply(int, int, int, int, size_t, cplx<T>, const Pre& p) const { return p.v; }
    __device__ __forceinline__ void end(double*, size_t) {}
};
template <typename T>
struct OpLoadOne {
    const cplx<T>* s;
    struct Pre {
        cplx<T> v;
    };
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ Pre load(int, size_t g) const { return Pre{s[g]}; }
    __device__ __forceinline__ cplx<T> apply(int, int, int, int, size_t, cplx<T>, const Pre& p) const { return p.v; }
    __device__ __forceinline__ void end(double*, size_t) {}
};

// Semi-implicit preconditioner in the x-pencil pass between the forward and
// inverse x transforms: k = v / (1 + dt_f dt_scale lambda_f G_f(k)), the
// learned table while the residual test allows it, optionally stashed, then
// scaled by 1/V for the unnormalised inverse.
template <typename T>
struct OpPrecond {
    const T* GA;             // analytic G_f(k), field-major
    const T* GL;             // learned G_f(k) (null: not in use)
    cplx<T>* dw;             // stash of the k-space increments (null: off)
    const DevScal* d;
    SigTab st;               // dt lambda_f per field
    T invV;
    int dc0 = -1;            // field whose k = 0 value is set to zero (psi: its mean removal), -1: none
    static constexpr int FUSED_MIN_BLOCKS = 8;
    struct Pre {};
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ Pre load(int, size_t) const { return Pre{}; }
    __device__ __forceinline__ cplx<T> apply(int f, int x, int y, int z, size_t g, cplx<T> v, const Pre&) const
    {
        const T G = (GL && d->lr_use) ? GL[g] : GA[g];
        const cplx<T> k = cscale(v, (T)(1.0 / (1.0 + (pick(st.s, f) * d->dt_scale) * (double)G)));
        if (dw) dw[g] = k;
        if (f == dc0 && (x | y | z) == 0) return mkc<cplx<T>>(T(0), T(0));
        return cscale(k, invV);
    }
    __device__ __forceinline__ void end(double*, size_t) {}
};

// k-space factors of the density evaluation, applied in the x-pencil pass
// between the forward and inverse x transforms (the y and z transforms run
// in the plane passes on either side): output field f is the transform of
// source field src[f] times c_f F_f(k), F_f the smearing Gamma(k) (lap_f = 0)
// or k^2 (lap_f = 1), c_f including the 1/V of the unnormalised inverse; the
// k-space values of the fields f < nst (whose source is f itself) are
// written to kst, the Fourier fields that the k-space observables read.
template <typename T>
struct OpKScale {
    using V = cplx<T>;
    static constexpr int NSRC = 4;
    static constexpr int FUSED_MIN_BLOCKS = 8;
    V* kst;
    const T* gm;             // Gamma per axis: x, then y, then z
    const double* kx;
    const double* ky;
    const double* kz;
    int m1, m2;
    int nst;
    int src[NSRC];
    int lap[NSRC];
    double2 c[NSRC];
    struct Pre {};
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ Pre load(int, size_t) const { return Pre{}; }
    __device__ __forceinline__ V apply(int f, int x, int y, int z, size_t g, V v, const Pre&) const
    {
        if (f < nst) kst[g] = v;
        double fac;
        if (pick(lap, f)) {
            const double ax = __ldg(kx + x), ay = __ldg(ky + y), az = __ldg(kz + z);
            fac = ax * ax + ay * ay + az * az;
        } else {
            fac = (double)(__ldg(gm + x) * __ldg(gm + m1 + y) * __ldg(gm + m1 + m2 + z));
        }
        return from_d<V>(dscale(dmul(to_d(v), pick(c, f)), fac));
    }
    __device__ __forceinline__ void end(double*, size_t) {}
};

// Loads of the fused density transform (one monomer type): field 0 the
// monomer density, field 1 the polymer charge density plus zf times the
// monomer density (the charge of a uniformly charged species, accumulated
// once here instead of per segment), field 2 the combined ion charge.
template <typename T>
struct OpLoadDensity {
    using V = cplx<T>;
    const V* rho;            // monomer density, charge density, ion charge
    size_t Vn;
    double zf;               // 0: no folded charge
    struct Pre {
        V v;
    };
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ Pre load(int f, size_t g) const
    {
        const size_t i = g - (size_t)f * Vn;
        V a = rho[(size_t)f * Vn + i];
        if (f == 1 && zf != 0.0) a = cadd(a, cscale(rho[i], (T)zf));
        return Pre{a};
    }
    __device__ __forceinline__ V apply(int, int, int, int, size_t, V, const Pre& p) const { return p.v; }
    __device__ __forceinline__ void end(double*, size_t) {}
};

// The increments of the semi-implicit update, computed as the field loads of
// its first transform pass (the load of field f at point g; f < nm the
// interaction modes, f = nm psi):
//   predictor: dt_scale c_f u_f + eta_f, psi: its noise and drift with their
//              means removed first (written back: the corrector reads them);
//   corrector: dt_scale c_f (u_f + u_bar_f) + eta_f, psi: the predictor drift
//              plus the mean-removed u_bar (written back); and the largest
//              |u + u_bar|^2 of the CTA's points, per field, into dpart
//              (the drift maxima, complexLangevin.cu:474-498).
// c_f = -dt lambda_f (predictor), -dt lambda_f / 2 (corrector).
template <typename T, bool CORR>
struct OpIncrement {
    using V = cplx<T>;
    const V* u0;             // drift at (omega, psi)
    const V* u1;             // drift at (omega_bar, psi_bar) (corrector)
    T* e;                    // noise, nm + 1 real fields
    V* dp;                   // psi drift at (omega, psi)
    V* db;                   // psi drift at (omega_bar, psi_bar) (corrector)
    const DevScal* d;
    SigTab cs;               // c_f of the modes, then of psi
    double invV;
    size_t Vn;
    int nm;
    bool elec;
    double* dpart;           // corrector: per-CTA drift maxima
    double dmax;
    // the raw operands of a point; the loads carry no side effect, so a
    // kernel keeps a whole batch of them in flight, and apply() does the
    // arithmetic and the write-backs
    struct Pre {
        V a, b;              // modes: u, u_bar; psi: psi drift, psi drift at the predictor
        T e;
    };
    __device__ __forceinline__ void begin() { dmax = 0.0; }
    __device__ __forceinline__ Pre load(int f, size_t g) const
    {
        const size_t i = g - (size_t)f * Vn;
        Pre p;
        if (f < nm) {
            const size_t j = (size_t)f * Vn + i;
            p.a = u0[j];
            if (CORR) p.b = u1[j];
            p.e = e[j];
        } else if (elec) {
            p.a = dp[i];
            if (CORR) p.b = db[i];
            p.e = e[(size_t)nm * Vn + i];
        }
        return p;
    }
    __device__ __forceinline__ V apply(int f, int, int, int, size_t g, V, const Pre& p)
    {
        const size_t i = g - (size_t)f * Vn;
        if (f < nm) {
            V s = p.a;
            if (CORR) {
                s = cadd(s, p.b);
                double m = (double)s.x * s.x + (double)s.y * s.y;
                if (!isfinite(m)) m = INFINITY;
                dmax = fmax(dmax, m);
            }
            V v = cscale(s, (T)(pick(cs.s, f) * d->dt_scale));
            v.x += p.e;
            return v;
        }
        if (!elec) return mkc<V>(T(0), T(0));
        T ep = p.e;
        // mean_dpsi: the sum of the psi drift of the last density evaluation
        // (at omega, psi for the predictor; at the predictor's fields for the
        // corrector); the mean-removed values are written back, the corrector
        // and the caller read them
        V s;
        if (!CORR) {
            ep = (T)((double)ep + (-(d->mean_eta * invV)));
            e[(size_t)nm * Vn + i] = ep;
            s = cadd(p.a, from_d<V>(dscale(d->mean_dpsi, -invV)));
            dp[i] = s;
        } else {
            const V dbv = cadd(p.b, from_d<V>(dscale(d->mean_dpsi, -invV)));
            db[i] = dbv;
            s = cadd(p.a, dbv);
            double m = (double)s.x * s.x + (double)s.y * s.y;
            if (!isfinite(m)) m = INFINITY;
            dmax = fmax(dmax, m);
        }
        V v = cscale(s, (T)(pick(cs.s, nm) * d->dt_scale));
        v.x += ep;
        return v;
    }
    __device__ __forceinline__ void end(double* scratch, size_t cta)
    {
        if (!CORR) return;
        __syncthreads();
        double m = dmax;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            double r = 0.0;
            for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) r = fmax(r, scratch[w]);
            dpart[cta] = r;
        }
    }
};

// The last pass of the semi-implicit update: field f = base f + increment
// (predictor: omega_bar, psi_bar from omega, psi; corrector: omega, psi in
// place), and the count of non-finite cells per CTA into npart.
template <typename T>
struct OpUpdate {
    using V = cplx<T>;
    const V* w0;             // modes before the update
    const V* p0;             // psi before the update
    V* w1;                   // modes after
    V* p1;                   // psi after
    size_t Vn;
    int nm;
    bool elec;
    double* npart;           // per-CTA non-finite counts (null: not counted)
    double bad;
    struct Pre {
        V b;
    };
    __device__ __forceinline__ void begin() { bad = 0.0; }
    __device__ __forceinline__ Pre load(int f, size_t g) const
    {
        const size_t i = g - (size_t)f * Vn;
        if (f < nm) return Pre{w0[(size_t)f * Vn + i]};
        return Pre{elec ? p0[i] : mkc<V>(T(0), T(0))};
    }
    __device__ __forceinline__ V apply(int f, int, int, int, size_t g, V v, const Pre& p)
    {
        const size_t i = g - (size_t)f * Vn;
        const V r = (f < nm || elec) ? cadd(p.b, v) : mkc<V>(T(0), T(0));
        if (f < nm) w1[(size_t)f * Vn + i] = r;
        else p1[i] = r;
        if (!(isfinite((double)r.x) && isfinite((double)r.y))) bad += 1.0;
        return r;
    }
    __device__ __forceinline__ void end(double* scratch, size_t cta)
    {
        if (!npart) return;
        double v[1] = {bad};
        __syncthreads();
        block_sum<1>(v, scratch);
        if (threadIdx.x == 0) npart[cta] = v[0];
    }
};

// Stores the pass's values (a pass with no second transform).
template <typename T>
struct OpStore {
    cplx<T>* out;
    struct Pre {};
    __device__ __forceinline__ void begin() {}
    __device__ __forceinline__ Pre load(int, size_t) const { return Pre{}; }
    __device__ __forceinline__ cplx<T> apply(int, int, int, int, size_t g, cplx<T> v, const Pre&) const
    {
        out[g] = v;
        return v;
    }
    __device__ __forceinline__ void end(double*, size_t) {}
};

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
struct ProfStat {
    double ms = 0.0;
    long long launches = 0;
    double bytes = 0.0;   // algorithmic bytes (minimum HBM traffic of the launch's work)
};

// Features of wave vector i for the learned preconditioner's network
// (learned.cuh): log(1 + k^2), log(1 + P_w), log(1 + P_psi), N / 50, lB,
// 10 c_salt.
struct LearnFeat {
    const double* kx;
    const double* ky;
    const double* kz;
    const float* Pw;
    const float* Pp;
    int m2, m3;
    float N, lB, salt;
    __device__ __forceinline__ bool operator()(size_t i, float* x) const
    {
        const size_t yz = (size_t)m2 * m3;
        const int ix = (int)(i / yz);
        const int r = (int)(i - (size_t)ix * yz);
        const int iy = r / m3, iz = r - iy * m3;
        const double k2 = kx[ix] * kx[ix] + ky[iy] * ky[iy] + kz[iz] * kz[iz];
        x[0] = (float)log1p(k2);
        x[1] = log1pf(fmaxf(Pw[i], 0.0f));
        x[2] = log1pf(fmaxf(Pp[i], 0.0f));
        x[3] = N / 50.0f;
        x[4] = lB;
        x[5] = 10.0f * salt;
        return true;
    }
};

struct EngineBase {
    HostCfg c;
    std::string err;
    cudaStream_t stream = nullptr;
    long long launches = 0;
    // per-kernel CUDA-event timing of the propagator passes (ftsp_profile_*)
    bool profiling = false;
    std::vector<std::pair<std::string, ProfStat>> prof;
    struct Pending {
        int slot;
        double bytes;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;

    int prof_slot(const std::string& name)
    {
        for (size_t i = 0; i < prof.size(); ++i)
            if (prof[i].first == name) return (int)i;
        prof.push_back({name, ProfStat{}});
        return (int)prof.size() - 1;
    }
    cudaEvent_t take_event()
    {
        if (pool.empty()) {
            cudaEvent_t e;
            FTSP_CUDA(cudaEventCreate(&e));
            return e;
        }
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    cudaEvent_t prof_begin()
    {
        if (!profiling) return nullptr;
        cudaEvent_t a = take_event();
        FTSP_CUDA(cudaEventRecord(a, stream));
        return a;
    }
    void prof_end(cudaEvent_t a, const std::string& name, double bytes)
    {
        if (!profiling || !a) return;
        cudaEvent_t b = take_event();
        FTSP_CUDA(cudaEventRecord(b, stream));
        pending.push_back(Pending{prof_slot(name), bytes, a, b});
    }
    void prof_collect()
    {
        if (pending.empty()) return;
        FTSP_CUDA(cudaStreamSynchronize(stream));
        for (auto& p : pending) {
            float ms = 0.0f;
            FTSP_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
            ProfStat& s = prof[p.slot].second;
            s.ms += ms;
            s.launches += 1;
            s.bytes += p.bytes;
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
    void prof_reset()
    {
        prof_collect();
        prof.clear();
    }
    virtual void release_events()
    {
        for (auto& p : pending) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        pending.clear();
        for (auto e : pool) cudaEventDestroy(e);
        pool.clear();
    }
    virtual ~EngineBase() {}
    virtual void set_fields(const double* omega, const double* psi) = 0;
    virtual void set_fields_async(const double* omega, const double* psi) = 0;
    virtual void install_pending_fields() = 0;
    virtual long long get_field(const std::string& name, double* out) = 0;
    virtual void compute_densities(int which, double* Q) = 0;
    virtual void measure(int which, double* rec) = 0;
    virtual void set_noise(const double* eta) = 0;
    virtual int step(double* Qbar, double* rec, double* dmax, bool sync) = 0;
    virtual int read_status(double* rec, double* dmax) = 0;
    virtual void views(ftsp_views* v) = 0;
    virtual void propagate_chain(const double2* w, int N, double bond, double2* q_end, double* Q) = 0;
    virtual long long restarts() = 0;
    virtual bool restarts_exhausted() = 0;
    virtual void average_start(long long skip, long long samples, int blocks) = 0;
    virtual long long average_read(double* mean, double* std_error) = 0;
    virtual void set_dt(double dt) = 0;
    virtual void set_adaptive(double u_ref) = 0;
    virtual void set_chain_symmetry(bool on) = 0;
    virtual int chain_symmetric_species() = 0;
    virtual void drop_step_graph() = 0;
    bool step_graph = true;   // replay a captured step in step() (see Engine::step)
    virtual void step_info(double* dt_eff, double* umax) = 0;
    virtual void tune_info(ftsp_tune_info* t) = 0;
    virtual void learn_configure(const ftsp_learn_config& cf) = 0;
    virtual void learn_collect(bool on) = 0;
    virtual void learn_reset() = 0;
    virtual double learn_train(int iterations) = 0;
    virtual void learn_use(bool on) = 0;
    virtual void learn_stats(ftsp_learn_stats* st) = 0;
    virtual int learn_weights(float* out, int n, bool set) = 0;
    virtual double learn_grad(const float* x, const float* t, const float* m, int n, float* grad) = 0;
};

template <typename T>
struct Buf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count)
    {
        n = count;
        if (count) FTSP_CUDA(cudaMalloc(&p, sizeof(T) * count));
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
    }
};

template <typename T>
struct Engine : EngineBase {
    using V = cplx<T>;
    size_t V_ = 0;
    bool plane_ok = false;
    PlaneGeom pg{};
    LineGeom gx{}, gy{}, gz{};
    int plane_threads = 0, x_threads = 0, y_threads = 0, z_threads = 0;
    size_t plane_smem = 0, x_smem = 0, y_smem = 0, z_smem = 0;
    static constexpr bool F32 = sizeof(T) == 4;
    static constexpr int EP = F32 ? 32 : 16;   // elements per thread, runtime-plan plane pass
    static constexpr int EL = F32 ? 16 : 8;    // elements per thread, runtime-plan line passes
    static constexpr int RMAX = F32 ? 16 : 8;  // largest radix of the compile-time transforms
    static constexpr int WCT = F32 ? 16 : 8;   // z-columns per tile of the compile-time strided passes (128-byte rows)
    Buf<FftPlan1> plans;                       // device-memory plans: x, y, z

    // device buffers
    Buf<V> tw1, tw2, tw3;
    Buf<double> kx, ky, kz;
    Buf<T> phi;          // per bond class: m1 + m2 + m3 separable factors
    Buf<T> gam;          // Gamma of the beads, separable (m1 + m2 + m3)
    Buf<T> gion;         // per ion: separable Gamma_j (m1 + m2 + m3)
    Buf<V> omega, psi, omega_bar, psi_bar, drift, drift_bar, dpsi, dpsi_bar;
    Buf<T> eta;          // (nm + 1) * V
    Buf<V> kA;           // (nm + 1) * V : DFT of (omega_w, psi_w)
    Buf<V> kB;           // (M + 1 + J) * V : W_type_s, psi_s, ion psi (real space)
    Buf<V> dB;           // (M + 1 + J) * V : density accumulators + ion Boltzmann -> k-space
    Buf<V> kC;           // (M + 3) * V : rho_type, rho_c_poly, rho_c_ion, psi-drift part
    Buf<V> rho_p, rho_c, ion_rho;
    Buf<V> E;            // class tables exp(-W_c)
    Buf<V> qF, Fst, G, H;
    Buf<double> part;    // reduction partials
    Buf<int> expo;       // propagator renormalisation exponents: forward [Nmax], backward [Nmax]
    Buf<T> si_G;         // semi-implicit linear-response coefficients G(k) (analytic): modes, then psi
    Buf<V> si_inc;       // semi-implicit increments (nm + 1 fields)
    Buf<V> ck;           // device checkpoint of (omega, psi) for rollback
    Buf<float> pmax;     // per-CTA propagator maxima, two slots (ping-pong by segment parity)
    Buf<double> spart;   // stress partials [ncta_x * 6] complex
    // mirror-symmetric species: pair tables of the density and stress kernels
    Buf<int2> pair_ix;
    Buf<double> pair_wt;
    Buf<PairRun> pair_run;
    struct SymTables {
        bool ok = false;
        PairTable dens{}, stress{};
        int dens_channels = 0;   // distinct density channels of the species
    };
    std::vector<SymTables> sym;
    bool chain_sym = true;       // use the pair kernels for mirror-symmetric species
    bool fused_strided = true;   // bond passes with register-resident middle stages (k_strided_fused)
    bool fused_plane = true;     // mid segment passes with register-resident end stages (k_plane_fused)
    bool zreg_plane = true;      // forward mid passes of 128^2 complex64 planes: z pair in registers (k_plane_zreg)
    // every ion smeared like the beads (and at most 3 ion species): the ion
    // potentials are psi_s itself, and the ion charge is one combined field
    // sum_j z_j (n_j/V)/Q_j exp(-i z_j psi_s), transformed once (see eval)
    bool ion_common = false;
    int qF_holds_u = -1;         // species whose u = q / E the qF buffer holds (-1: q)
    // a single mirror-symmetric species runs its stress kernel on a second
    // stream, overlapped with the rest of the density evaluation
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool aux_pending = false;
    DevScal* ds = nullptr;
    DevScal hs{};
    bool noise_injected = false;
    int Nmax = 1;

    explicit Engine(const HostCfg& cfg)
    {
        c = cfg;
        FTSP_CUDA(cudaSetDevice(c.device));
        V_ = c.V;
        setup_geometry();
        allocate();
        build_tables();
        plan_charge_fold();
        plan_symmetry();
        if (c.autotune) autotune();
    }

    ~Engine() override
    {
        drop_step_graph();
        if (cap_stream) cudaStreamDestroy(cap_stream);
        if (aux) cudaStreamDestroy(aux);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (cstream) {
            cudaStreamSynchronize(cstream);
            cudaStreamDestroy(cstream);
        }
        if (ev_staged) cudaEventDestroy(ev_staged);
        if (ev_installed) cudaEventDestroy(ev_installed);
        astage.release();
        Buf<V>* vb[] = {&tw1, &tw2, &tw3, &omega, &psi, &omega_bar, &psi_bar, &drift, &drift_bar, &dpsi, &dpsi_bar,
                        &kA, &kB, &dB, &kC, &rho_p, &rho_c, &ion_rho, &E, &qF, &Fst, &G, &H};
        for (auto* b : vb) b->release();
        plans.release();
        kx.release(); ky.release(); kz.release(); phi.release(); gam.release(); gion.release(); eta.release();
        part.release(); spart.release(); stage.release(); expo.release(); pmax.release();
        pair_ix.release(); pair_wt.release(); pair_run.release();
        si_G.release(); si_inc.release(); ck.release();
        avg.acc.release();
        upart.release();
        learn_release();
        if (ds) cudaFree(ds);
        release_events();
    }

    // ---- geometry and launch shapes ----
    static int round32(int t) { return std::max(32, (t + 31) / 32 * 32); }

    static int pick_W(int m3, int wmax)
    {
        int best = 1;
        for (int w = 1; w <= std::min(m3, wmax); ++w)
            if (m3 % w == 0) best = w;
        return best;
    }

    template <class K>
    void set_smem(K kernel, size_t bytes)
    {
        if (bytes > 48 * 1024) FTSP_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    }

    // Launch geometry of the runtime-plan passes.  max_bits: largest
    // power-of-two radix (as a bit count) of the FFT plans (0: the default,
    // 4 for complex64 and 3 for complex128); W: z-columns per tile of the
    // strided line passes (0: the largest divisor of m3 within the register
    // budget).  The autotuner times the alternatives (autotune()).
    int geo_max_bits = 0, geo_W = 0;
    static int default_max_bits() { return F32 ? 4 : 3; }
    int w_max() const { return std::max(1, std::min(sizeof(T) == 4 ? 32 : 16, (EL * 256) / std::max(c.m1, c.m2))); }

    void setup_geometry(int max_bits = 0, int Wsel = 0)
    {
        const int m1 = c.m1, m2 = c.m2, m3 = c.m3;
        int dev_smem = 0;
        FTSP_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device));
        pg.m1 = m1; pg.m2 = m2; pg.m3 = m3; pg.P = m3 + 1;
        if (max_bits <= 0) max_bits = default_max_bits();
        geo_max_bits = max_bits;
        const FftPlan1 hp[3] = {make_plan(m1, max_bits), make_plan(m2, max_bits), make_plan(m3, max_bits)};
        if (!plans.p) plans.alloc(3);
        FTSP_CUDA(cudaMemcpy(plans.p, hp, sizeof(hp), cudaMemcpyHostToDevice));
        pg.py = plans.p + 1;
        pg.pz = plans.p + 2;
        pg.fm2 = make_fastdiv(m2);
        pg.fm3 = make_fastdiv(m3);
        plane_smem = sizeof(V) * ((size_t)m2 * pg.P + m2 + m3);
        plane_smem = std::max(plane_smem, (size_t)32 * 16 * 8);
        plane_threads = round32((m2 * m3 + EP - 1) / EP);
        plane_ok = plane_smem <= (size_t)dev_smem && plane_threads <= 512;
        const int wmax = w_max();
        const int W = (Wsel > 0 && Wsel <= wmax && m3 % Wsel == 0) ? Wsel : pick_W(m3, wmax);
        geo_W = W;
        gx = LineGeom{m1, m2, m3, m1, W, 0, W, plans.p + 0, make_fastdiv(W), make_fastdiv(1), make_fastdiv(m2), make_fastdiv(m3)};
        gy = LineGeom{m1, m2, m3, m2, W, 0, W, plans.p + 1, make_fastdiv(W), make_fastdiv(1), make_fastdiv(m2), make_fastdiv(m3)};
        x_threads = round32((m1 * W + EL - 1) / EL);
        y_threads = round32((m2 * W + EL - 1) / EL);
        x_smem = std::max(sizeof(V) * ((size_t)m1 * W + m1), (size_t)32 * 16 * 8);
        y_smem = std::max(sizeof(V) * ((size_t)m2 * W + m2), (size_t)32 * 16 * 8);
        // z-lines: B rows with B*m3 ~ 2048 elements, B | m1*m2
        if (m3 > EL * 256) throw std::runtime_error("z extent too large for the line passes");
        int B = std::max(1, 2048 / m3);
        while ((m1 * m2) % B) --B;
        gz = LineGeom{m1, m2, m3, m3, 0, B, m3 + 1, plans.p + 2, make_fastdiv(1), make_fastdiv(B), make_fastdiv(m2), make_fastdiv(m3)};
        z_threads = round32((B * m3 + EL - 1) / EL);
        z_smem = std::max(sizeof(V) * ((size_t)B * (m3 + 1) + m3), (size_t)32 * 16 * 8);
        if (x_threads > 256 || y_threads > 256 || z_threads > 256) throw std::runtime_error("grid dimension too large for the line passes");
    }

    void allocate()
    {
        const size_t Vn = V_;
        const int nm = c.nm, M = c.M, J = (int)c.ions.size();
        tw1.alloc(c.m1); tw2.alloc(c.m2); tw3.alloc(c.m3);
        kx.alloc(c.m1); ky.alloc(c.m2); kz.alloc(c.m3);
        const int sum_m = c.m1 + c.m2 + c.m3;
        phi.alloc((size_t)std::max<size_t>(1, c.bond_lengths.size()) * sum_m);
        gam.alloc(sum_m);
        gion.alloc((size_t)std::max(1, J) * sum_m);
        const size_t nmv = Vn * std::max(1, nm);
        omega.alloc(nmv); omega_bar.alloc(nmv); drift.alloc(nmv); drift_bar.alloc(nmv);
        psi.alloc(Vn); psi_bar.alloc(Vn); dpsi.alloc(Vn); dpsi_bar.alloc(Vn);
        // partials of the fused semi-implicit update (allocated here: a step
        // may run under stream capture, where nothing can be allocated)
        if (c.scheme == FTSP_SCHEME_SI) upart.alloc(2 * (size_t)c.m1 * (nm + 1));
        eta.alloc((size_t)(nm + 1) * Vn);
        kA.alloc((size_t)2 * (nm + 1) * Vn);   // upper half: scratch of the fused evaluation's first pass
        kB.alloc((size_t)(M + 1 + J) * Vn);
        dB.alloc((size_t)(M + 1 + J) * Vn);
        kC.alloc((size_t)(M + 3) * Vn);
        rho_p.alloc(Vn); rho_c.alloc(Vn); ion_rho.alloc(Vn * std::max(1, J));
        E.alloc(Vn * std::max<size_t>(1, c.cls.size()));
        Nmax = 1;
        for (auto& s : c.sp) Nmax = std::max(Nmax, s.N);
        qF.alloc(Vn * Nmax);
        if (c.stress_on()) Fst.alloc(Vn * Nmax);
        G.alloc(Vn); H.alloc(Vn);
        part.alloc((size_t)std::max(RED_BLOCKS, std::max(c.m1, c.m1 * c.m2)) * 32);
        expo.alloc((size_t)2 * Nmax);
        pmax.alloc((size_t)2 * std::max(c.m1, c.m1 * c.m2));
        spart.alloc((size_t)c.m2 * c.m3 * 12);
        if (c.restart_interval > 0) ck.alloc((size_t)(std::max(1, c.nm) + 1) * V_);
        FTSP_CUDA(cudaMalloc(&ds, sizeof(DevScal)));
        FTSP_CUDA(cudaMemset(ds, 0, sizeof(DevScal)));
        {
            const double one = 1.0;
            FTSP_CUDA(cudaMemcpy(&ds->dt_scale, &one, sizeof(double), cudaMemcpyHostToDevice));
        }
        FTSP_CUDA(cudaMemset(omega.p, 0, sizeof(V) * nmv));
        FTSP_CUDA(cudaMemset(psi.p, 0, sizeof(V) * Vn));
        FTSP_CUDA(cudaMemset(eta.p, 0, sizeof(T) * eta.n));
    }

    // ---- autotuner ----
    // For every candidate geometry (FFT radix cap, strided tile width) the
    // forward and inverse 3-D transforms of one field are timed with CUDA
    // events (one warm-up, then the mean of three); the fastest is kept.
    // Results are cached per (grid, precision, device) for the process, so a
    // set of replicas of the same grid tunes once.  Grids whose passes are
    // all compile-time kernels (32/64/128 cubes) have nothing to tune.
    struct TuneKey {
        int m1, m2, m3, f32, dev;
        bool operator<(const TuneKey& o) const
        {
            return std::tie(m1, m2, m3, f32, dev) < std::tie(o.m1, o.m2, o.m3, o.f32, o.dev);
        }
    };
    struct TuneResult {
        int max_bits = 0, W = 0, candidates = 0;
        double best_ms = 0.0, default_ms = 0.0;
        bool tuned = false, cached = false;
    };
    static std::map<TuneKey, TuneResult>& tune_cache()
    {
        static std::map<TuneKey, TuneResult> m;
        return m;
    }
    static std::mutex& tune_mutex()
    {
        static std::mutex m;
        return m;
    }
    TuneResult tune{};

    bool all_compile_time() const
    {
        const bool plane = plane_ok && c.m2 == c.m3 && (c.m3 == 32 || c.m3 == 64 || c.m3 == 128) &&
                           (F32 || c.m3 != 128);
        return plane && strided_is_ct(c.m1);
    }

    double time_fft(int reps)
    {
        cudaEvent_t a, b;
        FTSP_CUDA(cudaEventCreate(&a));
        FTSP_CUDA(cudaEventCreate(&b));
        fft3<-1>(G.p, 1);
        fft3<+1>(G.p, 1);
        FTSP_CUDA(cudaEventRecord(a, stream));
        for (int r = 0; r < reps; ++r) {
            fft3<-1>(G.p, 1);
            fft3<+1>(G.p, 1);
        }
        FTSP_CUDA(cudaEventRecord(b, stream));
        FTSP_CUDA(cudaEventSynchronize(b));
        float ms = 0.0f;
        FTSP_CUDA(cudaEventElapsedTime(&ms, a, b));
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return (double)ms / reps;
    }

    void autotune()
    {
        const TuneKey key{c.m1, c.m2, c.m3, F32 ? 1 : 0, c.device};
        std::lock_guard<std::mutex> lock(tune_mutex());
        auto it = tune_cache().find(key);
        if (it != tune_cache().end()) {
            tune = it->second;
            tune.cached = true;
            setup_geometry(tune.max_bits, tune.W);
            return;
        }
        TuneResult r{};
        if (all_compile_time()) {
            r.max_bits = geo_max_bits;
            r.W = geo_W;
            tune_cache()[key] = r;
            tune = r;
            return;
        }
        FTSP_CUDA(cudaMemsetAsync(G.p, 0, sizeof(V) * V_, stream));
        std::vector<int> bits = F32 ? std::vector<int>{2, 3, 4} : std::vector<int>{2, 3};
        std::vector<int> Ws;
        for (int w = w_max(); w >= 1 && Ws.size() < 3; --w)
            if (c.m3 % w == 0) Ws.push_back(w);
        setup_geometry(0, 0);
        r.default_ms = time_fft(3);
        r.best_ms = r.default_ms;
        r.max_bits = geo_max_bits;
        r.W = geo_W;
        for (int mb : bits)
            for (int w : Ws) {
                setup_geometry(mb, w);
                const double t = time_fft(3);
                ++r.candidates;
                if (t < r.best_ms) {
                    r.best_ms = t;
                    r.max_bits = mb;
                    r.W = w;
                }
            }
        setup_geometry(r.max_bits, r.W);
        r.tuned = true;
        tune_cache()[key] = r;
        tune = r;
    }

    template <typename X>
    void upload(Buf<X>& b, const std::vector<X>& h)
    {
        FTSP_CUDA(cudaMemcpy(b.p, h.data(), sizeof(X) * h.size(), cudaMemcpyHostToDevice));
    }

    void build_tables()
    {
        auto tw = [](int n) {
            std::vector<V> t(n);
            for (int j = 0; j < n; ++j) {
                const long double ang = -2.0L * 3.141592653589793238462643383279502884L * j / n;
                t[j].x = (T)cosl(ang);
                t[j].y = (T)sinl(ang);
            }
            return t;
        };
        upload(tw1, tw(c.m1));
        upload(tw2, tw(c.m2));
        upload(tw3, tw(c.m3));
        std::vector<double> hx(c.m1), hy(c.m2), hz(c.m3);
        for (int i = 0; i < c.m1; ++i) hx[i] = wave_number(i, c.m1, c.L[0]);
        for (int i = 0; i < c.m2; ++i) hy[i] = wave_number(i, c.m2, c.L[1]);
        for (int i = 0; i < c.m3; ++i) hz[i] = wave_number(i, c.m3, c.L[2]);
        upload(kx, hx); upload(ky, hy); upload(kz, hz);
        // separable Gaussian factor tables exp(-f k_d^2) for each dimension
        auto sep = [&](double f) {
            std::vector<T> t;
            for (double k : hx) t.push_back((T)std::exp(-f * k * k));
            for (double k : hy) t.push_back((T)std::exp(-f * k * k));
            for (double k : hz) t.push_back((T)std::exp(-f * k * k));
            return t;
        };
        std::vector<T> ph;
        for (double b : c.bond_lengths) {
            auto t = sep(b * b / 6.0);
            ph.insert(ph.end(), t.begin(), t.end());
        }
        if (ph.empty()) ph = sep(0.0);
        upload(phi, ph);
        upload(gam, sep(0.5 * c.a * c.a));
        std::vector<T> gi;
        for (auto& ion : c.ions) {
            auto t = sep(0.5 * ion.smear * ion.smear);
            gi.insert(gi.end(), t.begin(), t.end());
        }
        if (gi.empty()) gi = sep(0.0);
        upload(gion, gi);
        ion_common = c.elec && !c.ions.empty() && c.ions.size() <= 3;
        for (auto& ion : c.ions) ion_common = ion_common && ion.smear == c.a;
        if (c.scheme == FTSP_SCHEME_SI) build_si_tables();
    }

    // ---- semi-implicit preconditioner (no reference counterpart) ----
    // Linear response of the drifts at the homogeneous state, per k:
    //   G_a(k)   = c_a - Re(gamma_a^2) Gamma(k)^2 sum_sp (n_sp/V) S_oo(k),  o_s = O_{a, type(s)}
    //   G_psi(k) = k^2/(4 pi lB) + Gamma(k)^2 sum_sp (n_sp/V) S_zz(k) + sum_j (n_j/V) z_j^2 Gamma_j(k)^2
    // with the discrete-Gaussian-chain correlation sum
    //   S_ww(k) = sum_{s,s'} w_s w_s' prod_{t between s and s'} exp(-b_t^2 k^2/6),
    // evaluated by the recursion F_s = phi_{s-1} F_{s-1} + w_s,
    // S += w_s (w_s + 2 phi_{s-1} F_{s-1}).  The chain terms vanish at k = 0
    // (the densities are normalised by Q).  G_a is clipped at zero.  The
    // update divides each increment by P^-1 = 1 + lambda dt G(k).
    void build_si_tables()
    {
        const size_t Vn = V_;
        const int nm = c.nm;
        si_G.alloc((size_t)(nm + 1) * Vn);
        si_inc.alloc((size_t)(nm + 1) * Vn);
        // segment data: per segment (type, charge, bond class of the bond to the next segment)
        std::vector<int> stype, sbond, soff, sN;
        std::vector<double> schg, snv;
        for (auto& s : c.sp) {
            soff.push_back((int)stype.size());
            sN.push_back(s.N);
            snv.push_back(s.nc / c.volume);
            for (int t = 0; t < s.N; ++t) {
                stype.push_back(s.type[t]);
                schg.push_back(c.elec ? s.charge[t] : 0.0);
                sbond.push_back(t + 1 < s.N ? s.bcls[t] : 0);
            }
        }
        Buf<int> d_type, d_bond, d_off, d_N;
        Buf<double> d_chg, d_nv, d_blen;
        d_type.alloc(stype.size()); upload(d_type, stype);
        d_bond.alloc(sbond.size()); upload(d_bond, sbond);
        d_off.alloc(soff.size()); upload(d_off, soff);
        d_N.alloc(sN.size()); upload(d_N, sN);
        d_chg.alloc(schg.size()); upload(d_chg, schg);
        d_nv.alloc(snv.size()); upload(d_nv, snv);
        std::vector<double> blen = c.bond_lengths;
        if (blen.empty()) blen.push_back(1.0);
        d_blen.alloc(blen.size()); upload(d_blen, blen);
        ModeTab co{};
        for (int a = 0; a < nm; ++a) {
            co.c[a] = c.coeff[a];
            co.s[a] = c.dt * c.lambda[a];
            co.g[a] = make_double2(c.gamma[a].x * c.gamma[a].x - c.gamma[a].y * c.gamma[a].y, 0.0);   // Re(gamma^2)
        }
        SiOTab so{};
        if (c.bond_lengths.size() > 8) throw std::runtime_error("semi-implicit scheme: at most 8 distinct bond lengths");
        for (int a = 0; a < nm; ++a)
            for (int al = 0; al < c.M; ++al) so.O[a * c.M + al] = c.O[a * c.M + al];
        IonTab it{};
        const int J = (int)c.ions.size();
        for (int j = 0; j < J; ++j) {
            it.z[j] = c.ions[j].z;
            it.nd[j] = c.ions[j].count / c.volume;
            it.a2[j] = c.ions[j].smear * c.ions[j].smear;
        }
        const int M = c.M, nsp = (int)c.sp.size(), nbc = (int)blen.size();
        const int m1 = c.m1, m2 = c.m2, m3 = c.m3;
        const double a2 = c.a * c.a, lB = c.lB;
        const bool elec = c.elec;
        const double* kxp = kx.p;
        const double* kyp = ky.p;
        const double* kzp = kz.p;
        const int* ty = d_type.p;
        const int* bo = d_bond.p;
        const int* of = d_off.p;
        const int* Ns = d_N.p;
        const double* ch = d_chg.p;
        const double* nvp = d_nv.p;
        const double* bl = d_blen.p;
        T* P = si_G.p;
        foreach(Vn, [=] __device__(size_t i) {
            const int x = (int)(i / ((size_t)m2 * m3));
            const int r = (int)(i - (size_t)x * m2 * m3);
            const int y = r / m3, z = r - y * m3;
            const double k2 = kxp[x] * kxp[x] + kyp[y] * kyp[y] + kzp[z] * kzp[z];
            const double G2 = exp(-a2 * k2);   // Gamma^2
            double phc[8];
            for (int q = 0; q < nbc && q < 8; ++q) phc[q] = exp(-bl[q] * bl[q] * k2 / 6.0);
            double Soo[MAXMODE], Szz = 0.0;
            for (int a = 0; a < nm; ++a) Soo[a] = 0.0;
            for (int sp = 0; sp < nsp; ++sp) {
                const double w = nvp[sp];
                double Fo[MAXMODE], Fz = 0.0;
                for (int a = 0; a < nm; ++a) Fo[a] = 0.0;
                const int o0 = of[sp];
                for (int t = 0; t < Ns[sp]; ++t) {
                    const double ph = t > 0 ? phc[bo[o0 + t - 1]] : 0.0;
                    const int tp = ty[o0 + t];
                    for (int a = 0; a < nm; ++a) {
                        const double o = so.O[a * M + tp];
                        Fo[a] *= ph;
                        Soo[a] += w * o * (o + 2.0 * Fo[a]);
                        Fo[a] += o;
                    }
                    const double zt = ch[o0 + t];
                    Fz *= ph;
                    Szz += w * zt * (zt + 2.0 * Fz);
                    Fz += zt;
                }
            }
            const bool k0 = k2 == 0.0;
            for (int a = 0; a < nm; ++a) {
                double G = co.c[a] - (k0 ? 0.0 : co.g[a].x * G2 * Soo[a]);
                if (G < 0.0) G = 0.0;
                P[(size_t)a * Vn + i] = (T)G;
            }
            double Gp = 0.0;
            if (elec && !k0) {
                Gp = k2 / (4.0 * PI * lB) + G2 * Szz;
                for (int j = 0; j < J; ++j) Gp += it.nd[j] * it.z[j] * it.z[j] * exp(-it.a2[j] * k2);
            }
            P[(size_t)nm * Vn + i] = (T)Gp;
        });
        FTSP_CUDA(cudaStreamSynchronize(stream));
        d_type.release(); d_bond.release(); d_off.release(); d_N.release(); d_chg.release(); d_nv.release(); d_blen.release();
    }

    // increments (nm + 1 fields of si_inc) -> P * increments, in place, with
    // P_f(k) = 1 / (1 + dt lambda_f G_f(k)) from the analytic table, or from
    // the learned one while the residual test allows it (device flag lr_use).
    // stash: keep the k-space increments FFT[omega_bar - omega] for the
    // learned preconditioner's statistics and residual test.
    void si_precondition(bool stash = false)
    {
        const size_t Vn = V_;
        const int nf = c.nm + 1;
        if (plane_ok) {
            // yz forward; x forward, P(k) / V, x inverse in one pencil pass; yz inverse
            cudaEvent_t ev = prof_begin();
            OpLoadN<T> self{};
            for (int f = 0; f < nf; ++f) self.s[f] = si_inc.p + (size_t)f * Vn;
            self.fs = Vn;
            plane<0, -1>(nullptr, si_inc.p, nf, self);
            OpPrecond<T> op{};
            op.GA = si_G.p;
            op.GL = lr.on_use ? lr.GL.p : nullptr;
            op.dw = stash ? lr.dw.p : nullptr;
            op.d = ds;
            for (int a = 0; a < c.nm; ++a) op.st.s[a] = c.dt * c.lambda[a];
            op.st.s[c.nm] = c.dt * c.lpsi;
            op.invV = (T)(1.0 / (double)Vn);
            strided<0, -1, +1>(si_inc.p, si_inc.p, nf, op);
            plane<+1, 0>(si_inc.p, nullptr, nf, OpStore<T>{si_inc.p});
            // three passes reading and writing every field, plus the G table
            prof_end(ev, "field_fft", (double)nf * (6.0 * sizeof(V) + sizeof(T)) * (double)Vn);
            return;
        }
        fft3<-1>(si_inc.p, nf);
        V* inc = si_inc.p;
        const T* GA = si_G.p;
        const T* GL = lr.on_use ? lr.GL.p : nullptr;
        V* dw = stash ? lr.dw.p : nullptr;
        SigTab st{};
        for (int a = 0; a < c.nm; ++a) st.s[a] = c.dt * c.lambda[a];
        st.s[c.nm] = c.dt * c.lpsi;
        const DevScal* d = ds;
        const T invV = (T)(1.0 / (double)Vn);
        foreach(Vn * nf, [=] __device__(size_t i) {
            const int f = (int)(i / Vn);
            const T G = (GL && d->lr_use) ? GL[i] : GA[i];
            const V k = cscale(inc[i], (T)(1.0 / (1.0 + (st.s[f] * d->dt_scale) * (double)G)));
            if (dw) dw[i] = k;
            inc[i] = cscale(k, invV);
        }, (double)(2 * sizeof(V) + sizeof(T)));
        fft3<+1>(si_inc.p, nf);
    }

    // The whole semi-implicit update of the predictor (corr = false) or the
    // corrector in three transform passes (grids with the plane pass): the
    // increments are computed as the loads of the forward yz pass
    // (OpIncrement, with the drift maxima of the corrector), the x pass
    // applies P(k) and removes the psi increment's k = 0 value, and the
    // inverse yz pass adds the increments to the fields (OpUpdate, with the
    // corrector's non-finite count).  Removing the mean of the psi increment
    // in k-space replaces the real-space mean removal of the updated psi
    // (complexLangevin.cu:313-317): psi keeps the zero mean it was given
    // (set_fields), up to rounding, and the physics does not depend on it.
    Buf<double> upart;   // per-CTA drift maxima and non-finite counts of the fused update

    void si_update_fused(bool corr, bool stash)
    {
        const size_t Vn = V_;
        const int nm = c.nm, nf = nm + 1;
        const size_t nparts = (size_t)c.m1 * nf;
        cudaEvent_t ev = prof_begin();
        if (corr) {
            OpIncrement<T, true> op{};
            op.u0 = drift.p; op.u1 = drift_bar.p; op.e = eta.p; op.dp = dpsi.p; op.db = dpsi_bar.p; op.d = ds;
            for (int a = 0; a < nm; ++a) op.cs.s[a] = -0.5 * c.dt * c.lambda[a];
            op.cs.s[nm] = -0.5 * c.dt * c.lpsi;
            op.invV = 1.0 / (double)Vn; op.Vn = Vn; op.nm = nm; op.elec = c.elec; op.dpart = upart.p;
            plane<0, -1>(nullptr, si_inc.p, nf, op);
        } else {
            OpIncrement<T, false> op{};
            op.u0 = drift.p; op.e = eta.p; op.dp = dpsi.p; op.d = ds;
            for (int a = 0; a < nm; ++a) op.cs.s[a] = -c.dt * c.lambda[a];
            op.cs.s[nm] = -c.dt * c.lpsi;
            op.invV = 1.0 / (double)Vn; op.Vn = Vn; op.nm = nm; op.elec = c.elec;
            plane<0, -1>(nullptr, si_inc.p, nf, op);
        }
        OpPrecond<T> pr{};
        pr.GA = si_G.p;
        pr.GL = lr.on_use ? lr.GL.p : nullptr;
        pr.dw = stash ? lr.dw.p : nullptr;
        pr.d = ds;
        for (int a = 0; a < nm; ++a) pr.st.s[a] = c.dt * c.lambda[a];
        pr.st.s[nm] = c.dt * c.lpsi;
        pr.invV = (T)(1.0 / (double)Vn);
        pr.dc0 = c.elec ? nm : -1;
        strided<0, -1, +1>(si_inc.p, si_inc.p, nf, pr);
        OpUpdate<T> up{};
        up.w0 = corr ? omega.p : omega.p;
        up.p0 = psi.p;
        up.w1 = corr ? omega.p : omega_bar.p;
        up.p1 = corr ? psi.p : psi_bar.p;
        up.Vn = Vn; up.nm = nm; up.elec = c.elec;
        up.npart = corr ? upart.p + nparts : nullptr;
        plane<+1, 0>(si_inc.p, nullptr, nf, up);
        // loads: drifts, noise (real), psi drift read and written; three
        // passes over the increments; the fields read and written
        const double units = corr ? (2.0 * nm + 0.5 * nf + 3.0 + nf) + 2.5 * nf + 3.0 * nf
                                  : (1.0 * nm + 0.5 * nf + 2.5 + nf) + 2.5 * nf + 3.0 * nf;
        prof_end(ev, "field_fft", units * sizeof(V) * (double)Vn);
        if (corr) {
            for (int f = 0; f < nf; ++f) {
                k_combine<true><<<1, COMBINE_THREADS, 0, stream>>>(upart.p + (size_t)f * c.m1, c.m1, 1, ds->dmax + f);
                ++launches;
            }
            k_combine<false><<<1, COMBINE_THREADS, 0, stream>>>(upart.p + nparts, (int)nparts, 1, ds->corr + 2);
            ++launches;
        }
    }

    // ---- learned semi-implicit preconditioner (learned.cuh) ----
    struct Learn {
        bool configured = false, on_collect = false, on_use = false, trained = false;
        int nout = 0, np = 0, nb = 0;
        float N = 50.0f, lB = 1.0f, salt = 0.0f;
        double lr = 1e-3, fallback = 1.5;
        int batch = 4096, refresh_every = 100;
        uint64_t seed = 7;
        long long collected = 0, power_updates = 0, since_refresh = 0;
        long long valid_targets = 0;   // (k, field) targets of the last training call
        int adam_t = 0;
        double last_loss = 0.0;
        Buf<float> A, B, Pw, Pp;      // statistics: <Re(du dw*)>, <|dw|^2> per field and k; spectral powers
        Buf<T> GL;                    // learned G(k): modes, then psi
        Buf<V> dw, du, fk;            // k-space increments, drift changes, field transforms
        Buf<float> w, m1, m2, partial;
        Buf<double> lpart, loss;
    } lr;

    void learn_release()
    {
        Buf<float>* fb[] = {&lr.A, &lr.B, &lr.Pw, &lr.Pp, &lr.w, &lr.m1, &lr.m2, &lr.partial};
        for (auto* b : fb) b->release();
        lr.GL.release(); lr.dw.release(); lr.du.release(); lr.fk.release();
        lr.lpart.release(); lr.loss.release();
    }

    LearnFeat learn_feat() const
    {
        return LearnFeat{kx.p, ky.p, kz.p, lr.Pw.p, lr.Pp.p, c.m2, c.m3, lr.N, lr.lB, lr.salt};
    }

    void tune_info(ftsp_tune_info* t) override
    {
        std::memset(t, 0, sizeof(*t));
        t->tuned = tune.tuned ? 1 : 0;
        t->cached = tune.cached ? 1 : 0;
        t->compile_time = all_compile_time() ? 1 : 0;
        t->max_radix = 1 << geo_max_bits;
        t->tile_width = geo_W;
        t->candidates = tune.candidates;
        t->best_ms = tune.best_ms;
        t->default_ms = tune.default_ms;
    }

    // ---- adaptive step ----
    // dt_eff = dt min(1, u_ref / max|u|) with max|u| the largest drift
    // magnitude of any field at the start of the step (the adaptive step size
    // of Aarts, James, Seiler and Stamatescu, Phys. Lett. B 687 (2010) 154, for
    // complex Langevin runaways).  Noise amplitudes, the predictor, the
    // corrector and the semi-implicit P(k) all use dt_eff; time averages
    // should be weighted by it (ftsp_step_info).
    double adaptive_u = 0.0;
    void set_adaptive(double u_ref) override
    {
        if (!(u_ref >= 0.0)) throw std::runtime_error("ftsp_set_adaptive: u_ref must be >= 0");
        adaptive_u = u_ref;
        drop_step_graph();
        if (u_ref == 0.0) {
            const double one = 1.0;
            FTSP_CUDA(cudaMemcpyAsync(&ds->dt_scale, &one, sizeof(double), cudaMemcpyHostToDevice, stream));
            FTSP_CUDA(cudaStreamSynchronize(stream));
        }
    }

    void adapt_dt()
    {
        const size_t Vn = V_;
        const int nm = c.nm;
        const V* u = drift.p;
        const V* dp = dpsi.p;
        const bool elec = c.elec;
        reduce<1, true>(Vn, [=] __device__(size_t i, double* acc) {
            double m = 0.0;
            for (int a = 0; a < nm; ++a) {
                const double2 v = to_d(u[(size_t)a * Vn + i]);
                m = fmax(m, v.x * v.x + v.y * v.y);
            }
            if (elec) {
                const double2 v = to_d(dp[i]);
                m = fmax(m, v.x * v.x + v.y * v.y);
            }
            if (!isfinite(m)) m = INFINITY;
            acc[0] = fmax(acc[0], m);
        }, &ds->umax, (double)(c.nm + 1) * sizeof(V));
        DevScal* d = ds;
        const double uref = adaptive_u;
        k_foreach<<<1, 32, 0, stream>>>(1, [=] __device__(size_t) {
            const double um = sqrt(d->umax);
            d->umax = um;
            d->dt_scale = (isfinite(um) && um > uref) ? uref / um : 1.0;
        });
        ++launches;
    }

    void step_info(double* dt_eff, double* umax) override
    {
        pull_scalars();
        if (dt_eff) *dt_eff = c.dt * hs.dt_scale;
        if (umax) *umax = hs.umax;
    }

    void set_chain_symmetry(bool on) override
    {
        chain_sym = on;
        drop_step_graph();
    }
    int chain_symmetric_species() override
    {
        int n = 0;
        for (const auto& t : sym) n += (chain_sym && t.ok) ? 1 : 0;
        return n;
    }

    void set_dt(double dt) override
    {
        if (!(dt > 0.0)) throw std::runtime_error("ftsp_set_dt: dt must be positive");
        c.dt = dt;
        drop_step_graph();
    }

    void learn_configure(const ftsp_learn_config& cf) override
    {
        drop_step_graph();
        if (c.scheme != FTSP_SCHEME_SI || !si_G.p) throw std::runtime_error("the learned preconditioner needs the semi-implicit scheme");
        const int nf = c.nm + 1;
        if (nf > mlp::NOUT_MAX) throw std::runtime_error("the learned preconditioner supports at most 3 interaction modes");
        learn_release();
        lr = Learn{};
        lr.nout = nf;
        lr.np = mlp::n_params(nf);
        lr.N = (float)cf.N;
        lr.lB = (float)cf.lB;
        lr.salt = (float)cf.salt;
        if (cf.lr > 0.0) lr.lr = cf.lr;
        if (cf.batch > 0) lr.batch = (cf.batch + mlp::GRAD_THREADS - 1) / mlp::GRAD_THREADS * mlp::GRAD_THREADS;
        if (cf.refresh_every > 0) lr.refresh_every = cf.refresh_every;
        if (cf.fallback_ratio > 0.0) lr.fallback = cf.fallback_ratio;
        lr.seed = cf.seed;
        lr.nb = lr.batch / mlp::GRAD_THREADS;
        const size_t Vn = V_;
        lr.A.alloc(nf * Vn); lr.B.alloc(nf * Vn); lr.Pw.alloc(Vn); lr.Pp.alloc(Vn);
        lr.GL.alloc(nf * Vn); lr.dw.alloc(nf * Vn); lr.du.alloc(nf * Vn); lr.fk.alloc(2 * Vn);
        lr.w.alloc(lr.np); lr.m1.alloc(lr.np); lr.m2.alloc(lr.np);
        lr.partial.alloc((size_t)lr.nb * lr.np); lr.lpart.alloc(2 * (size_t)lr.nb); lr.loss.alloc(2);
        FTSP_CUDA(cudaMemsetAsync(lr.A.p, 0, sizeof(float) * nf * Vn, stream));
        FTSP_CUDA(cudaMemsetAsync(lr.B.p, 0, sizeof(float) * nf * Vn, stream));
        FTSP_CUDA(cudaMemsetAsync(lr.Pw.p, 0, sizeof(float) * Vn, stream));
        FTSP_CUDA(cudaMemsetAsync(lr.Pp.p, 0, sizeof(float) * Vn, stream));
        FTSP_CUDA(cudaMemsetAsync(lr.m1.p, 0, sizeof(float) * lr.np, stream));
        FTSP_CUDA(cudaMemsetAsync(lr.m2.p, 0, sizeof(float) * lr.np, stream));
        // Glorot-uniform weights, zero biases, from the configured seed
        std::vector<float> w(lr.np, 0.0f);
        uint64_t st = cf.seed * 6364136223846793005ull + 1442695040888963407ull;
        auto uni = [&st]() {   // 64-bit LCG (Knuth's MMIX constants), top 24 bits
            st = st * 6364136223846793005ull + 1442695040888963407ull;
            return (float)((st >> 40) * (1.0 / 16777216.0));
        };
        auto fill = [&](int off, int fan_in, int fan_out, int n) {
            const float a = std::sqrt(6.0f / (float)(fan_in + fan_out));
            for (int k = 0; k < n; ++k) w[off + k] = (2.0f * uni() - 1.0f) * a;
        };
        fill(0, mlp::NIN, mlp::H, mlp::H * mlp::NIN);
        fill(mlp::off_w2(), mlp::H, mlp::H, mlp::H * mlp::H);
        fill(mlp::off_w3(), mlp::H, nf, nf * mlp::H);
        FTSP_CUDA(cudaMemcpyAsync(lr.w.p, w.data(), sizeof(float) * lr.np, cudaMemcpyHostToDevice, stream));
        FTSP_CUDA(cudaMemcpyAsync(lr.GL.p, si_G.p, sizeof(T) * nf * Vn, cudaMemcpyDeviceToDevice, stream));
        FTSP_CUDA(cudaMemsetAsync(&ds->lr_use, 0, 3 * sizeof(int), stream));
        FTSP_CUDA(cudaMemsetAsync(ds->lres_sum, 0, sizeof(ds->lres_sum), stream));
        FTSP_CUDA(cudaStreamSynchronize(stream));
        lr.configured = true;
    }

    void learn_require() const
    {
        if (!lr.configured) throw std::runtime_error("ftsp_learn_configure has not been called");
    }

    void learn_collect(bool on) override
    {
        drop_step_graph();
        learn_require();
        lr.on_collect = on;
    }

    // clears the collected (force, increment) statistics and the residual
    // sums; the network, its optimiser state and the spectral powers are kept
    void learn_reset() override
    {
        learn_require();
        const size_t n = (size_t)lr.nout * V_;
        FTSP_CUDA(cudaMemsetAsync(lr.A.p, 0, sizeof(float) * n, stream));
        FTSP_CUDA(cudaMemsetAsync(lr.B.p, 0, sizeof(float) * n, stream));
        FTSP_CUDA(cudaMemsetAsync(ds->lres_sum, 0, sizeof(ds->lres_sum), stream));
        FTSP_CUDA(cudaStreamSynchronize(stream));
        lr.collected = 0;
    }

    // after the predictor's densities and drifts: the drift change du =
    // u(omega_bar) - u(omega) in k-space, against the increment dw stashed by
    // the predictor.  Collects <Re(du dw*)>, <|dw|^2>; while the learned G is
    // in use, compares the force residuals |du - G dw|^2 of the learned and
    // the analytic G and selects the kernel of the next step.
    void learn_after_predictor()
    {
        const size_t Vn = V_;
        const int nm = c.nm, nf = nm + 1;
        V* du = lr.du.p;
        {
            const V* u0 = drift.p;
            const V* u1 = drift_bar.p;
            const V* p0 = dpsi.p;
            const V* p1 = dpsi_bar.p;
            const bool elec = c.elec;
            foreach(Vn, [=] __device__(size_t i) {
                for (int a = 0; a < nm; ++a) du[(size_t)a * Vn + i] = csub(u1[(size_t)a * Vn + i], u0[(size_t)a * Vn + i]);
                du[(size_t)nm * Vn + i] = elec ? csub(p1[i], p0[i]) : mkc<V>(T(0), T(0));
            });
        }
        fft3<-1>(du, nf);
        const V* dw = lr.dw.p;
        if (lr.on_collect) {
            float* A = lr.A.p;
            float* B = lr.B.p;
            // a step that runs away leaves non-finite values at some k: those
            // contributions are skipped so that they cannot poison the sums
            foreach(Vn * nf, [=] __device__(size_t i) {
                const V a = du[i], b = dw[i];
                const double ca = (double)a.x * b.x + (double)a.y * b.y;
                const double cb = (double)b.x * b.x + (double)b.y * b.y;
                if (isfinite(ca) && isfinite(cb)) {
                    A[i] += (float)ca;
                    B[i] += (float)cb;
                }
            });
            ++lr.collected;
        }
        if (lr.on_use) {
            const T* GL = lr.GL.p;
            const T* GA = si_G.p;
            reduce<2>(Vn * nf, [=] __device__(size_t i, double* acc) {
                const V a = du[i], b = dw[i];
                const double gl = (double)GL[i], ga = (double)GA[i];
                const double rlx = (double)a.x - gl * b.x, rly = (double)a.y - gl * b.y;
                const double rax = (double)a.x - ga * b.x, ray = (double)a.y - ga * b.y;
                acc[0] += rlx * rlx + rly * rly;
                acc[1] += rax * rax + ray * ray;
            }, ds->lres);
            DevScal* d = ds;
            const double ratio = lr.fallback;
            k_foreach<<<1, 32, 0, stream>>>(1, [=] __device__(size_t) {
                const bool ok = isfinite(d->lres[0]) && d->lres[0] <= ratio * d->lres[1];
                if (isfinite(d->lres[0]) && isfinite(d->lres[1])) {
                    d->lres_sum[0] += d->lres[0];
                    d->lres_sum[1] += d->lres[1];
                }
                d->lr_checks += 1;
                if (!ok) d->lr_fallbacks += 1;
                d->lr_use = ok ? 1 : 0;
            });
            ++launches;
        }
    }

    // running spectral powers |FFT f|^2 / V of the first mode and of psi
    // (mean over the first 200 updates, then an exponential average with the
    // same window)
    void learn_power()
    {
        const size_t Vn = V_;
        const V* src[2] = {c.nm > 0 ? omega.p : psi.p, psi.p};
        fft3<-1>(lr.fk.p, 2, src);
        const V* fk = lr.fk.p;
        float* Pw = lr.Pw.p;
        float* Pp = lr.Pp.p;
        const float alpha = 1.0f / (float)std::min<long long>(lr.power_updates + 1, 200);
        const float invV = (float)(1.0 / (double)Vn);
        const bool have_w = c.nm > 0, elec = c.elec;
        foreach(Vn, [=] __device__(size_t i) {
            const V a = fk[i], b = fk[Vn + i];
            const float pa = have_w ? (float)((double)a.x * a.x + (double)a.y * a.y) * invV : 0.0f;
            const float pb = elec ? (float)((double)b.x * b.x + (double)b.y * b.y) * invV : 0.0f;
            if (isfinite(pa)) Pw[i] += alpha * (pa - Pw[i]);
            if (isfinite(pb)) Pp[i] += alpha * (pb - Pp[i]);
        });
        ++lr.power_updates;
    }

    // G_L(k) = G_Debye(k) exp(z(k)) over the grid from the current features
    void learn_refresh()
    {
        const size_t Vn = V_;
        const int nf = lr.nout;
        T* GL = lr.GL.p;
        const T* GA = si_G.p;
        const LearnFeat ft = learn_feat();
        auto out = [=] __device__(size_t i, const float* z) {
            for (int f = 0; f < nf; ++f) {
                const size_t j = (size_t)f * Vn + i;
                const T ga = GA[j];
                // correction factor exp(z) on the analytic coefficient; where
                // the analytic coefficient vanishes it is kept
                GL[j] = ga > T(0) ? (T)((double)ga * exp((double)fminf(fmaxf(z[f], -20.0f), 20.0f))) : ga;
            }
        };
        const int blocks = (int)std::min<size_t>((Vn + 127) / 128, 148 * 8);
        mlp::k_eval<<<blocks, 128, sizeof(float) * lr.np, stream>>>(Vn, lr.w.p, nf, ft, out);
        ++launches;
        lr.since_refresh = 0;
    }

    void learn_after_step()
    {
        learn_power();
        if (lr.on_use && ++lr.since_refresh >= lr.refresh_every) learn_refresh();
    }

    // Adam on the collected statistics: each iteration draws `batch` wave
    // vectors (counter-based, from the seed and the iteration), with targets
    // log(A / (B G_Debye)) per field where A, B and G_Debye are positive.
    double learn_train(int iterations) override
    {
        learn_require();
        if (lr.collected < 1) throw std::runtime_error("ftsp_learn_train: no statistics collected");
        const size_t Vn = V_;
        const int nf = lr.nout;
        const float* A = lr.A.p;
        const float* B = lr.B.p;
        const T* GA = si_G.p;
        const LearnFeat ft = learn_feat();
        const uint32_t s0 = (uint32_t)lr.seed, s1 = (uint32_t)(lr.seed >> 32);
        // target: log of the measured coefficient over the analytic one
        auto target = [=] __device__(size_t i, int f, float& t, float& m) {
            const size_t j = (size_t)f * Vn + i;
            const double a = A[j], b = B[j], ga = (double)GA[j];
            const bool ok = ga > 0.0 && a > 0.0 && b > 0.0 && isfinite(a) && isfinite(b);
            t = ok ? (float)log(a / (b * ga)) : 0.0f;
            m = ok ? 1.0f : 0.0f;
        };
        // valid targets per field (and their sum, for the initial output biases)
        double h[2 * mlp::NOUT_MAX];
        {
            double* tsum = reinterpret_cast<double*>(ds->kobs);
            reduce<2 * mlp::NOUT_MAX>(Vn, [=] __device__(size_t i, double* acc) {
                for (int f = 0; f < nf; ++f) {
                    float t, m;
                    target(i, f, t, m);
                    acc[2 * f] += (double)(t * m);
                    acc[2 * f + 1] += (double)m;
                }
            }, tsum);
            FTSP_CUDA(cudaMemcpyAsync(h, tsum, sizeof(h), cudaMemcpyDeviceToHost, stream));
            FTSP_CUDA(cudaStreamSynchronize(stream));
        }
        lr.valid_targets = 0;
        for (int f = 0; f < nf; ++f) lr.valid_targets += (long long)h[2 * f + 1];
        if (lr.valid_targets == 0)
            throw std::runtime_error("ftsp_learn_train: no valid training target (every collected statistic is "
                                     "non-finite or non-positive)");
        if (!lr.trained) {
            // output biases start at the mean target of each field
            std::vector<float> b3(nf);
            for (int f = 0; f < nf; ++f) b3[f] = h[2 * f + 1] > 0.0 ? (float)(h[2 * f] / h[2 * f + 1]) : 0.0f;
            FTSP_CUDA(cudaMemcpyAsync(lr.w.p + mlp::off_b3(nf), b3.data(), sizeof(float) * nf, cudaMemcpyHostToDevice, stream));
        }
        const size_t smem = sizeof(float) * mlp::grad_smem_floats(nf);
        for (int it = 0; it < iterations; ++it) {
            const uint32_t iter = (uint32_t)lr.adam_t;
            auto sample = [=] __device__(int s, float* x, float* t, float* m) {
                const U4 r = philox(U4{(uint32_t)s, iter, 0x4c45524eu, 0u}, s0, s1);
                const size_t i = (size_t)((((uint64_t)r.x << 32) | r.y) % (uint64_t)Vn);
                ft(i, x);
                for (int f = 0; f < nf; ++f) target(i, f, t[f], m[f]);
            };
            auto kern = mlp::k_grad<decltype(sample)>;
            if (it == 0) set_smem(kern, smem);
            kern<<<lr.nb, mlp::GRAD_THREADS, smem, stream>>>(lr.batch, lr.w.p, nf, sample, lr.partial.p, lr.lpart.p);
            mlp::AdamArgs aa{(float)lr.lr, 0.9f, 0.999f, 1e-8f, ++lr.adam_t, 1};
            mlp::k_reduce_adam<<<(lr.np + 255) / 256, 256, 0, stream>>>(lr.np, lr.nb, lr.partial.p, lr.lpart.p, nullptr,
                                                                        lr.loss.p, lr.w.p, lr.m1.p, lr.m2.p, aa);
            launches += 2;
        }
        double l[2] = {0.0, 0.0};
        FTSP_CUDA(cudaMemcpyAsync(l, lr.loss.p, sizeof(l), cudaMemcpyDeviceToHost, stream));
        FTSP_CUDA(cudaStreamSynchronize(stream));
        lr.trained = true;
        lr.last_loss = l[0];
        if (lr.on_use) learn_refresh();
        return l[0];
    }

    void learn_use(bool on) override
    {
        drop_step_graph();
        learn_require();
        if (on && !lr.trained) throw std::runtime_error("ftsp_learn_use: the network has not been trained");
        lr.on_use = on;
        const int v = on ? 1 : 0;
        FTSP_CUDA(cudaMemcpyAsync(&ds->lr_use, &v, sizeof(int), cudaMemcpyHostToDevice, stream));
        if (on) learn_refresh();
        FTSP_CUDA(cudaStreamSynchronize(stream));
    }

    void learn_stats(ftsp_learn_stats* st) override
    {
        pull_scalars();
        std::memset(st, 0, sizeof(*st));
        st->collected = lr.collected;
        st->checks = hs.lr_checks;
        st->fallbacks = hs.lr_fallbacks;
        st->residual_learned = hs.lres[0];
        st->residual_analytic = hs.lres[1];
        st->residual_learned_sum = hs.lres_sum[0];
        st->residual_analytic_sum = hs.lres_sum[1];
        st->loss = lr.last_loss;
        st->iterations = lr.adam_t;
        st->using_learned = lr.on_use && hs.lr_use ? 1 : 0;
        st->n_params = lr.np;
        st->valid_targets = lr.valid_targets;
    }

    int learn_weights(float* out, int n, bool set) override
    {
        drop_step_graph();
        learn_require();
        if (!out) return lr.np;
        if (n != lr.np) throw std::runtime_error("learned weights: expected " + std::to_string(lr.np) + " floats");
        if (set) {
            FTSP_CUDA(cudaMemcpyAsync(lr.w.p, out, sizeof(float) * n, cudaMemcpyHostToDevice, stream));
            lr.trained = true;
            if (lr.on_use) learn_refresh();
        } else {
            FTSP_CUDA(cudaMemcpyAsync(out, lr.w.p, sizeof(float) * n, cudaMemcpyDeviceToHost, stream));
        }
        FTSP_CUDA(cudaStreamSynchronize(stream));
        return lr.np;
    }

    // Loss and gradient of the network at the current weights on caller
    // samples (x: n x 6 features, t and m: n x nout targets and weights),
    // through the training kernels.
    double learn_grad(const float* x, const float* t, const float* m, int n, float* grad) override
    {
        learn_require();
        if (n < 1) throw std::runtime_error("learn_grad: no samples");
        const int nf = lr.nout;
        Buf<float> dx, dt, dm, part, g;
        Buf<double> lp, lo;
        const int nb = (n + mlp::GRAD_THREADS - 1) / mlp::GRAD_THREADS;
        dx.alloc((size_t)n * mlp::NIN); dt.alloc((size_t)n * nf); dm.alloc((size_t)n * nf);
        part.alloc((size_t)nb * lr.np); g.alloc(lr.np); lp.alloc(2 * (size_t)nb); lo.alloc(2);
        FTSP_CUDA(cudaMemcpyAsync(dx.p, x, sizeof(float) * n * mlp::NIN, cudaMemcpyHostToDevice, stream));
        FTSP_CUDA(cudaMemcpyAsync(dt.p, t, sizeof(float) * n * nf, cudaMemcpyHostToDevice, stream));
        FTSP_CUDA(cudaMemcpyAsync(dm.p, m, sizeof(float) * n * nf, cudaMemcpyHostToDevice, stream));
        const float* X = dx.p;
        const float* Tt = dt.p;
        const float* Mm = dm.p;
        auto sample = [=] __device__(int s, float* xx, float* tt, float* mm) {
            for (int k = 0; k < mlp::NIN; ++k) xx[k] = X[(size_t)s * mlp::NIN + k];
            for (int f = 0; f < nf; ++f) {
                tt[f] = Tt[(size_t)s * nf + f];
                mm[f] = Mm[(size_t)s * nf + f];
            }
        };
        const size_t smem = sizeof(float) * mlp::grad_smem_floats(nf);
        auto kern = mlp::k_grad<decltype(sample)>;
        set_smem(kern, smem);
        kern<<<nb, mlp::GRAD_THREADS, smem, stream>>>(n, lr.w.p, nf, sample, part.p, lp.p);
        mlp::AdamArgs aa{0.0f, 0.9f, 0.999f, 1e-8f, 1, 0};
        mlp::k_reduce_adam<<<(lr.np + 255) / 256, 256, 0, stream>>>(lr.np, nb, part.p, lp.p, g.p, lo.p, nullptr, nullptr, nullptr, aa);
        double l[2];
        FTSP_CUDA(cudaMemcpyAsync(grad, g.p, sizeof(float) * lr.np, cudaMemcpyDeviceToHost, stream));
        FTSP_CUDA(cudaMemcpyAsync(l, lo.p, sizeof(l), cudaMemcpyDeviceToHost, stream));
        FTSP_CUDA(cudaStreamSynchronize(stream));
        dx.release(); dt.release(); dm.release(); part.release(); g.release(); lp.release(); lo.release();
        return l[0];
    }

    // ---- launch helpers ----
    // bpe: algorithmic bytes per element (fields read + written), recorded
    // as "field_elementwise" / "field_reduce" when profiling, so that the
    // bytes of a whole step are known (0: not counted, set-up work only)
    template <class F>
    void foreach(size_t n, F f, double bpe = 0.0)
    {
        const int threads = 256;
        const int blocks = (int)std::min<size_t>((n + threads - 1) / threads, 148 * 16);
        cudaEvent_t ev = bpe > 0.0 ? prof_begin() : nullptr;
        launch_pass(k_foreach<F>, dim3(std::max(1, blocks)), threads, 0, n, f);
        ++launches;
        prof_end(ev, "field_elementwise", bpe * (double)n);
    }

    // Blocks of kernel k resident at once on the current device (one wave),
    // at most RED_BLOCKS.
    template <class Kern>
    static int wave_blocks(Kern k, int threads, size_t smem)
    {
        int per_sm = 0, dev = 0, sms = 0;
        FTSP_CUDA(cudaGetDevice(&dev));
        FTSP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem));
        FTSP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        if (per_sm <= 0 || sms <= 0) return RED_BLOCKS;   // no answer: the largest grid
        return std::min(RED_BLOCKS, per_sm * sms);
    }

    // Reduce K channels over n items into out[0..K) (device memory).
    template <int K, bool MAX = false, class F>
    void reduce(size_t n, F f, double* out, double bpe = 0.0)
    {
        cudaEvent_t ev = bpe > 0.0 ? prof_begin() : nullptr;
        // one wave: as many blocks as are resident at once on this device (the
        // kernel's registers decide), at most RED_BLOCKS; fixed per kernel and
        // device, so the summation order is too
        static int grid_of[64] = {};
        int dev = 0;
        FTSP_CUDA(cudaGetDevice(&dev));
        int& grid = grid_of[dev & 63];
        if (grid == 0) grid = wave_blocks(k_reduce<K, MAX, F>, RED_THREADS, 0);
        launch_pass(k_reduce<K, MAX, F>, dim3(grid), RED_THREADS, 0, n, f, (double*)part.p);
        launch_pass(k_combine<MAX>, dim3(K), COMBINE_THREADS, 0, (const double*)part.p, grid, (int)K, out);
        launches += 2;
        prof_end(ev, "field_reduce", bpe * (double)n);
    }

    // Batched in-place (or out-of-place from per-field sources) 3-D FFT of nf
    // contiguous fields of dst.  src[f] (optional) gives the input of field f.
    // ---- pass launchers: compile-time kernels for the production lengths
    // (32, 64, 128), runtime-plan kernels for every other 2/3/5-smooth grid ----
    template <int N> static constexpr bool plane_ct_ok() { return F32 ? (N == 32 || N == 64 || N == 128) : (N == 32 || N == 64); }

    // Launches a pass kernel with programmatic dependent launch (the kernel
    // waits for its predecessor with griddepcontrol.wait).
    bool use_pdl = true;
    template <class K, class... Args>
    void launch_pass(K kernel, dim3 grid, int threads, size_t smem, Args... args)
    {
        if (!use_pdl) {
            kernel<<<grid, threads, smem, stream>>>(args...);
            return;
        }
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = grid;
        cfg.blockDim = dim3(threads);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        FTSP_CUDA(cudaLaunchKernelEx(&cfg, kernel, args...));
    }

    template <int N, int S1, int S2, class Op>
    void plane_ct(const V* src, V* dst, int nf, const Op& op)
    {
        constexpr int E = F32 ? (N >= 128 ? 16 : 16) : (N >= 64 ? 16 : 8);
        constexpr int NT = N * N / E;
        const size_t smem = std::max(sizeof(V) * (size_t)(N * (N + 1) + N), (size_t)4096);
        // field loads (one value per point) only: wider operators keep their batched loads
        if constexpr (S1 == 0 && S2 != 0 && sizeof(typename Op::Pre) == sizeof(V) && plane_fused_ok<N, RMAX, NT, E>()) {
            if (fused_plane) {
                auto k = k_plane_load_fused<T, N, RMAX, NT, E, S2, Op>;
                set_smem(k, smem);
                launch_pass(k, dim3(c.m1, nf), NT, smem, dst, (size_t)V_, (const V*)tw3.p, op);
                ++launches;
                return;
            }
        }
        if constexpr (S1 != 0 && S2 != 0 && F32 && N == 128 && NT == 1024 && op_loads<Op>::value <= 1) {
            if (zreg_plane) {
                auto k = k_plane_zreg<T, S1, S2, Op>;
                // tile of 128 x ZREG_P values, the twiddles, the [t][i] and [t][b] twiddle tables
                const size_t zsmem = sizeof(V) * ((size_t)128 * ZREG_P + 128 + 128 + 128);
                set_smem(k, zsmem);
                launch_pass(k, dim3(c.m1, nf), NT, zsmem, src, dst, (size_t)V_, (const V*)tw3.p, op);
                ++launches;
                return;
            }
        }
        if constexpr (S1 != 0 && S2 != 0 && plane_fused_ok<N, RMAX, NT, E>()) {
            if (fused_plane) {
                auto k = k_plane_fused<T, N, RMAX, NT, E, S1, S2, Op>;
                set_smem(k, smem);
                launch_pass(k, dim3(c.m1, nf), NT, smem, src, dst, (size_t)V_, (const V*)tw3.p, op);
                ++launches;
                return;
            }
        }
        auto k = k_plane_ct<T, N, RMAX, NT, E, S1, S2, Op>;
        set_smem(k, smem);
        launch_pass(k, dim3(c.m1, nf), NT, smem, src, dst, (size_t)V_, (const V*)tw3.p, op);
        ++launches;
    }

    template <int S1, int S2, class Op>
    void plane(const V* src, V* dst, int nf, const Op& op)
    {
        if (c.m2 == c.m3) {
            if constexpr (plane_ct_ok<128>())
                if (c.m3 == 128) return plane_ct<128, S1, S2>(src, dst, nf, op);
            if constexpr (plane_ct_ok<64>())
                if (c.m3 == 64) return plane_ct<64, S1, S2>(src, dst, nf, op);
            if constexpr (plane_ct_ok<32>())
                if (c.m3 == 32) return plane_ct<32, S1, S2>(src, dst, nf, op);
        }
        auto kp = k_plane<T, EP, S1, S2, Op>;
        set_smem(kp, plane_smem);
        kp<<<dim3(c.m1, nf), plane_threads, plane_smem, stream>>>(pg, src, dst, V_, tw2.p, tw3.p, op);
        ++launches;
    }

    template <int DIM, int N, int S1, int S2, class Op>
    void strided_ct(const V* src, V* dst, int nf, const Op& op)
    {
        constexpr int E = F32 ? 16 : 8;
        constexpr int NT = N * WCT / E;
        const size_t smem = std::max(sizeof(V) * (size_t)(N * WCT + N), (size_t)4096);
        const int outer = DIM == 1 ? c.m1 : c.m2;
        // field loads (one value per point) only: wider operators keep their batched loads
        if constexpr (S1 == 0 && S2 != 0 && sizeof(typename Op::Pre) == sizeof(V) && strided_fused_ok<N, WCT, RMAX, NT, E>()) {
            if (fused_strided) {
                auto k = k_strided_load_fused<T, N, WCT, DIM, RMAX, NT, E, S2, Op>;
                set_smem(k, smem);
                launch_pass(k, dim3(outer * (c.m3 / WCT), nf), NT, smem, c.m2, c.m3, dst, (size_t)V_,
                            (const V*)(DIM == 1 ? tw2.p : tw1.p), op);
                ++launches;
                return;
            }
        }
        if constexpr (S1 != 0 && S2 != 0 && strided_fused_ok<N, WCT, RMAX, NT, E>()) {
            if (fused_strided) {
                auto k = k_strided_fused<T, N, WCT, DIM, RMAX, NT, E, S1, S2, Op>;
                set_smem(k, smem);
                launch_pass(k, dim3(outer * (c.m3 / WCT), nf), NT, smem, c.m2, c.m3, src, dst, (size_t)V_,
                            (const V*)(DIM == 1 ? tw2.p : tw1.p), op);
                ++launches;
                return;
            }
        }
        if constexpr (op_has_src<Op>::value) {
            throw std::runtime_error("pencil op with a source map needs the fused pencil pass");
        } else {
            auto k = k_strided_ct<T, N, WCT, DIM, RMAX, NT, E, S1, S2, Op>;
            set_smem(k, smem);
            launch_pass(k, dim3(outer * (c.m3 / WCT), nf), NT, smem, c.m2, c.m3, src, dst, (size_t)V_,
                        (const V*)(DIM == 1 ? tw2.p : tw1.p), op);
            ++launches;
        }
    }

    bool strided_is_ct(int n) const { return c.m3 % WCT == 0 && (n == 32 || n == 64 || n == 128); }

    // the x pass of length n runs k_strided_fused (both transforms in one pass)
    template <int N>
    static constexpr bool x_fused_ct()
    {
        constexpr int E = F32 ? 16 : 8;
        return strided_fused_ok<N, WCT, RMAX, N * WCT / E, E>();
    }
    bool x_fused(int n) const
    {
        if (!fused_strided || !strided_is_ct(n)) return false;
        return n == 128 ? x_fused_ct<128>() : n == 64 ? x_fused_ct<64>() : x_fused_ct<32>();
    }
    // the density evaluation with its k-space factors inside x-pencil passes:
    // one interaction mode, one monomer type, every ion smeared like the beads
    bool eval_fused_ok() const { return plane_ok && c.nm == 1 && c.M == 1 && ion_common && x_fused(c.m1); }

    template <int DIM, int S1, int S2, class Op>
    void strided(const V* src, V* dst, int nf, const Op& op)
    {
        const int n = DIM == 1 ? c.m2 : c.m1;
        if constexpr (DIM == 0 || !F32) {
            if (strided_is_ct(n)) {
                if (n == 128) return strided_ct<DIM, 128, S1, S2>(src, dst, nf, op);
                if (n == 64) return strided_ct<DIM, 64, S1, S2>(src, dst, nf, op);
                return strided_ct<DIM, 32, S1, S2>(src, dst, nf, op);
            }
        }
        if constexpr (op_has_src<Op>::value) {
            throw std::runtime_error("pencil op with a source map needs the fused pencil pass");
        } else {
            const LineGeom& g = DIM == 1 ? gy : gx;
            auto k = k_strided<T, EL, DIM, S1, S2, Op>;
            const size_t smem = DIM == 1 ? y_smem : x_smem;
            set_smem(k, smem);
            const int outer = DIM == 1 ? c.m1 : c.m2;
            k<<<dim3(outer * (c.m3 / g.W), nf), DIM == 1 ? y_threads : x_threads, smem, stream>>>(g, src, dst, V_,
                                                                                                DIM == 1 ? tw2.p : tw1.p, op);
            ++launches;
        }
    }

    template <int S1, int S2, class Op>
    void zline(const V* src, V* dst, int nf, const Op& op)
    {
        if constexpr (!F32) {
            if (c.m3 == 128 && (c.m1 * c.m2) % 16 == 0) {
                constexpr int N = 128, BR = 16, E = 8, NT = BR * N / E;
                auto k = k_zline_ct<T, N, BR, RMAX, NT, E, S1, S2, Op>;
                const size_t smem = sizeof(V) * (size_t)(BR * (N + 1) + N);
                set_smem(k, smem);
                k<<<dim3(c.m1 * c.m2 / BR, nf), NT, smem, stream>>>(c.m2, src, dst, V_, tw3.p, op);
                ++launches;
                return;
            }
        }
        auto k = k_zline<T, EL, S1, S2, Op>;
        set_smem(k, z_smem);
        k<<<dim3(c.m1 * c.m2 / gz.B, nf), z_threads, z_smem, stream>>>(gz, src, dst, V_, tw3.p, op);
        ++launches;
    }

    // Batched in-place (or out-of-place from per-field sources) 3-D FFT of nf
    // contiguous fields of dst.  src[f] (optional) gives the input of field f.
    template <int S>
    void fft3(V* dst, int nf, const V* const* src = nullptr)
    {
        using OpLoad = OpLoadN<T>;
        if (nf > 16) throw std::runtime_error("fft3: too many fields in one batch");
        OpLoad in{};
        for (int f = 0; f < nf; ++f) in.s[f] = src ? src[f] : dst + (size_t)f * V_;
        in.fs = V_;
        OpLoad self{};
        for (int f = 0; f < nf; ++f) self.s[f] = dst + (size_t)f * V_;
        self.fs = V_;
        cudaEvent_t ev = prof_begin();
        if (plane_ok) {
            plane<0, S>(nullptr, dst, nf, in);
        } else {
            zline<0, S>(nullptr, dst, nf, in);
            strided<1, 0, S>(nullptr, dst, nf, self);
        }
        strided<0, 0, S>(nullptr, dst, nf, self);
        // two passes (three without the plane pass), each reading and writing every field
        prof_end(ev, "field_fft", (plane_ok ? 4.0 : 6.0) * nf * sizeof(V) * (double)V_);
    }

    // Real-space pass of one segment: [inverse S1] op [forward S2] with the
    // propagator op.  Plane pass when the plane fits, else y / z-line / y.
    static const char* kind_name(int k)
    {
        static const char* n[] = {"fwd_start", "fwd_mid", "fwd_last", "fwd_single", "bwd_start", "bwd_mid", "bwd_last", "bwd_single"};
        return n[k];
    }
    // algorithmic bytes of one real-space segment pass (complex elements moved per grid point)
    static int seg_units(int k, bool charged)
    {
        switch (k) {
        case FWD_START: return 3;                      // E, q store, G
        case FWD_MID: return 4;                        // H, E, q store, G
        case FWD_LAST: return 3;                       // H, E, q store
        case FWD_SINGLE: return 2;                     // E, q store
        case BWD_START: return 5 + (charged ? 2 : 0);  // E, qF, rho rmw, (rho_c rmw), G
        case BWD_MID: return 6 + (charged ? 2 : 0);    // H, qF, E, rho rmw, (rho_c rmw), G
        case BWD_LAST: return 4 + (charged ? 2 : 0);   // H, qF, rho rmw, (rho_c rmw)
        default: return 3 + (charged ? 2 : 0);         // qF, rho rmw, (rho_c rmw)
        }
    }

    template <int S1, int S2, int KIND>
    void seg_pass(const V* src, V* dst, const OpProp<T, KIND>& op)
    {
        cudaEvent_t ev = prof_begin();
        seg_pass_launch<S1, S2, KIND>(src, dst, op);
        prof_end(ev, std::string(plane_ok ? "plane_" : "zline_") + kind_name(KIND),
                 (double)(seg_units(KIND, op.rho_charge != nullptr) - (KIND == FWD_START && op.store_u ? 1 : 0)) *
                     sizeof(V) * (double)V_);   // u(0) = 1 is not stored
    }

    template <int S1, int S2, int KIND>
    void seg_pass_launch(const V* src, V* dst, const OpProp<T, KIND>& op)
    {
        using OpLoadOne = ftsp::OpLoadOne<T>;
        if (plane_ok) {
            plane<S1, S2>(src, dst, 1, op);
            return;
        }
        if (S1 != 0) strided<1, 0, S1>(nullptr, const_cast<V*>(src), 1, OpLoadOne{src});   // y-lines, in place
        zline<S1, S2>(src, dst, 1, op);
        if (S2 != 0) strided<1, 0, S2>(nullptr, dst, 1, OpLoadOne{dst});                    // y-lines, in place
    }

    int seg_pass_ctas() const
    {
        if (plane_ok) return c.m1;
        if (!F32 && c.m3 == 128 && (c.m1 * c.m2) % 16 == 0) return c.m1 * c.m2 / 16;
        return c.m1 * c.m2 / gz.B;
    }
    int x_ctas() const { return c.m2 * (c.m3 / (strided_is_ct(c.m1) ? WCT : gx.W)); }

    template <int S1, int S2, bool FWD, bool STRESS>
    void bond_pass(const V* src, V* dst, const OpBond<T, FWD, STRESS>& op)
    {
        cudaEvent_t ev = prof_begin();
        strided<0, S1, S2>(src, dst, 1, op);
        // G in, H out, plus the stored/read forward spectrum when the stress is on
        const bool extra = FWD ? op.Fstore != nullptr : STRESS;
        prof_end(ev, std::string("bond_") + (FWD ? "fwd" : "bwd") + (extra ? (FWD ? "_storeF" : "_stress") : ""),
                 (double)(2 + (extra ? 1 : 0)) * sizeof(V) * (double)V_);
    }

    // ---- chain propagators of one species; densities accumulate into dB ----
    void solve_species(int isp, bool stress)
    {
        const Species& s = c.sp[isp];
        const int N = s.N;
        const size_t Vn = V_;
        const int M = c.M;
        auto Ec = [&](int seg) { return E.p + (size_t)s.cls[seg] * Vn; };
        auto qf = [&](int seg) { return qF.p + (size_t)seg * Vn; };
        double2* factor = &ds->factor[isp];
        double* qpart = part.p;
        // renormalisation bookkeeping (see Renorm in passes.cuh)
        const int nparts = seg_pass_ctas();
        const size_t pslot = (size_t)std::max(c.m1, c.m1 * c.m2);
        auto pm = [&](int s) { return pmax.p + (size_t)(s & 1) * pslot; };
        auto rn = [&](int s) {
            Renorm r{};
            r.eF = expo.p;
            r.eB = expo.p + Nmax;
            r.nparts = nparts;
            r.s = s;
            r.N = N;
            r.pmax_cur = pm(s);
            r.pmax_prev = pm(s + 1);   // the pass before: segment s-1 (forward) or s+1 (backward), other parity
            return r;
        };
        // ---- forward sweep ----
        // a mirror-symmetric species stores u = q / E and needs no backward sweep
        const bool pairs = chain_sym && sym[isp].ok;
        qF_holds_u = pairs ? isp : -1;
        if (N == 1) {
            OpProp<T, FWD_SINGLE> op{};
            op.E = Ec(0); op.qstore = qf(0); op.partial = reinterpret_cast<double2*>(qpart); op.rn = rn(0);
            seg_pass<0, 0, FWD_SINGLE>(nullptr, nullptr, op);
        } else {
            OpProp<T, FWD_START> op0{};
            op0.E = Ec(0); op0.qstore = qf(0); op0.rn = rn(0); op0.store_u = pairs;
            seg_pass<0, -1, FWD_START>(nullptr, G.p, op0);
            for (int b = 0; b < N - 1; ++b) {
                OpBond<T, true, false> ob{};
                ob.Fstore = stress ? Fst.p + (size_t)b * Vn : nullptr;
                set_bond(ob, s.bcls[b]);
                bond_pass<-1, +1, true, false>(G.p, H.p, ob);
                if (b + 1 < N - 1) {
                    OpProp<T, FWD_MID> op{};
                    op.E = Ec(b + 1); op.qstore = qf(b + 1); op.rn = rn(b + 1); op.store_u = pairs;
                    seg_pass<+1, -1, FWD_MID>(H.p, G.p, op);
                } else {
                    OpProp<T, FWD_LAST> op{};
                    op.E = Ec(b + 1); op.qstore = qf(b + 1); op.partial = reinterpret_cast<double2*>(qpart);
                    op.rn = rn(b + 1); op.store_u = pairs;
                    seg_pass<+1, 0, FWD_LAST>(H.p, nullptr, op);
                }
            }
        }
        // ---- Q (of the stored, scaled qF[N-1]) and the species factor (n/V)/Q ----
        {
            const int cnt = seg_pass_ctas();
            const double nv = s.nc / c.volume;
            const double invV = 1.0 / (double)Vn;
            DevScal* d = ds;
            const int* eF = expo.p;
            const int last = N - 1;
            k_combine<false><<<2, COMBINE_THREADS, 0, stream>>>(qpart, cnt, 2, reinterpret_cast<double*>(&d->Q[isp]));
            k_foreach<<<1, 32, 0, stream>>>(1, [=] __device__(size_t) {
                const double2 Qs = dscale(d->Q[isp], invV);
                d->factor[isp] = dscale(dinv(Qs), nv);
                d->Q[isp] = make_double2(ldexp(Qs.x, eF[last]), ldexp(Qs.y, eF[last]));   // true Q
            });
            launches += 2;
        }
        if (pairs) {
            pair_passes(isp, stress);
            return;
        }
        // ---- backward sweep (opposite sign convention: B' = B(-k)) ----
        auto rho_of = [&](int seg) { return dB.p + (size_t)s.type[seg] * Vn; };
        // species whose charge density folds into its type channel after the
        // sweep (charge_fold) accumulate no separate charge density
        const bool folded = fold_type[isp] >= 0;
        auto rchg = [&](int seg) -> V* {
            return (c.elec && s.charge[seg] != 0.0 && !folded) ? dB.p + (size_t)M * Vn : nullptr;
        };
        if (N == 1) {
            OpProp<T, BWD_SINGLE> op{};
            op.qread = qf(0); op.rho_type = rho_of(0); op.rho_charge = rchg(0); op.z = (T)s.charge[0]; op.factor = factor;
            op.rn = rn(0);
            seg_pass<0, 0, BWD_SINGLE>(nullptr, nullptr, op);
            return;
        }
        {
            OpProp<T, BWD_START> op{};
            op.E = Ec(N - 1); op.qread = qf(N - 1); op.rho_type = rho_of(N - 1); op.rho_charge = rchg(N - 1);
            op.z = (T)s.charge[N - 1]; op.factor = factor; op.rn = rn(N - 1);
            seg_pass<0, +1, BWD_START>(nullptr, G.p, op);
        }
        for (int b = N - 2; b >= 0; --b) {
            if (stress) {
                OpBond<T, false, true> ob{};
                ob.Fread = Fst.p + (size_t)b * Vn;
                ob.factor = factor;
                ob.partial = reinterpret_cast<double2*>(spart.p);
                ob.b2 = s.bond[b] * s.bond[b];
                ob.eF = expo.p;
                ob.eB = expo.p + Nmax;
                ob.s = b;
                ob.N = N;
                set_bond(ob, s.bcls[b]);
                bond_pass<+1, -1, false, true>(G.p, H.p, ob);
            } else {
                OpBond<T, false, false> ob{};
                set_bond(ob, s.bcls[b]);
                bond_pass<+1, -1, false, false>(G.p, H.p, ob);
            }
            if (b > 0) {
                OpProp<T, BWD_MID> op{};
                op.E = Ec(b); op.qread = qf(b); op.rho_type = rho_of(b); op.rho_charge = rchg(b);
                op.z = (T)s.charge[b]; op.factor = factor; op.rn = rn(b);
                seg_pass<-1, +1, BWD_MID>(H.p, G.p, op);
            } else {
                OpProp<T, BWD_LAST> op{};
                op.qread = qf(0); op.rho_type = rho_of(0); op.rho_charge = rchg(0);
                op.z = (T)s.charge[0]; op.factor = factor; op.rn = rn(0);
                seg_pass<-1, 0, BWD_LAST>(H.p, nullptr, op);
            }
        }
    }

    // ---- mirror-symmetric species: densities and stress from the forward sweep ----
    void pair_passes(int isp, bool stress)
    {
        const Species& s = c.sp[isp];
        const SymTables& t = sym[isp];
        const size_t Vn = V_;
        const int threads = 256;
        const double2* factor = &ds->factor[isp];
        bool charged = false;
        for (double q : s.charge) charged |= q != 0.0;
        V* rc = (c.elec && charged && fold_type[isp] < 0) ? dB.p + (size_t)c.M * Vn : nullptr;
        if (stress) {
            const size_t sm = pair_smem(t.stress.npairs, t.stress.nruns, threads);
            // with one species nothing else reads the spectra or writes the
            // stress partials before the record is finalised: run the kernel
            // beside the rest of the evaluation (joined at its end)
            if (c.sp.size() == 1 && !profiling) {
                if (!aux) {
                    FTSP_CUDA(cudaStreamCreateWithFlags(&aux, cudaStreamNonBlocking));
                    FTSP_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
                    FTSP_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
                }
                FTSP_CUDA(cudaEventRecord(ev_fork, stream));
                FTSP_CUDA(cudaStreamWaitEvent(aux, ev_fork, 0));
                k_pair_stress<T><<<x_ctas(), threads, sm, aux>>>(
                    c.m1, c.m2, c.m3, t.stress, (const V*)Fst.p, (const T*)phi.p, (const double*)kx.p,
                    (const double*)ky.p, (const double*)kz.p, (const int*)expo.p, s.N, factor,
                    reinterpret_cast<double2*>(spart.p));
                FTSP_CUDA(cudaGetLastError());
                aux_pending = true;
            } else {
                cudaEvent_t ev = prof_begin();
                launch_pass(k_pair_stress<T>, dim3(x_ctas()), threads, sm, c.m1, c.m2, c.m3, t.stress,
                            (const V*)Fst.p, (const T*)phi.p, (const double*)kx.p, (const double*)ky.p,
                            (const double*)kz.p, (const int*)expo.p, s.N, factor, reinterpret_cast<double2*>(spart.p));
                prof_end(ev, "pair_stress", (double)(s.N - 1) * sizeof(V) * (double)Vn);
            }
            ++launches;
        }
        {
            cudaEvent_t ev = prof_begin();
            constexpr int PT = PairVec<T>::PT;
            const size_t smem = pair_smem(t.dens.npairs, t.dens.nruns, threads);
            if (Vn % PT == 0) {   // PT consecutive points per thread, 16-byte loads
                const int blocks = (int)std::min<size_t>((Vn / PT + threads - 1) / threads, (size_t)RED_BLOCKS);
                launch_pass(k_pair_density_vec<T>, dim3(blocks), threads, smem, Vn, t.dens, (const V*)qF.p,
                            (const V*)E.p, (const int*)expo.p, s.N, factor, dB.p, rc);
            } else {
                const int blocks = (int)std::min<size_t>((Vn + threads - 1) / threads, (size_t)RED_BLOCKS);
                launch_pass(k_pair_density<T>, dim3(blocks), threads, smem, Vn, t.dens, (const V*)qF.p,
                            (const V*)E.p, (const int*)expo.p, s.N, factor, dB.p, rc);
            }
            ++launches;
            // stored u fields, one class table per run, channel read-modify-writes
            const int units = (s.N - 1) + t.dens.nruns + 2 * t.dens_channels + (rc ? 2 : 0);
            prof_end(ev, "pair_density", (double)units * sizeof(V) * (double)Vn);
        }
    }

    // A species is mirror-symmetric when cls[s] == cls[N-1-s] for every
    // segment and bond b matches bond N-2-b in class and length.  Its pair
    // tables: density pairs (s, N-1-s), s <= N-1-s, ordered by (type, class)
    // and grouped in runs of one class; stress pairs (b, N-2-b), b <= N-2-b,
    // grouped by bond class.  At most 1024 pairs (N <= 2048) so that the
    // tables fit the kernels' shared memory.
    void plan_symmetry()
    {
        const int S = (int)c.sp.size();
        sym.assign(S, SymTables{});
        std::vector<int2> ix;
        std::vector<double> wt;
        std::vector<PairRun> runs;
        struct Off {
            size_t p0, r0;
        };
        std::vector<Off> doff(S), soff(S);
        for (int k = 0; k < S; ++k) {
            const Species& sp = c.sp[k];
            const int N = sp.N;
            bool ok = N >= 2 && N <= 2048;
            for (int i = 0; ok && i < N; ++i) ok = sp.cls[i] == sp.cls[N - 1 - i];
            for (int b = 0; ok && b + 1 < N; ++b)
                ok = sp.bcls[b] == sp.bcls[N - 2 - b] && sp.bond[b] == sp.bond[N - 2 - b];
            if (!ok) continue;
            SymTables& t = sym[k];
            t.ok = true;
            // density pairs
            std::vector<int> seg;
            for (int i = 0; 2 * i <= N - 1; ++i) seg.push_back(i);
            std::stable_sort(seg.begin(), seg.end(), [&](int a, int b) {
                return std::make_pair(sp.type[a], sp.cls[a]) < std::make_pair(sp.type[b], sp.cls[b]);
            });
            doff[k] = Off{ix.size(), runs.size()};
            std::vector<int> seen(c.M, 0);
            for (int j = 0; j < (int)seg.size(); ++j) {
                const int i = seg[j];
                if (j == 0 || runs.back().cls != sp.cls[i])
                    runs.push_back(PairRun{j, j, sp.cls[i], sp.type[i], sp.charge[i]});
                runs.back().j1 = j + 1;
                ix.push_back(make_int2(i, N - 1 - i));
                wt.push_back(i < N - 1 - i ? 2.0 : 1.0);
                t.dens_channels += seen[sp.type[i]] ? 0 : 1;
                seen[sp.type[i]] = 1;
            }
            t.dens.npairs = (int)seg.size();
            t.dens.nruns = (int)(runs.size() - doff[k].r0);
            // stress pairs
            std::vector<int> bd;
            for (int b = 0; 2 * b <= N - 2; ++b) bd.push_back(b);
            std::stable_sort(bd.begin(), bd.end(), [&](int a, int b) { return sp.bcls[a] < sp.bcls[b]; });
            soff[k] = Off{ix.size(), runs.size()};
            for (int j = 0; j < (int)bd.size(); ++j) {
                const int b = bd[j];
                if (j == 0 || runs.back().cls != sp.bcls[b]) runs.push_back(PairRun{j, j, sp.bcls[b], 0, 0.0});
                runs.back().j1 = j + 1;
                ix.push_back(make_int2(b, N - 2 - b));
                wt.push_back(sp.bond[b] * sp.bond[b] * (b < N - 2 - b ? 1.0 : 0.5));
            }
            t.stress.npairs = (int)bd.size();
            t.stress.nruns = (int)(runs.size() - soff[k].r0);
        }
        if (ix.empty()) return;
        pair_ix.alloc(ix.size());
        pair_wt.alloc(wt.size());
        pair_run.alloc(runs.size());
        FTSP_CUDA(cudaMemcpy(pair_ix.p, ix.data(), sizeof(int2) * ix.size(), cudaMemcpyHostToDevice));
        FTSP_CUDA(cudaMemcpy(pair_wt.p, wt.data(), sizeof(double) * wt.size(), cudaMemcpyHostToDevice));
        FTSP_CUDA(cudaMemcpy(pair_run.p, runs.data(), sizeof(PairRun) * runs.size(), cudaMemcpyHostToDevice));
        for (int k = 0; k < S; ++k) {
            if (!sym[k].ok) continue;
            SymTables& t = sym[k];
            t.dens.pair = pair_ix.p + doff[k].p0;
            t.dens.weight = pair_wt.p + doff[k].p0;
            t.dens.run = pair_run.p + doff[k].r0;
            t.stress.pair = pair_ix.p + soff[k].p0;
            t.stress.weight = pair_wt.p + soff[k].p0;
            t.stress.run = pair_run.p + soff[k].r0;
        }
    }

    template <class OB>
    void set_bond(OB& ob, int bc)
    {
        const int sum_m = c.m1 + c.m2 + c.m3;
        const T* base = phi.p + (size_t)bc * sum_m;
        ob.phix = base;
        ob.phiy = base + c.m1;
        ob.phiz = base + c.m1 + c.m2;
        ob.kx = kx.p; ob.ky = ky.p; ob.kz = kz.p;
        ob.invV = (T)(1.0 / (double)V_);
    }

    // ---- charge densities of single-class species ----
    // A species whose segments all share one type t and one valence z, and
    // which is the only species with segments of type t, has the charge
    // density z rho_t of its type channel.  Its backward sweep then skips the
    // read-modify-write of the charge accumulator (two of the eight complex
    // values per point that the backward segment pass moves), and one pass
    // after all sweeps adds z rho_t to the charge channel.  For z = +-1, +-2
    // (powers of two) the result is bit-identical to accumulating it.
    std::vector<int> fold_type;
    std::vector<double> fold_z;

    void plan_charge_fold()
    {
        const int S = (int)c.sp.size();
        fold_type.assign(S, -1);
        fold_z.assign(S, 0.0);
        if (!c.elec) return;
        std::vector<int> users(c.M, 0);
        for (const auto& sp : c.sp) {
            std::vector<int> seen(c.M, 0);
            for (int t : sp.type) seen[t] = 1;
            for (int t = 0; t < c.M; ++t) users[t] += seen[t];
        }
        for (int k = 0; k < S; ++k) {
            const auto& sp = c.sp[k];
            bool one = true;
            for (int i = 1; i < sp.N; ++i) one &= sp.type[i] == sp.type[0] && sp.charge[i] == sp.charge[0];
            if (one && sp.charge[0] != 0.0 && users[sp.type[0]] == 1) {
                fold_type[k] = sp.type[0];
                fold_z[k] = sp.charge[0];
            }
        }
    }

    void charge_fold()
    {
        ClsTab ft{};
        int n = 0;
        for (size_t k = 0; k < fold_type.size(); ++k)
            if (fold_type[k] >= 0 && n < 32) {
                ft.type[n] = fold_type[k];
                ft.z[n] = fold_z[k];
                ++n;
            }
        if (n == 0) return;
        const size_t Vn = V_;
        V* dBp = dB.p;
        const int M = c.M;
        foreach(Vn, [=] __device__(size_t i) {
            V acc = dBp[(size_t)M * Vn + i];
            for (int k = 0; k < n; ++k) acc = cadd(acc, cscale(dBp[(size_t)ft.type[k] * Vn + i], (T)ft.z[k]));
            dBp[(size_t)M * Vn + i] = acc;
        }, (2.0 + n) * sizeof(V));
    }

    // ---- densities at (omega_w, psi_w) ----
    void eval(int which, bool stress)
    {
        const size_t Vn = V_;
        const int nm = c.nm, M = c.M, J = (int)c.ions.size();
        const V* om = which ? omega_bar.p : omega.p;
        const V* ps = which ? psi_bar.p : psi.p;
        const int m1 = c.m1, m2 = c.m2, m3 = c.m3;
        const bool elec = c.elec;
        const bool fx = eval_fused_ok();
        if (fx) {
            // 1-2 fused: yz forward of omega and psi (into the scratch half of
            // kA); one x-pencil pass: x forward, the k-space omega and psi
            // stored in kA, W_type = gamma O Gamma omega / V, psi_s = Gamma
            // psi / V and the psi drift's k^2 psi / (4 pi l_B V) (from psi's
            // transform a second time), x inverse into kB; yz inverse
            cudaEvent_t ev = prof_begin();
            V* kAx = kA.p + (size_t)(nm + 1) * Vn;
            OpLoadN<T> in{};
            in.s[0] = om;
            in.s[1] = ps;
            in.fs = Vn;
            plane<0, -1>(nullptr, kAx, 2, in);
            const double invV = 1.0 / (double)Vn;
            OpKScale<T> op{};
            op.kst = kA.p;
            op.gm = gam.p;
            op.kx = kx.p;
            op.ky = ky.p;
            op.kz = kz.p;
            op.m1 = m1;
            op.m2 = m2;
            op.nst = 2;
            op.src[0] = 0; op.src[1] = 1; op.src[2] = 1; op.src[3] = 3;
            op.lap[2] = 1;
            op.c[0] = make_double2(c.gamma[0].x * c.O[0] * invV, c.gamma[0].y * c.O[0] * invV);
            op.c[1] = make_double2(elec ? invV : 0.0, 0.0);
            op.c[2] = make_double2(elec ? invV / (4.0 * PI * c.lB) : 0.0, 0.0);
            strided<0, -1, +1>(kAx, kB.p, 3, op);
            plane<+1, 0>(kB.p, nullptr, 3, OpStore<T>{kB.p});
            // plane: 2 in, 2 out; pencil: 3 in, 2 + 3 out; plane: 3 in, 3 out
            prof_end(ev, "field_fft", 18.0 * sizeof(V) * (double)Vn);
        }
        // 1. DFT of the mode fields and psi
        if (!fx) {
            std::vector<const V*> src;
            for (int a = 0; a < nm; ++a) src.push_back(om + (size_t)a * Vn);
            src.push_back(ps);
            fft3<-1>(kA.p, nm + 1, src.data());
        }
        // 2. k-space: W_type_s (M), psi_s, ion psi_j (J), all scaled by 1/V
        if (!fx) {
            GCoef co{};
            for (int a = 0; a < nm; ++a)
                for (int al = 0; al < M; ++al)
                    co.g[a * M + al] = make_double2(c.gamma[a].x * c.O[a * M + al], c.gamma[a].y * c.O[a * M + al]);
            const V* kAp = kA.p;
            V* kBp = kB.p;
            const T* gm = gam.p;
            const T* gi = gion.p;
            const int sum_m = m1 + m2 + m3;
            const double invV = 1.0 / (double)Vn;
            const int Jk = ion_common ? 0 : J;   // ion potentials of their own
            foreach(Vn, [=] __device__(size_t i) {
                const int x = (int)(i / ((size_t)m2 * m3));
                const int r = (int)(i - (size_t)x * m2 * m3);
                const int y = r / m3, z = r - y * m3;
                const T G0 = gm[x] * gm[m1 + y] * gm[m1 + m2 + z];
                const double gv = (double)G0 * invV;
                for (int al = 0; al < M; ++al) {
                    double2 w = make_double2(0.0, 0.0);
                    for (int a = 0; a < nm; ++a) w = dadd(w, dmul(to_d(kAp[(size_t)a * Vn + i]), co.g[a * M + al]));
                    kBp[(size_t)al * Vn + i] = from_d<V>(dscale(w, gv));
                }
                const double2 P = to_d(kAp[(size_t)nm * Vn + i]);
                kBp[(size_t)M * Vn + i] = from_d<V>(elec ? dscale(P, gv) : make_double2(0.0, 0.0));
                for (int j = 0; j < Jk; ++j) {
                    const T* t = gi + (size_t)j * sum_m;
                    const double gj = (double)(t[x] * t[m1 + y] * t[m1 + m2 + z]) * invV;
                    kBp[(size_t)(M + 1 + j) * Vn + i] = from_d<V>(elec ? dscale(P, gj) : make_double2(0.0, 0.0));
                }
            }, (double)(c.nm + 1 + c.M + 1 + Jk) * sizeof(V));
        }
        if (!fx) fft3<+1>(kB.p, M + 1 + (ion_common ? 0 : J));
        // 3. class tables exp(-(W_type + i z psi_s)), ion Boltzmann factors, zeroed accumulators
        {
            ClsTab ct{};
            const int ncls = (int)c.cls.size();
            if (ncls > 64) throw std::runtime_error("too many segment classes");
            for (int k = 0; k < ncls; ++k) {
                ct.type[k] = c.cls[k].type;
                ct.z[k] = elec ? c.cls[k].z : 0.0;
            }
            IonTab zi{};
            for (int j = 0; j < J; ++j) zi.z[j] = c.ions[j].z;
            const V* kBp = kB.p;
            V* Ep = E.p;
            V* dBp = dB.p;
            if (ion_common) {
                // the Boltzmann factors exp(-i z_j psi_s) are only summed here
                // (Q_j); the combined ion charge is formed after the sweeps
                // class 0 with constant indices (a single class is the usual case)
                const int t0 = ct.type[0];
                const T z0 = (T)ct.z[0];
                reduce<6>(Vn, [=] __device__(size_t i, double* acc) {
                    const V ps_ = __ldg(kBp + (size_t)M * Vn + i);
                    {
                        V w = __ldg(kBp + (size_t)t0 * Vn + i);
                        if (z0 != T(0)) {
                            w.x += -(ps_.y * z0);
                            w.y += ps_.x * z0;
                        }
                        Ep[i] = cexpT(-w.x, -w.y);
                    }
                    for (int k = 1; k < ncls; ++k) {
                        V w = __ldg(kBp + (size_t)ct.type[k] * Vn + i);
                        const T zz = (T)ct.z[k];
                        if (zz != T(0)) {
                            w.x += -(ps_.y * zz);
                            w.y += ps_.x * zz;
                        }
                        Ep[(size_t)k * Vn + i] = cexpT(-w.x, -w.y);
                    }
                    for (int al = 0; al <= M; ++al) dBp[(size_t)al * Vn + i] = mkc<V>(T(0), T(0));
#pragma unroll
                    for (int j = 0; j < 3; ++j) {   // J <= 3 on this path
                        if (j >= J) break;
                        const T zz = (T)zi.z[j];
                        const V b = cexpT(zz * ps_.y, -zz * ps_.x);
                        acc[2 * j] += (double)b.x;
                        acc[2 * j + 1] += (double)b.y;
                    }
                }, reinterpret_cast<double*>(&ds->Qion[0]), (double)(2 + 2 * c.M + (int)c.cls.size()) * sizeof(V));
                DevScal* d = ds;
                IonTab ic{};
                for (int j = 0; j < J; ++j) ic.nd[j] = c.ions[j].count / c.volume;
                const double invV = 1.0 / (double)Vn;
                k_foreach<<<1, 32, 0, stream>>>((size_t)J, [=] __device__(size_t j) {
                    const double2 Q = dscale(d->Qion[j], invV);
                    d->Qion[j] = Q;
                    d->ion_factor[j] = dscale(dinv(Q), ic.nd[j]);
                });
                ++launches;
            } else {
                foreach(Vn, [=] __device__(size_t i) {
                    const V ps_ = kBp[(size_t)M * Vn + i];
                    for (int k = 0; k < ncls; ++k) {
                        V w = kBp[(size_t)ct.type[k] * Vn + i];
                        const T zz = (T)ct.z[k];
                        if (zz != T(0)) {   // W += psi_s * (0 + i z)  (add_scaled_complex_const)
                            w.x += -(ps_.y * zz);
                            w.y += ps_.x * zz;
                        }
                        Ep[(size_t)k * Vn + i] = cexpT(-w.x, -w.y);
                    }
                    for (int al = 0; al <= M; ++al) dBp[(size_t)al * Vn + i] = mkc<V>(T(0), T(0));
                    for (int j = 0; j < J; ++j) {
                        const V pj = kBp[(size_t)(M + 1 + j) * Vn + i];
                        const T zz = (T)zi.z[j];
                        dBp[(size_t)(M + 1 + j) * Vn + i] = cexpT(zz * pj.y, -zz * pj.x);
                    }
                }, (double)(2 * (c.M + 1 + J) + (int)c.cls.size()) * sizeof(V));
            }
        }
        if (stress) FTSP_CUDA(cudaMemsetAsync(spart.p, 0, sizeof(double) * 12 * (size_t)x_ctas(), stream));
        // 4. chain propagators of every species
        for (int isp = 0; isp < (int)c.sp.size(); ++isp) solve_species(isp, stress);
        if (!fx) charge_fold();
        if (ion_common) {
            // the combined ion charge sum_j z_j (n_j/V)/Q_j exp(-i z_j psi_s)
            // (ion_density_from_psi, common.h:1117-1130, summed over the
            // species before the smoothing, which is common to all of them)
            const V* ps = kB.p + (size_t)M * Vn;
            V* cion = dB.p + (size_t)(M + 1) * Vn;
            IonTab zi{};
            for (int j = 0; j < J; ++j) zi.z[j] = c.ions[j].z;
            const DevScal* d = ds;
            foreach(Vn, [=] __device__(size_t i) {
                const V p = ps[i];
                double2 acc = make_double2(0.0, 0.0);
                for (int j = 0; j < J; ++j) {
                    const T zz = (T)zi.z[j];
                    acc = dadd(acc, dscale(dmul(to_d(cexpT(zz * p.y, -zz * p.x)), d->ion_factor[j]), zi.z[j]));
                }
                cion[i] = from_d<V>(acc);
            }, 2.0 * sizeof(V));
        }
        const int Jd = ion_common ? 1 : J;   // ion fields of the density transform
        if (fx) {
            // 5-7 fused: the raw densities (the folded charge added as the
            // charge density is loaded) and the combined ion charge, yz
            // forward (into kC); one x-pencil pass: x forward, their k-space
            // values stored in dB (the k-space observables read them), times
            // Gamma / V, x inverse (in place); yz inverse
            cudaEvent_t ev = prof_begin();
            OpLoadDensity<T> ld{};
            ld.rho = dB.p;
            ld.Vn = Vn;
            for (size_t k = 0; k < fold_type.size(); ++k)
                if (fold_type[k] >= 0) ld.zf += fold_z[k];   // one type: at most one species folds
            plane<0, -1>(nullptr, kC.p, 3, ld);
            const double invV = 1.0 / (double)Vn;
            OpKScale<T> op{};
            op.kst = dB.p;
            op.gm = gam.p;
            op.kx = kx.p;
            op.ky = ky.p;
            op.kz = kz.p;
            op.m1 = m1;
            op.m2 = m2;
            op.nst = 3;
            for (int f = 0; f < 4; ++f) {
                op.src[f] = f;
                op.c[f] = make_double2(invV, 0.0);
            }
            strided<0, -1, +1>(kC.p, kC.p, 3, op);
            plane<+1, 0>(kC.p, nullptr, 3, OpStore<T>{kC.p});
            // plane: 3 in, 3 out; pencil: 3 in, 3 + 3 out; plane: 3 in, 3 out
            prof_end(ev, "field_fft", 21.0 * sizeof(V) * (double)Vn);
        }
        // 5. DFT of the raw densities and the ion Boltzmann factors (or the combined ion charge)
        if (!fx) fft3<-1>(dB.p, M + 1 + Jd);
        // 6. ion partition functions from the DC bins
        if (J > 0 && !ion_common) {
            DevScal* d = ds;
            const V* dBp = dB.p;
            IonTab ic{};
            for (int j = 0; j < J; ++j) ic.nd[j] = c.ions[j].count / c.volume;
            const double invV = 1.0 / (double)Vn;
            k_foreach<<<1, 32, 0, stream>>>((size_t)J, [=] __device__(size_t j) {
                const double2 Q = dscale(to_d(dBp[(size_t)(M + 1 + j) * Vn]), invV);
                d->Qion[j] = Q;
                d->ion_factor[j] = dscale(dinv(Q), ic.nd[j]);
            });
            ++launches;
        }
        // 7. k-space: smoothed densities, ion charge, psi drift part
        if (!fx) {
            const V* dBp = dB.p;
            const V* kAp = kA.p;
            V* kCp = kC.p;
            const T* gm = gam.p;
            const T* gi = gion.p;
            const double* kxp = kx.p;
            const double* kyp = ky.p;
            const double* kzp = kz.p;
            const int sum_m = m1 + m2 + m3;
            const double invV = 1.0 / (double)Vn;
            const double dpsi_scale = elec ? 1.0 / (4.0 * PI * c.lB) : 0.0;
            IonTab zi{};
            for (int j = 0; j < J; ++j) zi.z[j] = elec ? c.ions[j].z : 0.0;
            const DevScal* d = ds;
            const bool common = ion_common;
            foreach(Vn, [=] __device__(size_t i) {
                const int x = (int)(i / ((size_t)m2 * m3));
                const int r = (int)(i - (size_t)x * m2 * m3);
                const int y = r / m3, z = r - y * m3;
                const double gv = (double)(gm[x] * gm[m1 + y] * gm[m1 + m2 + z]) * invV;
                for (int al = 0; al <= M; ++al) kCp[(size_t)al * Vn + i] = from_d<V>(dscale(to_d(dBp[(size_t)al * Vn + i]), gv));
                double2 ci = make_double2(0.0, 0.0);
                if (common) {   // the combined ion charge, smoothed like the beads
                    ci = dscale(to_d(dBp[(size_t)(M + 1) * Vn + i]), gv);
                } else {
                    for (int j = 0; j < J; ++j) {
                        const T* t = gi + (size_t)j * sum_m;
                        const double gj = (double)(t[x] * t[m1 + y] * t[m1 + m2 + z]) * invV;
                        const double2 f = d->ion_factor[j];
                        ci = dadd(ci, dscale(dmul(to_d(dBp[(size_t)(M + 1 + j) * Vn + i]), f), gj * zi.z[j]));
                    }
                }
                kCp[(size_t)(M + 1) * Vn + i] = from_d<V>(ci);
                const double k2 = kxp[x] * kxp[x] + kyp[y] * kyp[y] + kzp[z] * kzp[z];
                kCp[(size_t)(M + 2) * Vn + i] = from_d<V>(dscale(to_d(kAp[(size_t)nm * Vn + i]), k2 * invV * dpsi_scale));
            }, (double)(2 * c.M + 5 + Jd) * sizeof(V));
        }
        if (!fx) fft3<+1>(kC.p, M + 3);
        // 8. real-space epilogue: rho_p, rho_c, ion densities, raw psi drift (+ its sum)
        {
            const V* kCp = kC.p;
            const V* kBp = kB.p;
            V* rp = rho_p.p;
            V* rc = rho_c.p;
            V* ir = ion_rho.p;
            V* dp = which ? dpsi_bar.p : dpsi.p;
            const V* dk = fx ? kB.p + (size_t)(M + 1) * Vn : kC.p + (size_t)(M + 2) * Vn;   // k^2 psi part
            const DevScal* d = ds;
            IonTab iz{};
            for (int j = 0; j < J; ++j) {
                iz.z[j] = c.ions[j].z;
                iz.nd[j] = c.ions[j].count / c.volume;
            }
            const bool common = ion_common;
            reduce<2>(Vn, [=] __device__(size_t i, double* acc) {
                V sum = mkc<V>(T(0), T(0));
                for (int al = 0; al < M; ++al) sum = cadd(sum, __ldg(kCp + (size_t)al * Vn + i));
                rp[i] = sum;
                const V rcp = __ldg(kCp + (size_t)M * Vn + i);
                const V rci = __ldg(kCp + (size_t)(M + 1) * Vn + i);
                const V rcv = elec ? cadd(rcp, rci) : mkc<V>(T(0), T(0));
                rc[i] = rcv;
                for (int j = 0; j < J; ++j) {
                    if (elec) {
                        const V pj = __ldg(kBp + (size_t)(common ? M : M + 1 + j) * Vn + i);
                        const T zz = (T)iz.z[j];
                        const V b = cexpT(zz * pj.y, -zz * pj.x);
                        ir[(size_t)j * Vn + i] = cmul(b, from_d<V>(d->ion_factor[j]));
                    } else {
                        ir[(size_t)j * Vn + i] = mkc<V>((T)iz.nd[j], T(0));
                    }
                }
                V dv = __ldg(dk + i);
                if (elec) {
                    dv.x -= rcv.y;   // + i * rho_c
                    dv.y += rcv.x;
                } else {
                    dv = mkc<V>(T(0), T(0));
                }
                dp[i] = dv;
                acc[0] += (double)dv.x;
                acc[1] += (double)dv.y;
            }, reinterpret_cast<double*>(&ds->mean_dpsi), (double)(c.M + 6 + J + (common ? 0 : J)) * sizeof(V));
        }
        // when electrostatics are off the charge fields stay zero
        if (!elec) {
            FTSP_CUDA(cudaMemsetAsync(kC.p + (size_t)M * Vn, 0, sizeof(V) * 2 * Vn, stream));
        }
        if (aux_pending) {   // the stress kernel of the pair path
            FTSP_CUDA(cudaEventRecord(ev_join, aux));
            FTSP_CUDA(cudaStreamWaitEvent(stream, ev_join, 0));
            aux_pending = false;
        }
    }

    // ---- drifts u_a = c_a w_a + sum_alpha gamma_a O_{a alpha} rho_alpha (+ sum of w^2) ----
    void drifts(int which)
    {
        const size_t Vn = V_;
        const int nm = c.nm, M = c.M;
        const V* om = which ? omega_bar.p : omega.p;
        V* u = which ? drift_bar.p : drift.p;
        const V* rt = kC.p;
        // gamma_a O_{a alpha} at a * MAXM + alpha: the loops below run to the
        // compile-time maxima, so every table entry and accumulator has a
        // constant index (no local-memory copies)
        ModeTab co{};
        for (int a = 0; a < nm; ++a) {
            co.c[a] = c.coeff[a];
            for (int al = 0; al < M; ++al)
                co.g[a * MAXM + al] = make_double2(c.gamma[a].x * c.O[a * M + al], c.gamma[a].y * c.O[a * M + al]);
        }
        if (nm == 1 && M == 1) {   // one mode, one monomer type: two accumulators
            const double c0 = co.c[0];
            const double2 g0 = co.g[0];
            reduce<2>(Vn, [=] __device__(size_t i, double* acc) {
                const V w = __ldg(om + i);
                u[i] = cadd(cscale(w, (T)c0), cmul(__ldg(rt + i), from_d<V>(g0)));
                const double2 wd = to_d(w);
                acc[0] += wd.x * wd.x - wd.y * wd.y;
                acc[1] += 2.0 * wd.x * wd.y;
            }, ds->fsq, 3.0 * sizeof(V));
            return;
        }
        reduce<2 * MAXMODE>(Vn, [=] __device__(size_t i, double* acc) {
#pragma unroll
            for (int a = 0; a < MAXMODE; ++a) {
                if (a >= nm) break;
                const V w = om[(size_t)a * Vn + i];
                // clear, add_scaled_complex(w, c), add_scaled_complex_const(rho, gamma O)
                V v = cscale(w, (T)co.c[a]);
#pragma unroll
                for (int al = 0; al < MAXM; ++al) {
                    if (al >= M) break;
                    v = cadd(v, cmul(rt[(size_t)al * Vn + i], from_d<V>(co.g[a * MAXM + al])));
                }
                u[(size_t)a * Vn + i] = v;
                const double2 wd = to_d(w);
                acc[2 * a] += wd.x * wd.x - wd.y * wd.y;
                acc[2 * a + 1] += 2.0 * wd.x * wd.y;
            }
        }, ds->fsq, (double)(2 * c.nm + c.M) * sizeof(V));
    }

    // ---- noise for this step (generated, or injected by ftsp_set_noise) ----
    void noises()
    {
        const size_t Vn = V_;
        const int nm = c.nm;
        T* e = eta.p;
        if (!noise_injected) {
            SigTab sg{};
            for (int a = 0; a < nm; ++a) sg.s[a] = c.noise ? std::sqrt(2.0 * c.lambda[a] * c.dt / c.dV) : 0.0;
            sg.s[nm] = (c.elec && c.noise) ? std::sqrt(2.0 * c.lpsi * c.dt / c.dV) : 0.0;
            // the step index is read on the device, so a captured step replays
            // with fresh noise
            const uint64_t seed = c.seed;
            const DevScal* d = ds;
            // the psi noise is summed as it is drawn (its mean is removed by
            // the predictor, remove_real_mean, complexLangevin.cu:296)
            reduce<1>(Vn, [=] __device__(size_t i, double* acc) {
                const uint64_t st = d->step;
                const double sc = sqrt(d->dt_scale);
#pragma unroll
                for (int f = 0; f <= MAXMODE; f += 2) {   // fields f and f + 1 from one draw
                    if (f > nm) break;
                    double n0, n1;
                    normal_pair_at(seed, st, (uint32_t)(f >> 1), i, n0, n1);
                    const T v0 = sg.s[f] != 0.0 ? (T)((sg.s[f] * sc) * n0) : T(0);
                    e[(size_t)f * Vn + i] = v0;
                    if (f == nm) acc[0] += (double)v0;
                    if (f + 1 <= nm) {
                        const double s1 = f + 1 <= MAXMODE ? sg.s[f + 1] : 0.0;
                        const T v1 = s1 != 0.0 ? (T)((s1 * sc) * n1) : T(0);
                        e[(size_t)(f + 1) * Vn + i] = v1;
                        if (f + 1 == nm) acc[0] += (double)v1;
                    }
                }
            }, &ds->mean_eta, (double)(c.nm + 1) * sizeof(T));
        } else if (c.elec) {   // injected noise: remove_real_mean of its psi part (complexLangevin.cu:296)
            const T* ep = e + (size_t)nm * Vn;
            reduce<1>(Vn, [=] __device__(size_t i, double* acc) { acc[0] += (double)ep[i]; }, &ds->mean_eta, (double)sizeof(T));
        }
        noise_injected = false;
    }

    // ---- predictor (complexLangevin.cu:328-347) ----
    void predictor()
    {
        const size_t Vn = V_;
        const int nm = c.nm;
        ModeTab co{};
        for (int a = 0; a < nm; ++a) co.s[a] = -c.dt * c.lambda[a];
        const double sp = -c.dt * c.lpsi;
        const bool elec = c.elec;
        const V* om = omega.p;
        const V* u = drift.p;
        V* ob = omega_bar.p;
        const V* ps = psi.p;
        V* pb = psi_bar.p;
        V* dp = dpsi.p;
        T* e = eta.p;
        DevScal* d = ds;
        const double invV = 1.0 / (double)Vn;
        if (c.scheme == FTSP_SCHEME_SI && plane_ok) {
            si_update_fused(false, lr.on_collect || lr.on_use);
            return;
        }
        if (c.scheme == FTSP_SCHEME_SI) {
            V* inc = si_inc.p;
            foreach(Vn, [=] __device__(size_t i) {
                T ep = e[(size_t)nm * Vn + i];
                if (elec) {
                    ep = (T)((double)ep + (-(d->mean_eta * invV)));
                    e[(size_t)nm * Vn + i] = ep;
                }
#pragma unroll
                for (int a = 0; a < MAXMODE; ++a) {
                    if (a >= nm) break;
                    V v = cscale(u[(size_t)a * Vn + i], (T)(co.s[a] * d->dt_scale));
                    v.x += e[(size_t)a * Vn + i];
                    inc[(size_t)a * Vn + i] = v;
                }
                V pv = mkc<V>(T(0), T(0));
                if (elec) {
                    V dv = cadd(dp[i], from_d<V>(dscale(d->mean_dpsi, -invV)));
                    dp[i] = dv;
                    pv = cscale(dv, (T)(sp * d->dt_scale));
                    pv.x += ep;
                }
                inc[(size_t)nm * Vn + i] = pv;
            }, (double)(c.nm * (2 * sizeof(V) + sizeof(T)) + 2 * sizeof(T) + 3 * sizeof(V)));
            si_precondition(lr.on_collect || lr.on_use);
            reduce<2>(Vn, [=] __device__(size_t i, double* acc) {
#pragma unroll
                for (int a = 0; a < MAXMODE; ++a) {
                    if (a >= nm) break;
                    ob[(size_t)a * Vn + i] = cadd(om[(size_t)a * Vn + i], inc[(size_t)a * Vn + i]);
                }
                const V pv = elec ? cadd(ps[i], inc[(size_t)nm * Vn + i]) : mkc<V>(T(0), T(0));
                pb[i] = pv;
                acc[0] += (double)pv.x;
                acc[1] += (double)pv.y;
            }, reinterpret_cast<double*>(&ds->mean_psi), (double)(3 * c.nm + 3) * sizeof(V));
            remove_mean(psi_bar.p, &ds->mean_psi);
            return;
        }
        reduce<2>(Vn, [=] __device__(size_t i, double* acc) {
            const double me = elec ? d->mean_eta * invV : 0.0;
            T ep = e[(size_t)nm * Vn + i];
            if (elec) {
                ep = (T)((double)ep + (-me));
                e[(size_t)nm * Vn + i] = ep;
            }
#pragma unroll
            for (int a = 0; a < MAXMODE; ++a) {
                if (a >= nm) break;
                V v = om[(size_t)a * Vn + i];
                v = cadd(v, cscale(u[(size_t)a * Vn + i], (T)(co.s[a] * d->dt_scale)));
                v.x += e[(size_t)a * Vn + i];
                ob[(size_t)a * Vn + i] = v;
            }
            V pv = mkc<V>(T(0), T(0));
            if (elec) {
                const double2 md = dscale(d->mean_dpsi, -invV);
                V dv = dp[i];
                dv = cadd(dv, from_d<V>(md));
                dp[i] = dv;
                pv = cadd(ps[i], cscale(dv, (T)(sp * d->dt_scale)));
                pv.x += ep;
            }
            pb[i] = pv;
            acc[0] += (double)pv.x;
            acc[1] += (double)pv.y;
        }, reinterpret_cast<double*>(&ds->mean_psi), (double)(c.nm * (3 * sizeof(V) + sizeof(T)) + 2 * sizeof(T) + 4 * sizeof(V)));
        remove_mean(psi_bar.p, &ds->mean_psi);
    }

    // f -= (sum / V), the sum being a device-side complex value
    void remove_mean(V* f, const double2* sum)
    {
        if (!c.elec) return;
        const double invV = 1.0 / (double)V_;
        foreach(V_, [=] __device__(size_t i) {
            const double2 m = dscale(*sum, -invV);
            f[i] = cadd(f[i], from_d<V>(m));
        }, 2.0 * sizeof(V));
    }

    // ---- corrector (complexLangevin.cu:349-368) + drift maxima + finite flag ----
    void corrector()
    {
        const size_t Vn = V_;
        const int nm = c.nm;
        ModeTab co{};
        for (int a = 0; a < nm; ++a) co.s[a] = -0.5 * c.dt * c.lambda[a];
        const double sp = -0.5 * c.dt * c.lpsi;
        const bool elec = c.elec;
        V* om = omega.p;
        const V* u0 = drift.p;
        const V* u1 = drift_bar.p;
        V* ps = psi.p;
        const V* dp = dpsi.p;
        V* db = dpsi_bar.p;
        const T* e = eta.p;
        DevScal* d = ds;
        const double invV = 1.0 / (double)Vn;
        if (c.scheme == FTSP_SCHEME_SI && plane_ok) {
            si_update_fused(true, false);
            return;
        }
        // drift maxima: max |u + u_bar|^2 per mode and for psi
        reduce<MAXMODE + 1, true>(Vn, [=] __device__(size_t i, double* acc) {
#pragma unroll
            for (int a = 0; a < MAXMODE; ++a) {
                if (a >= nm) break;
                const V s = cadd(u0[(size_t)a * Vn + i], u1[(size_t)a * Vn + i]);
                double v = (double)s.x * s.x + (double)s.y * s.y;
                if (!isfinite(v)) v = INFINITY;
                acc[a] = fmax(acc[a], v);
            }
            V dbv = db[i];
            if (elec) dbv = cadd(dbv, from_d<V>(dscale(d->mean_dpsi, -invV)));
            const V s = cadd(dp[i], dbv);
            double v = (double)s.x * s.x + (double)s.y * s.y;
            if (!isfinite(v)) v = INFINITY;
#pragma unroll
            for (int k = 0; k <= MAXMODE; ++k)   // acc[nm] with a constant index
                if (k == nm) acc[k] = fmax(acc[k], v);
        }, ds->dmax, (double)(2 * c.nm + 2) * sizeof(V));
        if (c.scheme == FTSP_SCHEME_SI) {
            V* inc = si_inc.p;
            foreach(Vn, [=] __device__(size_t i) {
#pragma unroll
                for (int a = 0; a < MAXMODE; ++a) {
                    if (a >= nm) break;
                    V v = cscale(cadd(u0[(size_t)a * Vn + i], u1[(size_t)a * Vn + i]), (T)(co.s[a] * d->dt_scale));
                    v.x += e[(size_t)a * Vn + i];
                    inc[(size_t)a * Vn + i] = v;
                }
                V pv = mkc<V>(T(0), T(0));
                if (elec) {
                    const V dbv = cadd(db[i], from_d<V>(dscale(d->mean_dpsi, -invV)));
                    db[i] = dbv;
                    pv = cscale(cadd(dp[i], dbv), (T)(sp * d->dt_scale));
                    pv.x += e[(size_t)nm * Vn + i];
                }
                inc[(size_t)nm * Vn + i] = pv;
            }, (double)(c.nm * (3 * sizeof(V) + sizeof(T)) + 4 * sizeof(V) + sizeof(T)));
            si_precondition();
            reduce<3>(Vn, [=] __device__(size_t i, double* acc) {
                bool bad = false;
#pragma unroll
                for (int a = 0; a < MAXMODE; ++a) {
                    if (a >= nm) break;
                    const V w = cadd(om[(size_t)a * Vn + i], inc[(size_t)a * Vn + i]);
                    om[(size_t)a * Vn + i] = w;
                    bad |= !(isfinite((double)w.x) && isfinite((double)w.y));
                }
                const V pv = elec ? cadd(ps[i], inc[(size_t)nm * Vn + i]) : mkc<V>(T(0), T(0));
                ps[i] = pv;
                acc[0] += (double)pv.x;
                acc[1] += (double)pv.y;
                if (bad || !(isfinite((double)pv.x) && isfinite((double)pv.y))) acc[2] += 1.0;
            }, ds->corr, (double)(3 * c.nm + 3) * sizeof(V));
            remove_mean(psi.p, reinterpret_cast<const double2*>(ds->corr));
            return;
        }
        reduce<3>(Vn, [=] __device__(size_t i, double* acc) {
            bool bad = false;
#pragma unroll
            for (int a = 0; a < MAXMODE; ++a) {
                if (a >= nm) break;
                V w = om[(size_t)a * Vn + i];
                w = cadd(w, cscale(u0[(size_t)a * Vn + i], (T)(co.s[a] * d->dt_scale)));
                w = cadd(w, cscale(u1[(size_t)a * Vn + i], (T)(co.s[a] * d->dt_scale)));
                w.x += e[(size_t)a * Vn + i];
                om[(size_t)a * Vn + i] = w;
                bad |= !(isfinite((double)w.x) && isfinite((double)w.y));
            }
            V pv = ps[i];
            if (elec) {
                V dbv = cadd(db[i], from_d<V>(dscale(d->mean_dpsi, -invV)));
                db[i] = dbv;
                pv = cadd(pv, cscale(dp[i], (T)(sp * d->dt_scale)));
                pv = cadd(pv, cscale(dbv, (T)(sp * d->dt_scale)));
                pv.x += e[(size_t)nm * Vn + i];
            } else {
                pv = mkc<V>(T(0), T(0));
            }
            ps[i] = pv;
            acc[0] += (double)pv.x;
            acc[1] += (double)pv.y;
            if (bad || !(isfinite((double)pv.x) && isfinite((double)pv.y))) acc[2] += 1.0;
        }, ds->corr, (double)(c.nm * (4 * sizeof(V) + sizeof(T)) + 5 * sizeof(V) + sizeof(T)));
        remove_mean(psi.p, reinterpret_cast<const double2*>(ds->corr));
    }

    // ---- observables from k-space sums (Parseval) ----
    void kspace_obs()
    {
        const size_t Vn = V_;
        const int nm = c.nm, M = c.M, J = (int)c.ions.size();
        const int m1 = c.m1, m2 = c.m2, m3 = c.m3;
        const bool elec = c.elec;
        ObsConst oc{};
        for (int a = 0; a < nm; ++a)
            for (int al = 0; al < M; ++al)
                oc.g[a * M + al] = make_double2(c.gamma[a].x * c.O[a * M + al], c.gamma[a].y * c.O[a * M + al]);
        for (int j = 0; j < J; ++j) {
            oc.z[j] = c.ions[j].z;
            oc.a2ion[j] = c.ions[j].smear * c.ions[j].smear;
        }
        const double a2 = c.a * c.a;
        const V* kAp = kA.p;
        const V* dBp = dB.p;
        const T* gm = gam.p;
        const T* gi = gion.p;
        const double* kxp = kx.p;
        const double* kyp = ky.p;
        const double* kzp = kz.p;
        const int sum_m = m1 + m2 + m3;
        const DevScal* d = ds;
        const bool common = ion_common;
        // two reductions: the density-field channels (0..13) and the
        // electrostatic field term k_a k_b Psi(k) Psi(-k) (14..25), so that
        // neither kernel holds all 26 FP64 accumulators
        reduce<14>(Vn, [=] __device__(size_t i, double* acc) {
            const int x = (int)(i / ((size_t)m2 * m3));
            const int r = (int)(i - (size_t)x * m2 * m3);
            const int y = r / m3, z = r - y * m3;
            const int nx = x ? m1 - x : 0, ny = y ? m2 - y : 0, nz = z ? m3 - z : 0;
            const size_t ineg = ((size_t)nx * m2 + ny) * m3 + nz;
            const double ax = kxp[x], ay = kyp[y], az = kzp[z];
            const double kk[6] = {ax * ax, ay * ay, az * az, ax * ay, ax * az, ay * az};
            const double Gk = (double)(gm[x] * gm[m1 + y] * gm[m1 + m2 + z]);
            // A = sum_alpha R_alpha(-k) W_alpha(k),  W_alpha = Gamma sum_a g_{a alpha} Omega_a
            double2 A = make_double2(0.0, 0.0);
            for (int al = 0; al < M; ++al) {
                double2 w = make_double2(0.0, 0.0);
                for (int a = 0; a < nm; ++a) w = dadd(w, dmul(to_d(kAp[(size_t)a * Vn + i]), oc.g[a * M + al]));
                A = dadd(A, dmul(to_d(dBp[(size_t)al * Vn + ineg]), dscale(w, Gk)));
            }
            double2 Bc = make_double2(0.0, 0.0), Ij = make_double2(0.0, 0.0), I0 = make_double2(0.0, 0.0);
            if (elec) {
                const double2 Pk = to_d(kAp[(size_t)nm * Vn + i]);
                const double2 rc = dmul(to_d(dBp[(size_t)M * Vn + ineg]), dscale(Pk, Gk));
                Bc = make_double2(-rc.y, rc.x);   // i * R_c(-k) Gamma Psi(k)
                if (common) {
                    // combined ion charge (z_j (n_j/V)/Q_j already in it), common smearing
                    const double2 p = dmul(to_d(dBp[(size_t)(M + 1) * Vn + ineg]), dscale(Pk, Gk));
                    const double2 ip = make_double2(-p.y, p.x);
                    Ij = dscale(ip, -oc.a2ion[0]);
                    I0 = dscale(ip, 1.0 / 6.0);
                } else {
                    for (int j = 0; j < J; ++j) {
                        const T* t = gi + (size_t)j * sum_m;
                        const double gj = (double)(t[x] * t[m1 + y] * t[m1 + m2 + z]);
                        const double2 p = dmul(dmul(to_d(dBp[(size_t)(M + 1 + j) * Vn + ineg]), d->ion_factor[j]), dscale(Pk, gj * oc.z[j]));
                        const double2 ip = make_double2(-p.y, p.x);
                        Ij = dadd(Ij, dscale(ip, -oc.a2ion[j]));
                        I0 = dadd(I0, dscale(ip, 1.0 / 6.0));
                    }
                }
            }
            const double2 base = make_double2(-a2 * (A.x + Bc.x) + Ij.x, -a2 * (A.y + Bc.y) + Ij.y);
            for (int cc = 0; cc < 6; ++cc) {
                acc[2 * cc] += kk[cc] * base.x;
                acc[2 * cc + 1] += kk[cc] * base.y;
            }
            acc[12] += 0.5 * A.x + Bc.x / 6.0 + I0.x;
            acc[13] += 0.5 * A.y + Bc.y / 6.0 + I0.y;
        }, ds->kobs, (double)(c.nm + c.M + 1 + (ion_common ? 1 : (int)c.ions.size())) * sizeof(V));
        if (!elec) {
            FTSP_CUDA(cudaMemsetAsync(ds->kobs + 14, 0, 12 * sizeof(double), stream));
            return;
        }
        reduce<12>(Vn, [=] __device__(size_t i, double* acc) {
            const int x = (int)(i / ((size_t)m2 * m3));
            const int r = (int)(i - (size_t)x * m2 * m3);
            const int y = r / m3, z = r - y * m3;
            const int nx = x ? m1 - x : 0, ny = y ? m2 - y : 0, nz = z ? m3 - z : 0;
            const size_t ineg = ((size_t)nx * m2 + ny) * m3 + nz;
            const double ax = kxp[x], ay = kyp[y], az = kzp[z];
            const double kk[6] = {ax * ax, ay * ay, az * az, ax * ay, ax * az, ay * az};
            const double2 X = dmul(to_d(kAp[(size_t)nm * Vn + i]), to_d(kAp[(size_t)nm * Vn + ineg]));
            for (int cc = 0; cc < 6; ++cc) {
                acc[2 * cc] += kk[cc] * X.x;
                acc[2 * cc + 1] += kk[cc] * X.y;
            }
        }, ds->kobs + 14, 2.0 * sizeof(V));
    }

    void finalize_record(bool with_stress)
    {
        if (with_stress) {
            k_combine<false><<<12, COMBINE_THREADS, 0, stream>>>(spart.p, x_ctas(), 12, ds->sconn);
            ++launches;
        }
        const int S = (int)c.sp.size(), J = (int)c.ions.size(), nm = c.nm;
        RecConst rc{};
        for (int s = 0; s < S; ++s) {
            double zz = 0.0;
            for (double q : c.sp[s].charge) zz += q * q;
            rc.nv[s] = c.sp[s].nc / c.volume;
            rc.self_poly[s] = -c.lB * zz / (2.0 * std::sqrt(PI) * c.a);
            rc.ideal_poly[s] = std::log(c.sp[s].nc / c.volume);
        }
        double ion_total = 0.0;
        for (int j = 0; j < J; ++j) {
            rc.nvion[j] = c.ions[j].count / c.volume;
            rc.self_ion[j] = -c.lB * c.ions[j].z * c.ions[j].z / (2.0 * std::sqrt(PI) * c.ions[j].smear);
            rc.ideal_ion[j] = std::log(c.ions[j].count / c.volume);
            ion_total += c.ions[j].count;
        }
        for (int a = 0; a < nm; ++a) rc.coeff[a] = c.coeff[a];
        double chains = 0.0;
        for (auto& s : c.sp) chains += s.nc;
        const double ideal = (chains + ion_total) / c.volume;
        // mode term of stress::build_kernels (stress.cu:106-149)
        double sum[6] = {0, 0, 0, 0, 0, 0};
        long long modes = 0;
        if (c.elec) {
            std::vector<double> hx(c.m1), hy(c.m2), hz(c.m3);
            for (int i = 0; i < c.m1; ++i) hx[i] = wave_number(i, c.m1, c.L[0]);
            for (int i = 0; i < c.m2; ++i) hy[i] = wave_number(i, c.m2, c.L[1]);
            for (int i = 0; i < c.m3; ++i) hz[i] = wave_number(i, c.m3, c.L[2]);
            for (int x = 0; x < c.m1; ++x)
                for (int y = 0; y < c.m2; ++y)
                    for (int z = 0; z < c.m3; ++z) {
                        const double k2 = hx[x] * hx[x] + hy[y] * hy[y] + hz[z] * hz[z];
                        if (k2 > 0.0) {
                            ++modes;
                            const double v[6] = {hx[x] * hx[x], hy[y] * hy[y], hz[z] * hz[z], hx[x] * hy[y], hx[x] * hz[z], hy[y] * hz[z]};
                            for (int cc = 0; cc < 6; ++cc) sum[cc] += v[cc] / k2;
                        }
                    }
        }
        for (int cc = 0; cc < 6; ++cc) {
            const double delta = cc < 3 ? 1.0 : 0.0;
            const double mode_term = c.elec ? ((1.0 / 3.0) * (double)modes * delta - sum[cc]) / c.volume : 0.0;
            rc.ideal_stress[cc] = (ideal + c.self_pressure) * delta + mode_term;
        }
        rc.ideal_iso = ideal + c.self_pressure;
        int na = 0;
        for (int cc = 0; cc < 6; ++cc)
            if (c.stress_mask & (1 << cc)) rc.active[na++] = cc;
        const int iso = c.iso;
        const double V2 = (double)V_ * (double)V_;
        const double invV = 1.0 / (double)V_;
        const double lB = c.lB;
        const bool elec = c.elec;
        DevScal* d = ds;
        const bool ws = with_stress;
        k_foreach<<<1, 32, 0, stream>>>(1, [=] __device__(size_t) {
            double2* rec = reinterpret_cast<double2*>(d->rec);
            int k = 0;
            double2 chem[MAXSP + MAXION];
            for (int s = 0; s < S; ++s) chem[s] = dneglog(d->Q[s]);
            for (int j = 0; j < J; ++j) chem[S + j] = elec ? dneglog(d->Qion[j]) : make_double2(0.0, 0.0);
            for (int i = 0; i < S + J; ++i) rec[k++] = chem[i];
            for (int s = 0; s < S; ++s) rec[k++] = make_double2(rc.self_poly[s], 0.0);
            for (int j = 0; j < J; ++j) rec[k++] = make_double2(rc.self_ion[j], 0.0);
            for (int s = 0; s < S; ++s) rec[k++] = make_double2(rc.ideal_poly[s], 0.0);
            for (int j = 0; j < J; ++j) rec[k++] = make_double2(rc.ideal_ion[j], 0.0);
            double2 Hm = make_double2(0.0, 0.0);
            for (int a = 0; a < nm; ++a) Hm = dadd(Hm, make_double2(0.5 * rc.coeff[a] * d->fsq[2 * a] * invV, 0.5 * rc.coeff[a] * d->fsq[2 * a + 1] * invV));
            const double* ko = d->kobs;
            const double2 Xtr = make_double2(ko[14] + ko[16] + ko[18], ko[15] + ko[17] + ko[19]);
            if (elec) Hm = dadd(Hm, dscale(Xtr, 1.0 / (8.0 * PI * lB * V2)));
            for (int s = 0; s < S; ++s) Hm = dadd(Hm, dscale(chem[s], rc.nv[s]));
            for (int j = 0; j < J; ++j) Hm = dadd(Hm, dscale(chem[S + j], rc.nvion[j]));
            rec[k++] = Hm;
            if (ws) {
                // connectivity sums over the bond-pass CTAs
                double2 Sc[6];
                for (int cc = 0; cc < 6; ++cc) Sc[cc] = make_double2(d->sconn[2 * cc], d->sconn[2 * cc + 1]);
                const double2 V0 = make_double2(ko[12], ko[13]);
                for (int q = 0; q < na; ++q) {
                    const int cc = rc.active[q];
                    const double delta = cc < 3 ? 1.0 : 0.0;
                    double2 v = make_double2(rc.ideal_stress[cc], 0.0);
                    if (elec) {
                        const double2 e = make_double2(ko[14 + 2 * cc] - delta * Xtr.x / 3.0, ko[14 + 2 * cc + 1] - delta * Xtr.y / 3.0);
                        v = dadd(v, dscale(e, 1.0 / (4.0 * PI * lB * V2)));
                    }
                    v = dadd(v, dscale(Sc[cc], 1.0 / (3.0 * V2)));
                    v = dadd(v, dscale(make_double2(ko[2 * cc] + delta * V0.x, ko[2 * cc + 1] + delta * V0.y), 1.0 / V2));
                    rec[k++] = v;
                }
                if (iso) {
                    double2 v = make_double2(rc.ideal_iso, 0.0);
                    v = dadd(v, dscale(dadd(dadd(Sc[0], Sc[1]), Sc[2]), 1.0 / (9.0 * V2)));
                    const double2 tr = make_double2((ko[0] + ko[2] + ko[4]) / 3.0 + V0.x, (ko[1] + ko[3] + ko[5]) / 3.0 + V0.y);
                    v = dadd(v, dscale(tr, 1.0 / V2));
                    rec[k++] = v;
                }
            }
        });
        ++launches;
    }

    // ---- API ----
    Buf<double2> stage;   // FP64 host fields land here, then convert on the device

    void set_fields(const double* om, const double* ps) override
    {
        drop_pending_fields();
        const size_t Vn = V_;
        const int nm = c.nm;
        if (sizeof(T) == 8) {
            if (nm > 0) FTSP_CUDA(cudaMemcpyAsync(omega.p, om, sizeof(double2) * nm * Vn, cudaMemcpyHostToDevice, stream));
            FTSP_CUDA(cudaMemcpyAsync(psi.p, ps, sizeof(double2) * Vn, cudaMemcpyHostToDevice, stream));
        } else {
            if (!stage.p) stage.alloc((size_t)(nm + 1) * Vn);
            if (nm > 0) FTSP_CUDA(cudaMemcpyAsync(stage.p, om, sizeof(double2) * nm * Vn, cudaMemcpyHostToDevice, stream));
            FTSP_CUDA(cudaMemcpyAsync(stage.p + (size_t)nm * Vn, ps, sizeof(double2) * Vn, cudaMemcpyHostToDevice, stream));
            convert_staged(stage.p);
        }
        new_run();
        FTSP_CUDA(cudaStreamSynchronize(stream));
    }

    // FP64 fields in device memory (modes, then psi) into the working precision
    void convert_staged(const double2* s)
    {
        const size_t Vn = V_;
        const int nm = c.nm;
        V* o = omega.p;
        V* p = psi.p;
        foreach(Vn, [=] __device__(size_t i) {
            for (int a = 0; a < nm; ++a) o[(size_t)a * Vn + i] = from_d<V>(s[(size_t)a * Vn + i]);
            p[i] = from_d<V>(s[(size_t)nm * Vn + i]);
        });
    }

    // ---- fields uploaded while the previous step runs ----
    // set_fields_async copies the host fields into a device staging buffer on
    // a copy stream and returns; the next call that uses the fields installs
    // them on the handle's stream (after the copy, by an event): conversion,
    // psi mean removal, a new run.  A second upload first waits until the
    // staging buffer has been installed.
    Buf<double2> astage;
    cudaStream_t cstream = nullptr;
    cudaEvent_t ev_staged = nullptr, ev_installed = nullptr;
    bool fields_pending = false, astage_used = false;

    void set_fields_async(const double* om, const double* ps) override
    {
        const size_t Vn = V_;
        const int nm = c.nm;
        if (!cstream) {
            FTSP_CUDA(cudaStreamCreateWithFlags(&cstream, cudaStreamNonBlocking));
            FTSP_CUDA(cudaEventCreateWithFlags(&ev_staged, cudaEventDisableTiming));
            FTSP_CUDA(cudaEventCreateWithFlags(&ev_installed, cudaEventDisableTiming));
            astage.alloc((size_t)(nm + 1) * Vn);
        }
        if (fields_pending) install_pending_fields();   // one staging buffer
        if (astage_used) FTSP_CUDA(cudaStreamWaitEvent(cstream, ev_installed, 0));
        if (nm > 0) FTSP_CUDA(cudaMemcpyAsync(astage.p, om, sizeof(double2) * nm * Vn, cudaMemcpyHostToDevice, cstream));
        FTSP_CUDA(cudaMemcpyAsync(astage.p + (size_t)nm * Vn, ps, sizeof(double2) * Vn, cudaMemcpyHostToDevice, cstream));
        FTSP_CUDA(cudaEventRecord(ev_staged, cstream));
        fields_pending = true;
    }

    void install_pending_fields() override
    {
        if (!fields_pending) return;
        fields_pending = false;
        const size_t Vn = V_;
        const int nm = c.nm;
        FTSP_CUDA(cudaStreamWaitEvent(stream, ev_staged, 0));
        if (sizeof(T) == 8) {
            if (nm > 0) FTSP_CUDA(cudaMemcpyAsync(omega.p, astage.p, sizeof(double2) * nm * Vn, cudaMemcpyDeviceToDevice, stream));
            FTSP_CUDA(cudaMemcpyAsync(psi.p, astage.p + (size_t)nm * Vn, sizeof(double2) * Vn, cudaMemcpyDeviceToDevice, stream));
        } else {
            convert_staged(astage.p);
        }
        new_run();
        FTSP_CUDA(cudaEventRecord(ev_installed, stream));
        astage_used = true;
    }

    // a synchronous set_fields supersedes an upload not yet installed
    void drop_pending_fields()
    {
        if (!fields_pending) return;
        FTSP_CUDA(cudaEventSynchronize(ev_staged));
        fields_pending = false;
    }

    // psi zero mode, run state and first checkpoint of freshly loaded fields
    void new_run()
    {
        const size_t Vn = V_;
        const int nm = c.nm;
        if (c.elec) {
            const V* p = psi.p;
            reduce<2>(Vn, [=] __device__(size_t i, double* acc) {
                acc[0] += (double)p[i].x;
                acc[1] += (double)p[i].y;
            }, reinterpret_cast<double*>(&ds->mean_psi));
            remove_mean(psi.p, &ds->mean_psi);
        } else {
            FTSP_CUDA(cudaMemsetAsync(psi.p, 0, sizeof(V) * Vn, stream));
        }
        // a new run: no pending rollback, no rollbacks taken
        FTSP_CUDA(cudaMemsetAsync(&ds->bad_last, 0, sizeof(int), stream));
        FTSP_CUDA(cudaMemsetAsync(&ds->restarts, 0, sizeof(int), stream));
        FTSP_CUDA(cudaMemsetAsync(&ds->exhausted, 0, sizeof(int), stream));
        if (c.restart_interval > 0) {
            if (nm > 0) FTSP_CUDA(cudaMemcpyAsync(ck.p, omega.p, sizeof(V) * nm * Vn, cudaMemcpyDeviceToDevice, stream));
            FTSP_CUDA(cudaMemcpyAsync(ck.p + (size_t)nm * Vn, psi.p, sizeof(V) * Vn, cudaMemcpyDeviceToDevice, stream));
        }
    }

    long long get_field(const std::string& name, double* out) override
    {
        install_pending_fields();
        const size_t Vn = V_;
        const int nm = c.nm, M = c.M, J = (int)c.ions.size();
        const V* p = nullptr;
        size_t n = 0;
        if (name == "omega") { p = omega.p; n = nm * Vn; }
        else if (name == "psi") { p = psi.p; n = Vn; }
        else if (name == "omega_bar") { p = omega_bar.p; n = nm * Vn; }
        else if (name == "psi_bar") { p = psi_bar.p; n = Vn; }
        else if (name == "drift") { p = drift.p; n = nm * Vn; }
        else if (name == "drift_bar") { p = drift_bar.p; n = nm * Vn; }
        else if (name == "dpsi") { p = dpsi.p; n = Vn; }
        else if (name == "dpsi_bar") { p = dpsi_bar.p; n = Vn; }
        else if (name == "rho_type") { p = kC.p; n = (size_t)M * Vn; }
        else if (name == "rho_c_poly") { p = kC.p + (size_t)M * Vn; n = Vn; }
        else if (name == "rho_c_ion") { p = kC.p + (size_t)(M + 1) * Vn; n = Vn; }
        else if (name == "rho_p") { p = rho_p.p; n = Vn; }
        else if (name == "rho_c") { p = rho_c.p; n = Vn; }
        else if (name == "ion_rho") { p = ion_rho.p; n = (size_t)J * Vn; }
        else if (name == "W_type_s") { p = kB.p; n = (size_t)M * Vn; }
        else if (name == "psi_s") { p = kB.p + (size_t)M * Vn; n = Vn; }
        else if (name == "qF") { p = qF.p; n = (size_t)Nmax * Vn; }
        else if (name == "si_precond" && si_G.p) {
            const size_t nr = (size_t)(nm + 1) * Vn;
            if (out) {
                std::vector<T> tmp(nr);
                FTSP_CUDA(cudaMemcpyAsync(tmp.data(), si_G.p, sizeof(T) * nr, cudaMemcpyDeviceToHost, stream));
                FTSP_CUDA(cudaStreamSynchronize(stream));
                for (size_t i = 0; i < nr; ++i) {
                    const size_t f = i / Vn;
                    const double sf = c.dt * (f < (size_t)nm ? c.lambda[f] : c.lpsi);
                    out[2 * i] = (double)(T)(1.0 / (1.0 + sf * (double)tmp[i]));
                    out[2 * i + 1] = 0.0;
                }
            }
            return (long long)(2 * nr);
        }
        else if ((name == "learn_A" && lr.A.p) || (name == "learn_B" && lr.B.p) || (name == "learn_Pw" && lr.Pw.p) ||
                 (name == "learn_Pp" && lr.Pp.p)) {
            const bool one = name == "learn_Pw" || name == "learn_Pp";
            const size_t nr = one ? Vn : (size_t)(nm + 1) * Vn;
            const float* src = name == "learn_A" ? lr.A.p : name == "learn_B" ? lr.B.p : name == "learn_Pw" ? lr.Pw.p : lr.Pp.p;
            if (out) {
                std::vector<float> tmp(nr);
                FTSP_CUDA(cudaMemcpyAsync(tmp.data(), src, sizeof(float) * nr, cudaMemcpyDeviceToHost, stream));
                FTSP_CUDA(cudaStreamSynchronize(stream));
                for (size_t i = 0; i < nr; ++i) {
                    out[2 * i] = (double)tmp[i];
                    out[2 * i + 1] = 0.0;
                }
            }
            return (long long)(2 * nr);
        }
        else if (name == "eta") {
            // the last step's real noise, modes then psi (psi after its mean removal)
            const size_t nr = (size_t)(nm + 1) * Vn;
            if (out) {
                std::vector<T> tmp(nr);
                FTSP_CUDA(cudaMemcpyAsync(tmp.data(), eta.p, sizeof(T) * nr, cudaMemcpyDeviceToHost, stream));
                FTSP_CUDA(cudaStreamSynchronize(stream));
                for (size_t i = 0; i < nr; ++i) {
                    out[2 * i] = (double)tmp[i];
                    out[2 * i + 1] = 0.0;
                }
            }
            return (long long)(2 * nr);
        }
        else if ((name == "si_G" && si_G.p) || (name == "learned_G" && lr.GL.p)) {
            const size_t nr = (size_t)(nm + 1) * Vn;
            if (out) {
                std::vector<T> tmp(nr);
                FTSP_CUDA(cudaMemcpyAsync(tmp.data(), name == "si_G" ? si_G.p : lr.GL.p, sizeof(T) * nr, cudaMemcpyDeviceToHost, stream));
                FTSP_CUDA(cudaStreamSynchronize(stream));
                for (size_t i = 0; i < nr; ++i) {
                    out[2 * i] = (double)tmp[i];
                    out[2 * i + 1] = 0.0;
                }
            }
            return (long long)(2 * nr);
        }
        else return -1;
        if (out && n) {
            std::vector<V> tmp(n);
            FTSP_CUDA(cudaMemcpyAsync(tmp.data(), p, sizeof(V) * n, cudaMemcpyDeviceToHost, stream));
            std::vector<int> ex((size_t)Nmax, 0);
            if (name == "qF") FTSP_CUDA(cudaMemcpyAsync(ex.data(), expo.p, sizeof(int) * Nmax, cudaMemcpyDeviceToHost, stream));
            // a mirror-symmetric species stores u = q / E (u = 1 at s = 0): q = u E
            const int su = name == "qF" ? qF_holds_u : -1;
            std::vector<V> et;
            if (su >= 0) {
                et.resize(E.n);
                FTSP_CUDA(cudaMemcpyAsync(et.data(), E.p, sizeof(V) * E.n, cudaMemcpyDeviceToHost, stream));
            }
            FTSP_CUDA(cudaStreamSynchronize(stream));
            for (size_t i = 0; i < n; ++i) {
                // qF is stored renormalised by 2^-aF[s]; return the true propagator
                const int e2 = name == "qF" ? ex[i / Vn] : 0;
                double qx = (double)tmp[i].x, qy = (double)tmp[i].y;
                const size_t seg = i / Vn;
                if (su >= 0 && seg < (size_t)c.sp[su].N) {
                    const V e = et[(size_t)c.sp[su].cls[seg] * Vn + i % Vn];
                    const double ux = seg == 0 ? 1.0 : qx, uy = seg == 0 ? 0.0 : qy;
                    qx = ux * (double)e.x - uy * (double)e.y;
                    qy = ux * (double)e.y + uy * (double)e.x;
                }
                out[2 * i] = std::ldexp(qx, e2);
                out[2 * i + 1] = std::ldexp(qy, e2);
            }
        }
        return (long long)(2 * n);
    }

    void pull_scalars()
    {
        FTSP_CUDA(cudaMemcpyAsync(&hs, ds, sizeof(DevScal), cudaMemcpyDeviceToHost, stream));
        FTSP_CUDA(cudaStreamSynchronize(stream));
    }

    void compute_densities(int which, double* Q) override
    {
        install_pending_fields();
        eval(which, false);
        pull_scalars();
        if (Q)
            for (size_t s = 0; s < c.sp.size(); ++s) {
                Q[2 * s] = hs.Q[s].x;
                Q[2 * s + 1] = hs.Q[s].y;
            }
    }

    void field_squares(int which)
    {
        const size_t Vn = V_;
        const int nm = c.nm;
        const V* om = which ? omega_bar.p : omega.p;
        if (nm == 1) {
            reduce<2>(Vn, [=] __device__(size_t i, double* acc) {
                const double2 wd = to_d(om[i]);
                acc[0] += wd.x * wd.x - wd.y * wd.y;
                acc[1] += 2.0 * wd.x * wd.y;
            }, ds->fsq);
            return;
        }
        reduce<2 * MAXMODE>(Vn, [=] __device__(size_t i, double* acc) {
#pragma unroll
            for (int a = 0; a < MAXMODE; ++a) {
                if (a >= nm) break;
                const double2 wd = to_d(om[(size_t)a * Vn + i]);
                acc[2 * a] += wd.x * wd.x - wd.y * wd.y;
                acc[2 * a + 1] += 2.0 * wd.x * wd.y;
            }
        }, ds->fsq);
    }

    void measure(int which, double* rec) override
    {
        install_pending_fields();
        const bool st = c.stress_on();
        eval(which, st);
        field_squares(which);
        kspace_obs();
        finalize_record(st);
        pull_scalars();
        if (rec) std::memcpy(rec, hs.rec, sizeof(double) * 2 * c.record_len());
    }

    void set_noise(const double* e) override
    {
        const size_t n = (size_t)(c.nm + 1) * V_;
        std::vector<T> tmp(n);
        for (size_t i = 0; i < n; ++i) tmp[i] = (T)e[i];
        FTSP_CUDA(cudaMemcpyAsync(eta.p, tmp.data(), sizeof(T) * n, cudaMemcpyHostToDevice, stream));
        FTSP_CUDA(cudaStreamSynchronize(stream));
        noise_injected = true;
    }

    // ---- device-side checkpoint and rollback (complexLangevin.cu:583-636 semantics) ----
    // A step that ends with a non-finite field, Q or observable sets bad_last;
    // the next step first restores (omega, psi) from the last checkpoint and
    // counts a restart.  Once max_restarts rollbacks have been taken, a
    // further non-finite step is final (the reference stops with "maximum
    // non-finite restarts exceeded", complexLangevin.cu:626-636): nothing is
    // restored any more and the exhausted flag keeps every later step
    // non-finite until set_fields starts a new run.  Checkpoints are taken
    // every restart_interval steps from a finite state.  Everything stays on
    // the device.
    void restore_if_bad()
    {
        const size_t Vn = V_;
        const int nm = c.nm;
        V* om = omega.p;
        V* ps = psi.p;
        const V* ckp = ck.p;
        DevScal* d = ds;
        const int cap = c.max_restarts;
        foreach(Vn, [=] __device__(size_t i) {
            if (!d->bad_last || d->exhausted || d->restarts >= cap) return;
            for (int a = 0; a < nm; ++a) om[(size_t)a * Vn + i] = ckp[(size_t)a * Vn + i];
            ps[i] = ckp[(size_t)nm * Vn + i];
        });
        double* pend = avg.on ? avg.acc.p + (size_t)avg.nblk * (c.record_len() + 2) : nullptr;
        const int R2 = c.record_len() + 2;
        k_foreach<<<1, 32, 0, stream>>>(1, [=] __device__(size_t) {
            if (d->bad_last && !d->exhausted) {
                if (d->restarts >= cap) {
                    d->exhausted = 1;
                } else {
                    d->restarts += 1;
                    d->bad_last = 0;
                    if (pend) {   // the records since the checkpoint are undone with the fields
                        d->avg_count -= (long long)pend[R2 - 1];
                        for (int i = 0; i < R2; ++i) pend[i] = 0.0;
                    }
                }
            }
        });
        ++launches;
    }

    void mark_step_status()
    {
        DevScal* d = ds;
        const int S = (int)c.sp.size(), R = c.record_len();
        k_foreach<<<1, 32, 0, stream>>>(1, [=] __device__(size_t) {
            bool bad = d->nonfinite != 0 || d->corr[2] != 0.0 || d->exhausted != 0;
            for (int s = 0; s < S; ++s) bad |= !(isfinite(d->Q[s].x) && isfinite(d->Q[s].y));
            for (int i = 0; i < 2 * R; ++i) bad |= !isfinite(d->rec[i]);
            d->bad_last = bad ? 1 : 0;
            d->step += 1;
        });
        ++launches;
    }

    // copies (omega, psi) to the device checkpoint after every
    // restart_interval-th finite step; the schedule is decided on the device
    void checkpoint_if_good()
    {
        const size_t Vn = V_;
        const int nm = c.nm;
        const V* om = omega.p;
        const V* ps = psi.p;
        V* ckp = ck.p;
        const DevScal* d = ds;
        const unsigned long long every = (unsigned long long)c.restart_interval;
        foreach(Vn, [=] __device__(size_t i) {
            if (d->bad_last || d->step % every != 0) return;
            for (int a = 0; a < nm; ++a) ckp[(size_t)a * Vn + i] = om[(size_t)a * Vn + i];
            ckp[(size_t)nm * Vn + i] = ps[i];
        }, 2.0 * (c.nm + 1) * sizeof(V) / (double)c.restart_interval);
    }

    void step_device()
    {
        if (c.restart_interval > 0) restore_if_bad();
        const bool st = c.stress_on();
        eval(0, false);
        // save Q of the first evaluation for the finite check
        FTSP_CUDA(cudaMemsetAsync(&ds->nonfinite, 0, sizeof(int), stream));
        {
            DevScal* d = ds;
            const int S = (int)c.sp.size();
            k_foreach<<<1, 32, 0, stream>>>(1, [=] __device__(size_t) {
                for (int s = 0; s < S; ++s)
                    if (!isfinite(d->Q[s].x) || !isfinite(d->Q[s].y)) d->nonfinite = 1;
            });
            ++launches;
        }
        drifts(0);
        if (adaptive_u > 0.0) adapt_dt();
        noises();
        predictor();
        eval(1, st);
        drifts(1);
        const bool learn = lr.on_collect || lr.on_use;
        if (learn) learn_after_predictor();
        kspace_obs();
        finalize_record(st);
        corrector();
        if (learn) learn_after_step();
        mark_step_status();
        if (avg.on) {
            k_average<<<1, 128, 0, stream>>>(ds, avg.acc.p, c.record_len(), avg.nblk, avg.skip, avg.samples,
                                             avg.per_block, (unsigned long long)c.restart_interval);
            ++launches;
        }
        if (c.restart_interval > 0) checkpoint_if_good();
    }

    // ---- time averages of the record (complexLangevin.cu:424-467) ----
    struct Avg {
        bool on = false;
        long long skip = 0, samples = 0, per_block = 1;
        int blocks = 0, nblk = 0;
        Buf<double> acc;   // nblk blocks of (R + 2), then the pending accumulator
    } avg;

    void average_start(long long skip, long long samples, int blocks) override
    {
        if (skip < 0 || samples < 1) throw std::runtime_error("ftsp_average_start: need skip >= 0 and samples >= 1");
        if (blocks < 1 || blocks > 1000 || blocks > samples)
            throw std::runtime_error("ftsp_average_start: blocks must be in 1..min(samples, 1000)");
        drop_step_graph();
        avg.acc.release();
        avg.skip = skip;
        avg.samples = samples;
        avg.blocks = blocks;
        avg.per_block = (samples + blocks - 1) / blocks;
        const int R = c.record_len();
        avg.nblk = (int)((samples + avg.per_block - 1) / avg.per_block);
        avg.acc.alloc((size_t)(avg.nblk + 1) * (R + 2));
        FTSP_CUDA(cudaMemsetAsync(avg.acc.p, 0, sizeof(double) * avg.acc.n, stream));
        FTSP_CUDA(cudaMemsetAsync(&ds->avg_seen, 0, 3 * sizeof(long long), stream));
        FTSP_CUDA(cudaStreamSynchronize(stream));
        avg.on = true;
    }

    // mean over every accumulated record (weighted by dt scale) and the
    // standard error from the means of the complete blocks (NaN with fewer
    // than two); returns the number of records accumulated
    long long average_read(double* mean, double* se) override
    {
        if (!avg.on) throw std::runtime_error("ftsp_average_read: averaging was not started");
        const int R = c.record_len();
        std::vector<double> a(avg.acc.n);
        FTSP_CUDA(cudaMemcpyAsync(a.data(), avg.acc.p, sizeof(double) * a.size(), cudaMemcpyDeviceToHost, stream));
        pull_scalars();
        const int nblk = avg.nblk;
        std::vector<double> sum(R, 0.0);
        double wsum = 0.0;
        std::vector<std::vector<double>> bm;
        for (int b = 0; b < nblk; ++b) {
            const double* x = a.data() + (size_t)b * (R + 2);
            for (int i = 0; i < R; ++i) sum[i] += x[i];
            wsum += x[R];
            if (x[R + 1] >= (double)avg.per_block && x[R] > 0.0) {
                std::vector<double> m(R);
                for (int i = 0; i < R; ++i) m[i] = x[i] / x[R];
                bm.push_back(m);
            }
        }
        for (int i = 0; i < R; ++i) {
            if (mean) mean[i] = wsum > 0.0 ? sum[i] / wsum : NAN;
            if (se) {
                if (bm.size() < 2) {
                    se[i] = NAN;
                    continue;
                }
                double mu = 0.0;
                for (auto& m : bm) mu += m[i];
                mu /= (double)bm.size();
                double v = 0.0;
                for (auto& m : bm) v += (m[i] - mu) * (m[i] - mu);
                se[i] = std::sqrt(v / (double)(bm.size() - 1) / (double)bm.size());
            }
        }
        return hs.avg_committed;
    }

    int status_from_host()
    {
        const int S = (int)c.sp.size();
        bool bad = hs.nonfinite != 0;
        for (int s = 0; s < S; ++s) bad |= !(std::isfinite(hs.Q[s].x) && std::isfinite(hs.Q[s].y));
        for (int i = 0; i < 2 * c.record_len(); ++i) bad |= !std::isfinite(hs.rec[i]);
        // the corrector's third reduction channel counts non-finite cells
        return bad ? FTSP_NONFINITE : FTSP_OK;
    }

    // ---- the step as a replayed CUDA graph ----
    // step() captures step_device() once and replays it: the step index,
    // noise key, adaptive scale and checkpoint schedule live on the device,
    // so every replay is the next step with fresh noise, bit-identical to
    // launching the kernels one by one.  Steps with injected noise, with
    // per-kernel profiling or with the learned preconditioner collecting or
    // in use launch directly; so do steps queued while the stream is being
    // captured by someone else (a replica batch).  Every setter that changes
    // what a step launches drops the graph.  The capture runs on a private
    // stream (the engine's own stream may be the legacy default stream,
    // which cannot be captured); the graph is launched on the engine's stream.
    cudaGraph_t sg_graph = nullptr;
    cudaGraphExec_t sg_exec = nullptr;
    cudaStream_t cap_stream = nullptr;
    long long sg_launches = 0;

    void drop_step_graph() override
    {
        if (sg_exec) cudaGraphExecDestroy(sg_exec);
        if (sg_graph) cudaGraphDestroy(sg_graph);
        sg_exec = nullptr;
        sg_graph = nullptr;
    }

    bool step_graph_usable()
    {
        if (!step_graph || noise_injected || profiling || lr.on_collect || lr.on_use) return false;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        FTSP_CUDA(cudaStreamIsCapturing(stream, &cs));
        return cs == cudaStreamCaptureStatusNone;
    }

    void capture_step()
    {
        if (!cap_stream) FTSP_CUDA(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
        const cudaStream_t own = stream;
        stream = cap_stream;
        launches = 0;
        FTSP_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
            step_device();
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(stream, &g);
            if (g) cudaGraphDestroy(g);
            stream = own;
            throw;
        }
        const cudaError_t e = cudaStreamEndCapture(stream, &sg_graph);
        stream = own;
        FTSP_CUDA(e);
        FTSP_CUDA(cudaGraphInstantiate(&sg_exec, sg_graph, 0));
        sg_launches = launches;
    }

    int step(double* Qbar, double* rec, double* dmax, bool sync) override
    {
        install_pending_fields();
        launches = 0;
        if (step_graph_usable()) {
            if (!sg_exec) capture_step();
            FTSP_CUDA(cudaGraphLaunch(sg_exec, stream));
            launches = sg_launches;
        } else {
            step_device();
        }
        if (!sync) return FTSP_OK;
        return read_status_impl(Qbar, rec, dmax);
    }

    int read_status_impl(double* Qbar, double* rec, double* dmax)
    {
        pull_scalars();
        if (Qbar)
            for (size_t s = 0; s < c.sp.size(); ++s) {
                Qbar[2 * s] = hs.Q[s].x;
                Qbar[2 * s + 1] = hs.Q[s].y;
            }
        if (rec) std::memcpy(rec, hs.rec, sizeof(double) * 2 * c.record_len());
        if (dmax) {
            for (int a = 0; a < c.nm; ++a) dmax[a] = std::fabs(0.5 * c.lambda[a]) * std::sqrt(std::max(0.0, hs.dmax[a]));
            dmax[c.nm] = std::fabs(0.5 * c.lpsi) * std::sqrt(std::max(0.0, hs.dmax[c.nm]));
        }
        int st = status_from_host();
        if (hs.corr[2] != 0.0 || hs.exhausted) st = FTSP_NONFINITE;
        return st;
    }

    int read_status(double* rec, double* dmax) override { return read_status_impl(nullptr, rec, dmax); }

    // Forward propagators of N identical segments in the field w (device,
    // complex128): q_1 = exp(-w), q_{s+1} = exp(-w) IFFT[Phi FFT[q_s] / V],
    // Phi = exp(-b^2 k^2 / 6); q_N to q_end (device), Q = mean(q_N) to the
    // host.  Uses the handle's class-table slot 0, G and the reduction
    // partials as scratch.
    Buf<T> phi_user;
    double phi_user_b = -1.0;

    void propagate_chain(const double2* w, int N, double bond, double2* q_end, double* Qh) override
    {
        if (sizeof(T) != 8) throw std::runtime_error("ftsp_propagate_chain needs a complex128 (FP64) handle");
        if (N < 1) throw std::runtime_error("ftsp_propagate_chain: N must be >= 1");
        if (!(bond > 0.0)) throw std::runtime_error("ftsp_propagate_chain: bond length must be positive");
        const size_t Vn = V_;
        V* Ep = E.p;
        const V* wp = reinterpret_cast<const V*>(w);
        foreach(Vn, [=] __device__(size_t i) {
            const V x = wp[i];
            Ep[i] = cexpT(-x.x, -x.y);
        });
        const int sum_m = c.m1 + c.m2 + c.m3;
        if (!phi_user.p) phi_user.alloc(sum_m);
        if (phi_user_b != bond) {
            std::vector<T> t;
            for (int i = 0; i < c.m1; ++i) { const double k = wave_number(i, c.m1, c.L[0]); t.push_back((T)std::exp(-bond * bond * k * k / 6.0)); }
            for (int i = 0; i < c.m2; ++i) { const double k = wave_number(i, c.m2, c.L[1]); t.push_back((T)std::exp(-bond * bond * k * k / 6.0)); }
            for (int i = 0; i < c.m3; ++i) { const double k = wave_number(i, c.m3, c.L[2]); t.push_back((T)std::exp(-bond * bond * k * k / 6.0)); }
            FTSP_CUDA(cudaMemcpyAsync(phi_user.p, t.data(), sizeof(T) * t.size(), cudaMemcpyHostToDevice, stream));
            FTSP_CUDA(cudaStreamSynchronize(stream));
            phi_user_b = bond;
        }
        V* qe = reinterpret_cast<V*>(q_end);
        double2* qpart = reinterpret_cast<double2*>(part.p);
        auto bond_op = [&]() {
            OpBond<T, true, false> ob{};
            ob.phix = phi_user.p;
            ob.phiy = phi_user.p + c.m1;
            ob.phiz = phi_user.p + c.m1 + c.m2;
            ob.kx = kx.p; ob.ky = ky.p; ob.kz = kz.p;
            ob.invV = (T)(1.0 / (double)Vn);
            return ob;
        };
        if (N == 1) {
            OpProp<T, FWD_SINGLE> op{};
            op.E = Ep; op.qstore = qe; op.partial = qpart;
            seg_pass<0, 0, FWD_SINGLE>(nullptr, nullptr, op);
        } else {
            OpProp<T, FWD_START> op0{};
            op0.E = Ep; op0.qstore = qe;
            seg_pass<0, -1, FWD_START>(nullptr, G.p, op0);
            for (int b = 0; b < N - 1; ++b) {
                bond_pass<-1, +1, true, false>(G.p, G.p, bond_op());
                if (b + 1 < N - 1) {
                    OpProp<T, FWD_MID> op{};
                    op.E = Ep; op.qstore = qe;
                    seg_pass<+1, -1, FWD_MID>(G.p, G.p, op);
                } else {
                    OpProp<T, FWD_LAST> op{};
                    op.E = Ep; op.qstore = qe; op.partial = qpart;
                    seg_pass<+1, 0, FWD_LAST>(G.p, nullptr, op);
                }
            }
        }
        double* out = reinterpret_cast<double*>(&ds->Q[0]);
        k_combine<false><<<2, COMBINE_THREADS, 0, stream>>>(part.p, seg_pass_ctas(), 2, out);
        ++launches;
        double q[2];
        FTSP_CUDA(cudaMemcpyAsync(q, out, sizeof(q), cudaMemcpyDeviceToHost, stream));
        FTSP_CUDA(cudaStreamSynchronize(stream));
        if (Qh) {
            Qh[0] = q[0] / (double)Vn;
            Qh[1] = q[1] / (double)Vn;
        }
    }

    long long restarts() override
    {
        pull_scalars();
        return hs.restarts;
    }

    bool restarts_exhausted() override
    {
        pull_scalars();
        return hs.exhausted != 0;
    }

    void views(ftsp_views* v) override
    {
        if (sizeof(T) != 8) throw std::runtime_error("state views are available for FP64 handles only");
        const size_t Vn = V_;
        v->omega = omega.p; v->psi = psi.p; v->omega_bar = omega_bar.p; v->psi_bar = psi_bar.p;
        v->rho_type = kC.p; v->rho_p = rho_p.p; v->rho_c = rho_c.p;
        v->rho_c_poly = kC.p + (size_t)c.M * Vn; v->rho_c_ion = kC.p + (size_t)(c.M + 1) * Vn;
        v->ion_rho = ion_rho.p; v->drift = drift.p; v->drift_bar = drift_bar.p; v->dpsi = dpsi.p; v->dpsi_bar = dpsi_bar.p;
    }
};


EngineBase* make_engine_f32(const HostCfg& c);
EngineBase* make_engine_f64(const HostCfg& c);

}  // namespace ftsp
