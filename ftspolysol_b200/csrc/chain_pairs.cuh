// Densities and connectivity stress of a mirror-symmetric chain from its
// forward sweep alone.
//
// The reference propagates q (head to tail) and q-dagger (tail to head) with
// the same segment step (polymerSpecies::propagate_chain, polymer.cu:402-416)
// and forms the segment densities from the products q(s) q-dagger(s) e^{+W_s}
// (accumulate_species_densities, polymer.cu:434-447); its connectivity stress
// pairs q(s) with the bond-filtered e^{+W} q-dagger (stress.cu:225-250).
// When the segment classes read the same from both ends (cls[s] ==
// cls[N-1-s]; a class is a monomer type with a valence, so the segment
// fields W_s + i z_s psi agree) and so do the bonds (bond b and bond N-2-b
// have one length), the tail-to-head recursion is the head-to-tail one in
// mirror order, so q-dagger(s) = q(N-1-s) exactly.  Then:
//
//   rho_s  = (n/V)/Q  q(s) q(N-1-s) e^{+W_s}
//          = factor 2^{aF[s] + aF[N-1-s] - aF[N-1]}  u(s) u(N-1-s) E_s
//
// with u(s) = e^{+W_s} q(s) (the inverse transform of the bond pass, before
// the segment factor E_s = e^{-W_s}), stored renormalised by 2^{-aF[s]}
// (u(0) = 1 is not stored), and the backward bond-pass spectrum
// DFT_{+}(q-dagger(b+1))(k) = DFT_{-}(q(N-2-b))(-k), so the connectivity
// stress of bond b is
//
//   S_b = b_b^2 2^{aF[b] + aF[N-2-b] - aF[N-1]}
//         sum_k k_a k_b Phi_b(k) F_b(k) F_{N-2-b}(-k)
//
// (F_s the stored forward spectrum of the renormalised q(s)).  Mirror pairs
// contribute equal terms, so each pair is read once: the density sums
// segment pairs (s, N-1-s), weight 2 (1 for the middle segment), and the
// stress kernel sums bond pairs (b, N-2-b) over conjugate grid points
// {k, -k} together: the two bonds of a pair give the same product
//   t = F_b(k) F_q(-k) + F_q(k) F_b(-k)
// at k and at -k, which then take the k_a k_b Phi of their own grid point
// (so the Nyquist planes, where the k table is not odd, are summed exactly
// as the two sweeps sum them); weight 1/2 for the middle bond.
//
// Both kernels are bandwidth-bound elementwise passes: the density reads
// the N-1 stored u fields once plus one class table per run and
// read-modify-writes the density channels; the stress reads the N-1 stored
// spectra once.  They replace the backward sweep (N-1 bond passes and N
// segment passes of 6-8 complex values per point).
#pragma once
#include "passes.cuh"

namespace ftsp {

// Consecutive pairs that share a class (density: segment class, stress:
// bond class).  Density runs are ordered by density channel so that every
// channel is flushed once.
struct PairRun {
    int j0, j1;     // pair range [j0, j1)
    int cls;        // segment class / bond class
    int type;       // density channel of the run's segments (density)
    double z;       // valence of the run's segments (density)
};

struct PairTable {
    const int2* pair;       // (s, p), s <= p
    const double* weight;   // density: 2 (s < p) or 1; stress: b^2 (b < q) or b^2 / 2
    const PairRun* run;
    int npairs, nruns;
};

// Dynamic shared memory of the pair kernels: per-pair scales, pairs, runs,
// and (stress) the block-sum scratch.
inline size_t pair_smem(int npairs, int nruns, int threads)
{
    return sizeof(double) * (size_t)npairs + sizeof(int2) * (size_t)npairs + sizeof(PairRun) * (size_t)nruns +
           sizeof(double) * 12 * (size_t)((threads + 31) / 32);
}

// Copies the tables to shared memory with the per-pair scale
// weight * 2^{aF[s] + aF[p] - aF[N-1]} (exponents written by this
// evaluation's forward sweep; eF null: no renormalisation).
__device__ __forceinline__ void pair_tables(const PairTable& tb, const int* eF, int N, double*& sc, int2*& sp,
                                            PairRun*& sr, double*& scratch)
{
    extern __shared__ __align__(16) unsigned char pair_smem_raw[];
    sc = reinterpret_cast<double*>(pair_smem_raw);
    sp = reinterpret_cast<int2*>(sc + tb.npairs);
    sr = reinterpret_cast<PairRun*>(sp + tb.npairs);
    scratch = reinterpret_cast<double*>(sr + tb.nruns);
    const int eN = eF ? eF[N - 1] : 0;
    for (int j = threadIdx.x; j < tb.npairs; j += blockDim.x) {
        const int2 pr = tb.pair[j];
        sp[j] = pr;
        sc[j] = eF ? ldexp(tb.weight[j], eF[pr.x] + eF[pr.y] - eN) : tb.weight[j];
    }
    for (int r = threadIdx.x; r < tb.nruns; r += blockDim.x) sr[r] = tb.run[r];
    __syncthreads();
}

// rho[type] += factor sum_pairs scale u(s) u(p) E_cls and, when rho_charge
// is given, rho_charge += factor sum_pairs z scale u(s) u(p) E_cls.  FP64
// accumulation per grid point; one read-modify-write per channel.
template <typename T>
__global__ void __launch_bounds__(256) k_pair_density(size_t n, PairTable tb, const cplx<T>* __restrict__ u,
                                                      const cplx<T>* __restrict__ E, const int* __restrict__ eF,
                                                      int N, const double2* __restrict__ factor, cplx<T>* rho,
                                                      cplx<T>* rho_charge)
{
    using V = cplx<T>;
    pdl_wait();
    double* sc;
    int2* sp;
    PairRun* sr;
    double* scratch;
    pair_tables(tb, eF, N, sc, sp, sr, scratch);
    const double2 fc = *factor;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double ax = 0.0, ay = 0.0, cx = 0.0, cy = 0.0;
        for (int r = 0; r < tb.nruns; ++r) {
            const PairRun R = sr[r];
            const V e = E[(size_t)R.cls * n + i];
            double sx = 0.0, sy = 0.0;
#pragma unroll 4
            for (int j = R.j0; j < R.j1; ++j) {
                const int2 pr = sp[j];
                const V us = pr.x == 0 ? mkc<V>(T(1), T(0)) : u[(size_t)pr.x * n + i];
                const V up = u[(size_t)pr.y * n + i];
                const V t = cmul(us, up);
                sx += sc[j] * (double)t.x;
                sy += sc[j] * (double)t.y;
            }
            const double wx = sx * (double)e.x - sy * (double)e.y;
            const double wy = sx * (double)e.y + sy * (double)e.x;
            ax += wx;
            ay += wy;
            cx += R.z * wx;
            cy += R.z * wy;
            if (r + 1 == tb.nruns || sr[r + 1].type != R.type) {
                V* d = rho + (size_t)R.type * n + i;
                const V o = *d;
                *d = mkc<V>(o.x + (T)(ax * fc.x - ay * fc.y), o.y + (T)(ax * fc.y + ay * fc.x));
                ax = ay = 0.0;
            }
        }
        if (rho_charge) {
            const V o = rho_charge[i];
            rho_charge[i] = mkc<V>(o.x + (T)(cx * fc.x - cy * fc.y), o.y + (T)(cx * fc.y + cy * fc.x));
        }
    }
    pdl_trigger();
}

// The same density with PT consecutive grid points per thread, read as
// 16-byte vectors (complex64: PT = 4, two float4 per field; complex128:
// PT = 2, two double2), so a warp reads 1 KB contiguous per stored field
// instead of 256 B.  Needs n % PT == 0.
template <typename T>
struct PairVec;
template <>
struct PairVec<float> {
    static constexpr int PT = 4;
    __device__ static void load(const cplx<float>* p, cplx<float> (&o)[4])
    {
        const float4 a = __ldg(reinterpret_cast<const float4*>(p));
        const float4 b = __ldg(reinterpret_cast<const float4*>(p) + 1);
        o[0] = mkc<cplx<float>>(a.x, a.y);
        o[1] = mkc<cplx<float>>(a.z, a.w);
        o[2] = mkc<cplx<float>>(b.x, b.y);
        o[3] = mkc<cplx<float>>(b.z, b.w);
    }
    // read-modify-write operands (the density channels): plain loads
    __device__ static void load_rw(const cplx<float>* p, cplx<float> (&o)[4])
    {
        const float4 a = reinterpret_cast<const float4*>(p)[0];
        const float4 b = reinterpret_cast<const float4*>(p)[1];
        o[0] = mkc<cplx<float>>(a.x, a.y);
        o[1] = mkc<cplx<float>>(a.z, a.w);
        o[2] = mkc<cplx<float>>(b.x, b.y);
        o[3] = mkc<cplx<float>>(b.z, b.w);
    }
    __device__ static void store(cplx<float>* p, const cplx<float> (&o)[4])
    {
        reinterpret_cast<float4*>(p)[0] = make_float4(o[0].x, o[0].y, o[1].x, o[1].y);
        reinterpret_cast<float4*>(p)[1] = make_float4(o[2].x, o[2].y, o[3].x, o[3].y);
    }
};
template <>
struct PairVec<double> {
    static constexpr int PT = 2;
    __device__ static void load(const cplx<double>* p, cplx<double> (&o)[2])
    {
        o[0] = p[0];
        o[1] = p[1];
    }
    __device__ static void load_rw(const cplx<double>* p, cplx<double> (&o)[2]) { load(p, o); }
    __device__ static void store(cplx<double>* p, const cplx<double> (&o)[2])
    {
        p[0] = o[0];
        p[1] = o[1];
    }
};

template <typename T>
__global__ void __launch_bounds__(256) k_pair_density_vec(size_t n, PairTable tb, const cplx<T>* __restrict__ u,
                                                          const cplx<T>* __restrict__ E, const int* __restrict__ eF,
                                                          int N, const double2* __restrict__ factor, cplx<T>* rho,
                                                          cplx<T>* rho_charge)
{
    using V = cplx<T>;
    using PV = PairVec<T>;
    constexpr int PT = PV::PT;
    pdl_wait();
    double* sc;
    int2* sp;
    PairRun* sr;
    double* scratch;
    pair_tables(tb, eF, N, sc, sp, sr, scratch);
    const double2 fc = *factor;
    const size_t ng = n / PT;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += stride) {
        const size_t i = g * PT;
        double ax[PT], ay[PT], cx[PT], cy[PT];
#pragma unroll
        for (int k = 0; k < PT; ++k) ax[k] = ay[k] = cx[k] = cy[k] = 0.0;
        for (int r = 0; r < tb.nruns; ++r) {
            const PairRun R = sr[r];
            V e[PT];
            PV::load(E + (size_t)R.cls * n + i, e);
            double sx[PT], sy[PT];
#pragma unroll
            for (int k = 0; k < PT; ++k) sx[k] = sy[k] = 0.0;
#pragma unroll 4
            for (int j = R.j0; j < R.j1; ++j) {
                const int2 pr = sp[j];
                V us[PT], up[PT];
                if (pr.x == 0) {
#pragma unroll
                    for (int k = 0; k < PT; ++k) us[k] = mkc<V>(T(1), T(0));
                } else {
                    PV::load(u + (size_t)pr.x * n + i, us);
                }
                PV::load(u + (size_t)pr.y * n + i, up);
                const double w = sc[j];
#pragma unroll
                for (int k = 0; k < PT; ++k) {
                    const V t = cmul(us[k], up[k]);
                    sx[k] += w * (double)t.x;
                    sy[k] += w * (double)t.y;
                }
            }
#pragma unroll
            for (int k = 0; k < PT; ++k) {
                const double wx = sx[k] * (double)e[k].x - sy[k] * (double)e[k].y;
                const double wy = sx[k] * (double)e[k].y + sy[k] * (double)e[k].x;
                ax[k] += wx;
                ay[k] += wy;
                cx[k] += R.z * wx;
                cy[k] += R.z * wy;
            }
            if (r + 1 == tb.nruns || sr[r + 1].type != R.type) {
                V* d = rho + (size_t)R.type * n + i;
                V o[PT];
                PV::load_rw(d, o);
#pragma unroll
                for (int k = 0; k < PT; ++k) {
                    o[k] = mkc<V>(o[k].x + (T)(ax[k] * fc.x - ay[k] * fc.y), o[k].y + (T)(ax[k] * fc.y + ay[k] * fc.x));
                    ax[k] = ay[k] = 0.0;
                }
                PV::store(d, o);
            }
        }
        if (rho_charge) {
            V o[PT];
            PV::load_rw(rho_charge + i, o);
#pragma unroll
            for (int k = 0; k < PT; ++k)
                o[k] = mkc<V>(o[k].x + (T)(cx[k] * fc.x - cy[k] * fc.y), o[k].y + (T)(cx[k] * fc.y + cy[k] * fc.x));
            PV::store(rho_charge + i, o);
        }
    }
    pdl_trigger();
}

// partial[cta][c] += factor sum_k k_a k_b Phi(k) sum_pairs scale t(k), the
// six components (xx, yy, zz, xy, xz, yz) in the layout of the backward
// bond pass, so the same fixed-order combine reads them.  Launched with as
// many CTAs as that pass has.
template <typename T>
__global__ void __launch_bounds__(256) k_pair_stress(int m1, int m2, int m3, PairTable tb,
                                                     const cplx<T>* __restrict__ F, const T* __restrict__ phi,
                                                     const double* __restrict__ kx, const double* __restrict__ ky,
                                                     const double* __restrict__ kz, const int* __restrict__ eF, int N,
                                                     const double2* __restrict__ factor, double2* partial)
{
    using V = cplx<T>;
    pdl_wait();
    double* sc;
    int2* sp;
    PairRun* sr;
    double* scratch;
    pair_tables(tb, eF, N, sc, sp, sr, scratch);
    const size_t n = (size_t)m1 * m2 * m3;
    const int sum_m = m1 + m2 + m3;
    double acc[12];
#pragma unroll
    for (int c = 0; c < 12; ++c) acc[c] = 0.0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int z = (int)(i % m3);
        const size_t rest = i / m3;
        const int y = (int)(rest % m2), x = (int)(rest / m2);
        const int nx = x ? m1 - x : 0, ny = y ? m2 - y : 0, nz = z ? m3 - z : 0;
        const size_t ni = ((size_t)nx * m2 + ny) * m3 + nz;
        if (ni < i) continue;   // the pair {k, -k} is summed by the thread of its lower index
        double s0x = 0.0, s0y = 0.0, s1x = 0.0, s1y = 0.0;   // at k and at -k
        for (int r = 0; r < tb.nruns; ++r) {
            const PairRun R = sr[r];
            const T* ph = phi + (size_t)R.cls * sum_m;
            const double p0 = (double)(ph[x] * ph[m1 + y] * ph[m1 + m2 + z]);
            const double p1 = (double)(ph[nx] * ph[m1 + ny] * ph[m1 + m2 + nz]);
            double tx = 0.0, ty = 0.0;
#pragma unroll 2
            for (int j = R.j0; j < R.j1; ++j) {
                const int2 pr = sp[j];
                const V* Fb = F + (size_t)pr.x * n;
                const V* Fq = F + (size_t)pr.y * n;
                const V t = cadd(cmul(Fb[i], Fq[ni]), cmul(Fq[i], Fb[ni]));
                tx += sc[j] * (double)t.x;
                ty += sc[j] * (double)t.y;
            }
            s0x += p0 * tx;
            s0y += p0 * ty;
            s1x += p1 * tx;
            s1y += p1 * ty;
        }
        {
            const double ax = kx[x], ay = ky[y], az = kz[z];
            const double kk[6] = {ax * ax, ay * ay, az * az, ax * ay, ax * az, ay * az};
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                acc[2 * c] += kk[c] * s0x;
                acc[2 * c + 1] += kk[c] * s0y;
            }
        }
        if (ni != i) {
            const double ax = kx[nx], ay = ky[ny], az = kz[nz];
            const double kk[6] = {ax * ax, ay * ay, az * az, ax * ay, ax * az, ay * az};
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                acc[2 * c] += kk[c] * s1x;
                acc[2 * c + 1] += kk[c] * s1y;
            }
        }
    }
    pdl_trigger();
    block_sum<12>(acc, scratch);
    if (threadIdx.x == 0) {
        const double2 fc = *factor;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double sr_ = acc[2 * c], si_ = acc[2 * c + 1];
            double2 o = partial[(size_t)blockIdx.x * 6 + c];
            o.x += sr_ * fc.x - si_ * fc.y;
            o.y += sr_ * fc.y + si_ * fc.x;
            partial[(size_t)blockIdx.x * 6 + c] = o;
        }
    }
}

}  // namespace ftsp
