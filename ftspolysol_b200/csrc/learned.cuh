// Per-k-mode MLP of the learned semi-implicit preconditioner: forward,
// backward and Adam kernels (FP32, CUDA cores).
//
// The network maps the features of one wave vector k
//   x = (log(1 + k^2), log(1 + P_w(k)), log(1 + P_psi(k)), N / 50, lB, 10 c_salt)
// (P_w, P_psi: running spectral powers |FFT f|^2 / V of the first interaction
// mode and of psi) through two tanh layers of width 64 to z_f, f = 0..nout-1
// (one per Langevin field: interaction modes, then psi), and the linear-
// response coefficient of field f at k is G_f(k) = G_f^Debye(k) exp(z_f): the
// network corrects the analytic (homogeneous-state Debye) coefficient, which
// is exact wherever the chain response vanishes.  Training regresses z_f on
// log(G_emp,f(k) / G_f^Debye(k)), where G_emp = <Re(du conj(dw))> / <|dw|^2>
// is the least-squares linear response of the drift du to the field
// increment dw at k over the collected (force, increment) pairs:
//   L = sum_s sum_f m_sf (z_sf - t_sf)^2 / sum_sf m_sf.
// Parameter layout (floats): W1[H][NIN] b1[H] W2[H][H] b2[H] W3[nout][H] b3[nout].
//
// Shapes: one sample per thread.  The gradient kernel keeps, for the 128
// samples of a CTA, the layer inputs and back-propagated deltas in shared
// memory and forms the weight gradients as fixed-order sums over those
// samples (per-CTA partials, then a fixed-order sum over CTAs in the Adam
// kernel), so a training run is bit-reproducible.
#pragma once

#include <cuda_runtime.h>

namespace ftsp {
namespace mlp {

constexpr int NIN = 6;
constexpr int H = 64;
constexpr int NOUT_MAX = 4;
constexpr int GRAD_THREADS = 128;

__host__ __device__ constexpr int n_params(int nout) { return H * NIN + H + H * H + H + nout * H + nout; }
__host__ __device__ constexpr int off_b1() { return H * NIN; }
__host__ __device__ constexpr int off_w2() { return H * NIN + H; }
__host__ __device__ constexpr int off_b2() { return H * NIN + H + H * H; }
__host__ __device__ constexpr int off_w3() { return H * NIN + H + H * H + H; }
__host__ __device__ constexpr int off_b3(int nout) { return off_w3() + nout * H; }

// Forward pass of one sample (inference) with the weights in shared
// memory: the first hidden layer in registers, the second streamed into the
// outputs.
__device__ __forceinline__ void forward_eval(const float* __restrict__ w, int nout, const float* x, float* z)
{
    float h1[H];
#pragma unroll
    for (int i = 0; i < H; ++i) {
        float a = w[off_b1() + i];
#pragma unroll
        for (int k = 0; k < NIN; ++k) a = fmaf(w[i * NIN + k], x[k], a);
        h1[i] = tanhf(a);
    }
#pragma unroll
    for (int f = 0; f < NOUT_MAX; ++f) z[f] = f < nout ? w[off_b3(nout) + f] : 0.0f;
    for (int j = 0; j < H; ++j) {
        float a = w[off_b2() + j];
        const float* row = w + off_w2() + j * H;
#pragma unroll
        for (int i = 0; i < H; ++i) a = fmaf(row[i], h1[i], a);
        const float h = tanhf(a);
#pragma unroll
        for (int f = 0; f < NOUT_MAX; ++f)
            if (f < nout) z[f] = fmaf(w[off_w3() + f * H + j], h, z[f]);
    }
}

__device__ __forceinline__ void load_weights(float* sw, const float* __restrict__ w, int np)
{
    for (int i = threadIdx.x; i < np; i += blockDim.x) sw[i] = w[i];
    __syncthreads();
}

// Inference over n items: feat(i, x) fills the features of item i (returns
// false to skip it), out(i, z) consumes the outputs.  Dynamic shared memory:
// n_params(nout) floats.
template <class Feat, class Out>
__global__ void __launch_bounds__(128) k_eval(size_t n, const float* __restrict__ w, int nout, Feat feat, Out out)
{
    extern __shared__ float sw[];
    load_weights(sw, w, n_params(nout));
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float x[NIN], z[NOUT_MAX];
        if (!feat(i, x)) continue;
        forward_eval(sw, nout, x, z);
        out(i, z);
    }
}

// Per-sample rows in shared memory are padded to an odd stride, so that both
// the per-sample phase (thread t, element i) and the reduction phase (thread
// i, sample q) read distinct banks.
constexpr int HS = H + 1;
constexpr int XS = NIN + 1;
constexpr int ZS = NOUT_MAX + 1;

__host__ __device__ constexpr int grad_smem_floats(int nout)
{
    return n_params(nout) + GRAD_THREADS * (XS + 4 * HS + ZS);
}

// Loss and gradient partials of one batch: CTA b takes samples
// [b * 128, b * 128 + 128); sample(s, x, t, m) fills the features, targets
// and target weights of sample s (m = 0 drops an output).  Writes
// partial[b][0 .. np) = sum_s sum_f 2 m (z - t) dz/dw (unnormalised) and
// lpart[b] = (sum m (z - t)^2, sum m).  Dynamic shared memory:
// grad_smem_floats(nout) floats.
template <class Sample>
__global__ void __launch_bounds__(GRAD_THREADS) k_grad(int n_samples, const float* __restrict__ w, int nout, Sample sample,
                                                        float* __restrict__ partial, double* __restrict__ lpart)
{
    extern __shared__ float sm[];
    const int np = n_params(nout);
    float* sw = sm;
    float* sx = sw + np;                        // [128][XS]
    float* sh1 = sx + GRAD_THREADS * XS;        // [128][HS] layer-1 activations
    float* sd1 = sh1 + GRAD_THREADS * HS;       // [128][HS] delta of the layer-1 pre-activation
    float* sh2 = sd1 + GRAD_THREADS * HS;       // [128][HS] layer-2 activations
    float* sd2 = sh2 + GRAD_THREADS * HS;       // [128][HS] delta of the layer-2 pre-activation
    float* sdz = sd2 + GRAD_THREADS * HS;       // [128][ZS] output deltas
    __shared__ double sl[2][GRAD_THREADS];
    load_weights(sw, w, np);

    const int t = threadIdx.x;
    const int s = blockIdx.x * GRAD_THREADS + t;
    float x[NIN], tg[NOUT_MAX], mk[NOUT_MAX], z[NOUT_MAX];
#pragma unroll
    for (int k = 0; k < NIN; ++k) x[k] = 0.0f;
#pragma unroll
    for (int f = 0; f < NOUT_MAX; ++f) tg[f] = mk[f] = 0.0f;
    if (s < n_samples) sample(s, x, tg, mk);
    float* h1 = sh1 + t * HS;
    float* h2 = sh2 + t * HS;
    float* d1 = sd1 + t * HS;
    float* d2 = sd2 + t * HS;
    // forward
    for (int i = 0; i < H; ++i) {
        float a = sw[off_b1() + i];
#pragma unroll
        for (int k = 0; k < NIN; ++k) a = fmaf(sw[i * NIN + k], x[k], a);
        h1[i] = tanhf(a);
    }
#pragma unroll
    for (int f = 0; f < NOUT_MAX; ++f) z[f] = f < nout ? sw[off_b3(nout) + f] : 0.0f;
    for (int j = 0; j < H; ++j) {
        float a = sw[off_b2() + j];
        const float* row = sw + off_w2() + j * H;
#pragma unroll 16
        for (int i = 0; i < H; ++i) a = fmaf(row[i], h1[i], a);
        const float h = tanhf(a);
        h2[j] = h;
#pragma unroll
        for (int f = 0; f < NOUT_MAX; ++f)
            if (f < nout) z[f] = fmaf(sw[off_w3() + f * H + j], h, z[f]);
    }
    // loss and output deltas
    double l = 0.0, msum = 0.0;
    float dz[NOUT_MAX];
#pragma unroll
    for (int f = 0; f < NOUT_MAX; ++f) {
        const float e = f < nout ? z[f] - tg[f] : 0.0f;
        const float m = f < nout ? mk[f] : 0.0f;
        dz[f] = 2.0f * m * e;
        l += (double)m * (double)e * (double)e;
        msum += (double)m;
        sdz[t * ZS + f] = dz[f];
    }
    // back-propagation
    for (int j = 0; j < H; ++j) {
        float a = 0.0f;
#pragma unroll
        for (int f = 0; f < NOUT_MAX; ++f)
            if (f < nout) a = fmaf(dz[f], sw[off_w3() + f * H + j], a);
        d2[j] = a * (1.0f - h2[j] * h2[j]);
    }
    for (int i = 0; i < H; ++i) {
        float a = 0.0f;
#pragma unroll 16
        for (int j = 0; j < H; ++j) a = fmaf(d2[j], sw[off_w2() + j * H + i], a);
        d1[i] = a * (1.0f - h1[i] * h1[i]);
    }
#pragma unroll
    for (int k = 0; k < NIN; ++k) sx[t * XS + k] = x[k];
    sl[0][t] = l;
    sl[1][t] = msum;
    __syncthreads();

    // fixed-order sums over the CTA's samples
    float* out = partial + (size_t)blockIdx.x * np;
    for (int p = t; p < np; p += GRAD_THREADS) {
        float g = 0.0f;
        if (p < off_b1()) {                       // W1[i][k]
            const int i = p / NIN, k = p - i * NIN;
            for (int q = 0; q < GRAD_THREADS; ++q) g = fmaf(sd1[q * HS + i], sx[q * XS + k], g);
        } else if (p < off_w2()) {                // b1[i]
            const int i = p - off_b1();
            for (int q = 0; q < GRAD_THREADS; ++q) g += sd1[q * HS + i];
        } else if (p < off_b2()) {                // W2[j][i]
            const int r = p - off_w2(), j = r / H, i = r - j * H;
            for (int q = 0; q < GRAD_THREADS; ++q) g = fmaf(sd2[q * HS + j], sh1[q * HS + i], g);
        } else if (p < off_w3()) {                // b2[j]
            const int j = p - off_b2();
            for (int q = 0; q < GRAD_THREADS; ++q) g += sd2[q * HS + j];
        } else if (p < off_b3(nout)) {            // W3[f][j]
            const int r = p - off_w3(), f = r / H, j = r - f * H;
            for (int q = 0; q < GRAD_THREADS; ++q) g = fmaf(sdz[q * ZS + f], sh2[q * HS + j], g);
        } else {                                  // b3[f]
            const int f = p - off_b3(nout);
            for (int q = 0; q < GRAD_THREADS; ++q) g += sdz[q * ZS + f];
        }
        out[p] = g;
    }
    if (t == 0) {
        double a = 0.0, b = 0.0;
        for (int q = 0; q < GRAD_THREADS; ++q) {
            a += sl[0][q];
            b += sl[1][q];
        }
        lpart[2 * blockIdx.x] = a;
        lpart[2 * blockIdx.x + 1] = b;
    }
}

// Sums the per-CTA partials in CTA order and normalises by the batch's total
// target weight: grad[p] = sum_b partial[b][p] / sum m, loss = (sum m (z-t)^2
// / sum m, sum m).  With apply != 0 also takes one Adam step (Kingma & Ba,
// 2015, with bias correction at step t) on w with the moments m1, m2.
struct AdamArgs {
    float lr, beta1, beta2, eps;
    int t;
    int apply;
};

static __global__ void k_reduce_adam(int np, int nparts, const float* __restrict__ partial, const double* __restrict__ lpart,
                                     float* __restrict__ grad, double* __restrict__ loss, float* __restrict__ w,
                                     float* __restrict__ m1, float* __restrict__ m2, AdamArgs a)
{
    __shared__ double norm;
    if (threadIdx.x == 0) {
        double l = 0.0, ms = 0.0;
        for (int b = 0; b < nparts; ++b) {
            l += lpart[2 * b];
            ms += lpart[2 * b + 1];
        }
        norm = ms > 0.0 ? 1.0 / ms : 0.0;
        if (blockIdx.x == 0 && loss) {
            loss[0] = l * norm;
            loss[1] = ms;
        }
    }
    __syncthreads();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    float g = 0.0f;
    for (int b = 0; b < nparts; ++b) g += partial[(size_t)b * np + p];
    g = (float)((double)g * norm);
    if (grad) grad[p] = g;
    if (a.apply) {
        const float mm = a.beta1 * m1[p] + (1.0f - a.beta1) * g;
        const float vv = a.beta2 * m2[p] + (1.0f - a.beta2) * g * g;
        m1[p] = mm;
        m2[p] = vv;
        const float mh = mm / (1.0f - powf(a.beta1, (float)a.t));
        const float vh = vv / (1.0f - powf(a.beta2, (float)a.t));
        w[p] -= a.lr * mh / (sqrtf(vh) + a.eps);
    }
}

}  // namespace mlp
}  // namespace ftsp
