/* FP64 CPU oracle of the FTSPolySol complex-Langevin step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker): see ftsp_oracle.h for who may use
 * it.  Every routine below names the reference routine it restates; the
 * operation order follows the reference so that the only differences from
 * the reference's CUDA build are floating-point roundoff (cuFFT against the
 * mixed-radix transform here, tree against pairwise reductions).
 */
#include "ftsp_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double x, y; } cd;

static const double PI = 3.141592653589793238462643383279502884;

/* ---- complex helpers: common.h:79-201 ---- */
static inline cd mk(double x, double y) { cd z; z.x = x; z.y = y; return z; }
static inline cd cadd(cd a, cd b) { return mk(a.x + b.x, a.y + b.y); }
static inline cd csub(cd a, cd b) { return mk(a.x - b.x, a.y - b.y); }
static inline cd cmul(cd a, cd b) { return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
static inline cd cscale(cd z, double s) { return mk(s * z.x, s * z.y); }
static inline cd cinv(cd z) /* common.h:146-157 */
{
    const double ax = fabs(z.x), ay = fabs(z.y);
    if (ax >= ay) {
        const double r = z.y / z.x, den = z.x * (1.0 + r * r);
        return mk(1.0 / den, -r / den);
    }
    const double r = z.x / z.y, den = z.y * (1.0 + r * r);
    return mk(r / den, -1.0 / den);
}
static inline cd cexp_(cd z) /* common.h:188-192 */
{
    const double r = exp(z.x);
    return mk(r * cos(z.y), r * sin(z.y));
}
static inline cd cneglog(cd z) /* common.h:194-198 */
{
    const double r = sqrt(z.x * z.x + z.y * z.y);
    return mk(-log(r), -atan2(z.y, z.x));
}

/* ---- FFT: own mixed-radix Stockham transform, cuFFT conventions ---- */
typedef struct {
    int n;
    int nr;
    int rad[40];
    cd* tw; /* tw[j] = exp(-2 pi i j / n) */
} plan1;

static void plan1_init(plan1* p, int n)
{
    p->n = n;
    p->nr = 0;
    int r = n;
    while (r % 4 == 0) { p->rad[p->nr++] = 4; r /= 4; }
    while (r % 2 == 0) { p->rad[p->nr++] = 2; r /= 2; }
    while (r % 3 == 0) { p->rad[p->nr++] = 3; r /= 3; }
    while (r % 5 == 0) { p->rad[p->nr++] = 5; r /= 5; }
    for (int f = 7; r > 1; f += 2) {
        while (r % f == 0) { p->rad[p->nr++] = f; r /= f; }
    }
    p->tw = (cd*)malloc(sizeof(cd) * (size_t)n);
    for (int j = 0; j < n; ++j) {
        const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)j / (long double)n;
        p->tw[j] = mk((double)cosl(ang), (double)sinl(ang));
    }
}

static void plan1_free(plan1* p) { free(p->tw); p->tw = NULL; }

static inline cd twid(const plan1* p, long idx, int sign)
{
    idx %= p->n;
    cd w = p->tw[idx];
    if (sign > 0) w.y = -w.y;
    return w;
}

/* x: data (in/out), y: scratch of length n. */
static void fft1d(const plan1* p, cd* x, cd* y, int sign)
{
    const int n = p->n;
    cd* src = x;
    cd* dst = y;
    int span = 1;
    cd u[64], v[64];
    for (int st = 0; st < p->nr; ++st) {
        const int R = p->rad[st];
        const int m = n / R;
        const long tstep = n / (R * span);
        for (int i = 0; i < m; ++i) {
            const int k = i % span;
            for (int t = 0; t < R; ++t) {
                cd val = src[i + t * m];
                if (t && k) val = cmul(val, twid(p, (long)t * k * tstep, sign));
                u[t] = val;
            }
            if (R == 2) {
                v[0] = cadd(u[0], u[1]);
                v[1] = csub(u[0], u[1]);
            } else if (R == 4) {
                const cd a0 = cadd(u[0], u[2]), a1 = csub(u[0], u[2]);
                const cd b0 = cadd(u[1], u[3]), b1 = csub(u[1], u[3]);
                /* multiply b1 by exp(sign*i*pi/2) = sign*i */
                const cd jb1 = sign < 0 ? mk(b1.y, -b1.x) : mk(-b1.y, b1.x);
                v[0] = cadd(a0, b0);
                v[2] = csub(a0, b0);
                v[1] = cadd(a1, jb1);
                v[3] = csub(a1, jb1);
            } else {
                const long base_step = n / R;
                for (int t = 0; t < R; ++t) {
                    cd acc = u[0];
                    for (int j = 1; j < R; ++j) acc = cadd(acc, cmul(u[j], twid(p, (long)((j * t) % R) * base_step, sign)));
                    v[t] = acc;
                }
            }
            const int base = (i - k) * R + k;
            for (int t = 0; t < R; ++t) dst[base + t * span] = v[t];
        }
        span *= R;
        cd* tmp = src;
        src = dst;
        dst = tmp;
    }
    if (src != x) memcpy(x, src, sizeof(cd) * (size_t)n);
}

typedef struct {
    int m1, m2, m3;
    plan1 p1, p2, p3;
} plan3;

static void plan3_init(plan3* p, int m1, int m2, int m3)
{
    p->m1 = m1; p->m2 = m2; p->m3 = m3;
    plan1_init(&p->p1, m1);
    plan1_init(&p->p2, m2);
    plan1_init(&p->p3, m3);
}

static void plan3_free(plan3* p)
{
    plan1_free(&p->p1);
    plan1_free(&p->p2);
    plan1_free(&p->p3);
}

static void fft3d(const plan3* p, cd* data, int sign)
{
    const int m1 = p->m1, m2 = p->m2, m3 = p->m3;
    const int mx = m1 > m2 ? (m1 > m3 ? m1 : m3) : (m2 > m3 ? m2 : m3);
#pragma omp parallel
    {
        cd* line = (cd*)malloc(sizeof(cd) * (size_t)mx);
        cd* scratch = (cd*)malloc(sizeof(cd) * (size_t)mx);
        /* z (contiguous) */
#pragma omp for schedule(static)
        for (long r = 0; r < (long)m1 * m2; ++r) fft1d(&p->p3, data + r * m3, scratch, sign);
        /* y */
#pragma omp for schedule(static)
        for (long r = 0; r < (long)m1 * m3; ++r) {
            const long x = r / m3, z = r % m3;
            cd* base = data + x * (long)m2 * m3 + z;
            for (int y = 0; y < m2; ++y) line[y] = base[(long)y * m3];
            fft1d(&p->p2, line, scratch, sign);
            for (int y = 0; y < m2; ++y) base[(long)y * m3] = line[y];
        }
        /* x */
#pragma omp for schedule(static)
        for (long r = 0; r < (long)m2 * m3; ++r) {
            cd* base = data + r;
            for (int x = 0; x < m1; ++x) line[x] = base[(long)x * m2 * m3];
            fft1d(&p->p1, line, scratch, sign);
            for (int x = 0; x < m1; ++x) base[(long)x * m2 * m3] = line[x];
        }
        free(line);
        free(scratch);
    }
}

void oracle_fft3d(int m1, int m2, int m3, double* data, int sign)
{
    plan3 p;
    plan3_init(&p, m1, m2, m3);
    fft3d(&p, (cd*)data, sign);
    plan3_free(&p);
}

/* ---- state: the reference's deviceState (deviceState.h:6-48) ---- */
typedef struct {
    double count, valence, smear;
} ion_sp;

struct oracle_state {
    oracle_config c;
    int size;
    double volume;
    int elec;
    plan3 plan;
    int Nmax;
    int n_species;
    double* num_chains;
    int* N;
    int* seg_off;     /* segment offset of each species */
    int* seg_type;
    double* seg_charge;
    double* seg_bond;
    int* bond_off;    /* bond-kernel offset of each species (polymer.cu:294-301) */
    int total_bonds;
    ion_sp* ions;
    double* mode_coeff;
    cd* mode_gamma;
    double* mode_O;
    double* mode_lambda;
    /* fields */
    cd *omega, *omega_bar, *omega_s, *drift, *drift_bar;
    double* eta_omega;
    cd *psi, *psi_bar, *psi_s, *dpsi, *dpsi_bar;
    double* etaPsi;
    cd *W_type_s, *rho_type, *rho_c, *rho_c_poly, *rho_c_ion, *rho_c_old, *rho_p;
    cd *W, *exp_mW, *exp_W, *qF, *qB;
    cd *ion_psi, *ion_boltzmann, *ion_charge, *ion_rho;
    cd *obs_a, *obs_b, *obs_c;
    cd *s_a, *s_b, *s_c, *s_dfield, *s_dpsi;     /* stress scratch */
    cd *iso_b, *iso_c, *iso_a;                    /* isotropic pressure scratch */
    double *Gamma, *PHI, *k2, *ion_kernels;
    double *kab, *minus_kab;
    double mode_term[6];
};

static cd* calloc_c(size_t n) { return (cd*)calloc(n ? n : 1, sizeof(cd)); }
static double* calloc_d(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

static int spectral_mode(int i, int m) { return i > m / 2 ? i - m : i; }
static double wave_number(int i, int m, double L) { return 2.0 * PI * spectral_mode(i, m) / L; }

int oracle_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* spectral::build_kernels (spectral.cu:3-35), ion::build_kernels
 * (common.h:318-327) and stress::build_kernels (stress.cu:106-149). */
static void build_tables(oracle_state* h)
{
    const oracle_config* c = &h->c;
    const int size = h->size;
    for (int x = 0; x < c->m1; ++x) {
        const double kx = wave_number(x, c->m1, c->L1);
        for (int y = 0; y < c->m2; ++y) {
            const double ky = wave_number(y, c->m2, c->L2);
            for (int z = 0; z < c->m3; ++z) {
                const double kz = wave_number(z, c->m3, c->L3);
                const int i = (x * c->m2 + y) * c->m3 + z;
                const double ksq = kx * kx + ky * ky + kz * kz;
                h->k2[i] = ksq;
                h->Gamma[i] = exp(-0.5 * c->a * c->a * ksq);
                for (int sp = 0; sp < h->n_species; ++sp) {
                    for (int s = 0; s < h->N[sp] - 1; ++s) {
                        const double b = h->seg_bond[h->seg_off[sp] + s];
                        h->PHI[(size_t)(h->bond_off[sp] + s) * size + i] = exp(-b * b * ksq / 6.0);
                    }
                }
                const double vals[6] = {kx * kx, ky * ky, kz * kz, kx * ky, kx * kz, ky * kz};
                for (int cc = 0; cc < 6; ++cc) {
                    h->kab[(size_t)cc * size + i] = vals[cc];
                    h->minus_kab[(size_t)cc * size + i] = -vals[cc];
                }
            }
        }
    }
    for (int j = 0; j < c->n_ions; ++j)
        for (int i = 0; i < size; ++i) h->ion_kernels[(size_t)j * size + i] = exp(-0.5 * h->ions[j].smear * h->ions[j].smear * h->k2[i]);
    /* stress mode term */
    double sum[6] = {0, 0, 0, 0, 0, 0};
    long long modes = 0;
    for (int i = 0; i < size; ++i) {
        if (h->k2[i] > 0.0) {
            ++modes;
            for (int cc = 0; cc < 6; ++cc) sum[cc] += h->kab[(size_t)cc * size + i] / h->k2[i];
        }
    }
    for (int cc = 0; cc < 6; ++cc) {
        const double delta = cc < 3 ? 1.0 : 0.0;
        h->mode_term[cc] = h->elec ? (((1.0 / 3.0) * (double)modes * delta - sum[cc]) / h->volume) : 0.0;
    }
}

oracle_state* oracle_create(const oracle_config* cfg)
{
    oracle_state* h = (oracle_state*)calloc(1, sizeof(oracle_state));
    h->c = *cfg;
    const oracle_config* c = &h->c;
    h->size = c->m1 * c->m2 * c->m3;
    h->volume = c->L1 * c->L2 * c->L3;
    h->elec = c->lB > 0.0;
    const size_t V = (size_t)h->size;
    plan3_init(&h->plan, c->m1, c->m2, c->m3);

    h->n_species = c->n_species;
    h->num_chains = calloc_d(c->n_species);
    h->N = (int*)calloc((size_t)c->n_species + 1, sizeof(int));
    h->seg_off = (int*)calloc((size_t)c->n_species + 1, sizeof(int));
    h->bond_off = (int*)calloc((size_t)c->n_species + 1, sizeof(int));
    int total_segments = 0;
    h->Nmax = 0;
    h->total_bonds = 0;
    for (int sp = 0; sp < c->n_species; ++sp) {
        h->num_chains[sp] = c->num_chains[sp];
        h->N[sp] = c->N[sp];
        h->seg_off[sp] = total_segments;
        h->bond_off[sp] = h->total_bonds;
        total_segments += c->N[sp];
        h->total_bonds += c->N[sp] > 1 ? c->N[sp] - 1 : 0;
        if (c->N[sp] > h->Nmax) h->Nmax = c->N[sp];
    }
    h->seg_type = (int*)calloc((size_t)total_segments + 1, sizeof(int));
    h->seg_charge = calloc_d(total_segments);
    h->seg_bond = calloc_d(total_segments);
    for (int s = 0; s < total_segments; ++s) {
        h->seg_type[s] = c->seg_type[s];
        h->seg_charge[s] = c->seg_charge[s];
        h->seg_bond[s] = c->seg_bond[s];
    }
    h->ions = (ion_sp*)calloc((size_t)c->n_ions + 1, sizeof(ion_sp));
    for (int j = 0; j < c->n_ions; ++j) {
        h->ions[j].count = c->ion_count[j];
        h->ions[j].valence = c->ion_valence[j];
        h->ions[j].smear = c->ion_smear[j];
    }
    const int nm = c->n_modes;
    h->mode_coeff = calloc_d(nm);
    h->mode_gamma = calloc_c(nm);
    h->mode_O = calloc_d((size_t)nm * c->M);
    h->mode_lambda = calloc_d(nm);
    for (int a = 0; a < nm; ++a) {
        h->mode_coeff[a] = c->mode_coeff[a];
        h->mode_gamma[a] = mk(c->mode_gamma[2 * a], c->mode_gamma[2 * a + 1]);
        h->mode_lambda[a] = c->mode_lambda[a];
        for (int al = 0; al < c->M; ++al) h->mode_O[a * c->M + al] = c->mode_O[a * c->M + al];
    }
    h->c.mode_coeff = h->mode_coeff;
    h->c.mode_O = h->mode_O;
    h->c.mode_lambda = h->mode_lambda;
    h->c.mode_gamma = NULL;
    h->c.num_chains = h->num_chains;
    h->c.N = h->N;
    h->c.seg_type = h->seg_type;
    h->c.seg_charge = h->seg_charge;
    h->c.seg_bond = h->seg_bond;
    h->c.ion_valence = h->c.ion_count = h->c.ion_smear = NULL;

    const size_t nmv = V * (size_t)(nm > 0 ? nm : 1);
    const size_t Mv = V * (size_t)(c->M > 0 ? c->M : 1);
    const size_t chain = V * (size_t)(h->Nmax > 0 ? h->Nmax : 1);
    h->omega = calloc_c(nmv); h->omega_bar = calloc_c(nmv); h->omega_s = calloc_c(nmv);
    h->drift = calloc_c(nmv); h->drift_bar = calloc_c(nmv); h->eta_omega = calloc_d(nmv);
    h->psi = calloc_c(V); h->psi_bar = calloc_c(V); h->psi_s = calloc_c(V);
    h->dpsi = calloc_c(V); h->dpsi_bar = calloc_c(V); h->etaPsi = calloc_d(V);
    h->W_type_s = calloc_c(Mv); h->rho_type = calloc_c(Mv);
    h->rho_c = calloc_c(V); h->rho_c_poly = calloc_c(V); h->rho_c_ion = calloc_c(V);
    h->rho_c_old = calloc_c(V); h->rho_p = calloc_c(V);
    h->W = calloc_c(chain); h->exp_mW = calloc_c(chain); h->exp_W = calloc_c(chain);
    h->qF = calloc_c(chain); h->qB = calloc_c(chain);
    h->ion_psi = calloc_c(V); h->ion_boltzmann = calloc_c(V); h->ion_charge = calloc_c(V);
    h->ion_rho = calloc_c(V * (size_t)(c->n_ions > 0 ? c->n_ions : 1));
    h->obs_a = calloc_c(V); h->obs_b = calloc_c(V); h->obs_c = calloc_c(V);
    h->s_a = calloc_c(V); h->s_b = calloc_c(V); h->s_c = calloc_c(V); h->s_dfield = calloc_c(V); h->s_dpsi = calloc_c(V);
    h->iso_a = calloc_c(V); h->iso_b = calloc_c(V); h->iso_c = calloc_c(V);
    h->Gamma = calloc_d(V); h->k2 = calloc_d(V);
    h->PHI = calloc_d(V * (size_t)(h->total_bonds > 0 ? h->total_bonds : 1));
    for (size_t i = 0; i < V * (size_t)(h->total_bonds > 0 ? h->total_bonds : 1); ++i) h->PHI[i] = 1.0;
    h->ion_kernels = calloc_d(V * (size_t)(c->n_ions > 0 ? c->n_ions : 1));
    h->kab = calloc_d(6 * V); h->minus_kab = calloc_d(6 * V);
    build_tables(h);
    return h;
}

void oracle_destroy(oracle_state* h)
{
    if (!h) return;
    plan3_free(&h->plan);
    void* bufs[] = {h->num_chains, h->N, h->seg_off, h->bond_off, h->seg_type, h->seg_charge, h->seg_bond, h->ions,
                    h->mode_coeff, h->mode_gamma, h->mode_O, h->mode_lambda,
                    h->omega, h->omega_bar, h->omega_s, h->drift, h->drift_bar, h->eta_omega,
                    h->psi, h->psi_bar, h->psi_s, h->dpsi, h->dpsi_bar, h->etaPsi,
                    h->W_type_s, h->rho_type, h->rho_c, h->rho_c_poly, h->rho_c_ion, h->rho_c_old, h->rho_p,
                    h->W, h->exp_mW, h->exp_W, h->qF, h->qB, h->ion_psi, h->ion_boltzmann, h->ion_charge, h->ion_rho,
                    h->obs_a, h->obs_b, h->obs_c, h->s_a, h->s_b, h->s_c, h->s_dfield, h->s_dpsi,
                    h->iso_a, h->iso_b, h->iso_c, h->Gamma, h->k2, h->PHI, h->ion_kernels, h->kab, h->minus_kab};
    for (size_t i = 0; i < sizeof(bufs) / sizeof(bufs[0]); ++i) free(bufs[i]);
    free(h);
}

/* ---- elementwise primitives: common.h:474-598, 813-929 ---- */
static void fill_c(cd* d, cd v, int n) { for (int i = 0; i < n; ++i) d[i] = v; }
static void copy_c(cd* d, const cd* s, int n) { memcpy(d, s, sizeof(cd) * (size_t)n); }
static void add_c(cd* d, const cd* s, int n) { for (int i = 0; i < n; ++i) d[i] = cadd(d[i], s[i]); }
static void add_scaled_c(cd* d, const cd* s, double sc, int n) { for (int i = 0; i < n; ++i) d[i] = cadd(d[i], cscale(s[i], sc)); }
static void add_scaled_cc(cd* d, const cd* s, cd sc, int n) { for (int i = 0; i < n; ++i) d[i] = cadd(d[i], cmul(s[i], sc)); }
static void add_scaled_real(cd* d, const double* s, double sc, int n) { for (int i = 0; i < n; ++i) d[i].x += sc * s[i]; }
static void add_const_c(cd* d, cd v, int n) { for (int i = 0; i < n; ++i) d[i] = cadd(d[i], v); }
static void scale_real(cd* d, const double* s, int n) { for (int i = 0; i < n; ++i) d[i] = cscale(d[i], s[i]); }
static void scale_real_const(cd* d, double s, int n) { for (int i = 0; i < n; ++i) d[i] = cscale(d[i], s); }
static void mul_c(cd* d, const cd* s, int n) { for (int i = 0; i < n; ++i) d[i] = cmul(d[i], s[i]); }
static void add_i_times(cd* d, const cd* s, int n) { for (int i = 0; i < n; ++i) { d[i].x -= s[i].y; d[i].y += s[i].x; } }

/* Pairwise summation (the reference uses a fixed tree; both are accurate to
 * a few ulp of the sum's magnitude). */
static cd sum_c_rec(const cd* d, long n)
{
    if (n <= 64) {
        cd a = mk(0, 0);
        for (long i = 0; i < n; ++i) a = cadd(a, d[i]);
        return a;
    }
    const long h = n / 2;
    return cadd(sum_c_rec(d, h), sum_c_rec(d + h, n - h));
}
static double sum_r_rec(const double* d, long n)
{
    if (n <= 64) {
        double a = 0;
        for (long i = 0; i < n; ++i) a += d[i];
        return a;
    }
    const long h = n / 2;
    return sum_r_rec(d, h) + sum_r_rec(d + h, n - h);
}
static cd sum_c(const cd* d, int n) { return n > 0 ? sum_c_rec(d, n) : mk(0, 0); }
static cd mean_c(const cd* d, int n) { return cscale(sum_c(d, n), 1.0 / (double)n); }
static void remove_complex_mean(cd* d, int n) { if (n > 0) add_const_c(d, cscale(mean_c(d, n), -1.0), n); }
static void remove_real_mean(double* d, int n)
{
    if (n <= 0) return;
    const double m = sum_r_rec(d, n) / (double)n;
    for (int i = 0; i < n; ++i) d[i] += -m;
}
static double max_complex_magnitude(const cd* d, double scale, int n) /* common.h:1014-1051 */
{
    double m = 0.0;
    for (int i = 0; i < n; ++i) {
        double v = d[i].x * d[i].x + d[i].y * d[i].y;
        if (!isfinite(v)) v = INFINITY;
        if (v > m) m = v;
    }
    return fabs(scale) * sqrt(m > 0.0 ? m : 0.0);
}

/* fft_apply_real_kernel (common.h:1079-1085): FFT, x(1/size), x kernel, IFFT. */
static void fft_apply(oracle_state* h, const cd* src, cd* dst, const double* kernel)
{
    const int n = h->size;
    if (dst != src) copy_c(dst, src, n);
    fft3d(&h->plan, dst, -1);
    scale_real_const(dst, 1.0 / (double)n, n);
    scale_real(dst, kernel, n);
    fft3d(&h->plan, dst, +1);
}

/* ---- polymers: polymer.cu:341-478 ---- */
static void build_smoothed_sources(oracle_state* h, const cd* omega, const cd* psi)
{
    const int n = h->size;
    const oracle_config* c = &h->c;
    for (int a = 0; a < c->n_modes; ++a) fft_apply(h, omega + (size_t)a * n, h->omega_s + (size_t)a * n, h->Gamma);
    for (int al = 0; al < c->M; ++al) {
        cd* Wa = h->W_type_s + (size_t)al * n;
        fill_c(Wa, mk(0, 0), n);
        for (int a = 0; a < c->n_modes; ++a) {
            const cd coeff = cscale(h->mode_gamma[a], h->mode_O[a * c->M + al]);
            add_scaled_cc(Wa, h->omega_s + (size_t)a * n, coeff, n);
        }
    }
    if (h->elec) fft_apply(h, psi, h->psi_s, h->Gamma);
    else fill_c(h->psi_s, mk(0, 0), n);
}

static cd solve_chain_species_prepared(oracle_state* h, int sp)
{
    const int n = h->size;
    const int N = h->N[sp];
    const int off = h->seg_off[sp];
    /* build_segment_fields (polymer.cu:365-375) */
    for (int s = 0; s < N; ++s) {
        cd* W = h->W + (size_t)s * n;
        copy_c(W, h->W_type_s + (size_t)h->seg_type[off + s] * n, n);
        const double z = h->elec ? h->seg_charge[off + s] : 0.0;
        if (z != 0.0) add_scaled_cc(W, h->psi_s, mk(0.0, z), n);
    }
    /* build_exponentials (polymer.cu:377-384) */
    for (int s = 0; s < N; ++s) {
        const cd* W = h->W + (size_t)s * n;
        cd* em = h->exp_mW + (size_t)s * n;
        cd* ep = h->exp_W + (size_t)s * n;
        for (int i = 0; i < n; ++i) {
            em[i] = cexp_(mk(-W[i].x, -W[i].y));
            ep[i] = cexp_(W[i]);
        }
    }
    /* propagate_chain (polymer.cu:402-416) */
    copy_c(h->qF, h->exp_mW, n);
    copy_c(h->qB + (size_t)(N - 1) * n, h->exp_mW + (size_t)(N - 1) * n, n);
    for (int s = 0; s < N - 1; ++s) {
        const double* phi = h->PHI + (size_t)(h->bond_off[sp] + s) * n;
        cd* dst = h->qF + (size_t)(s + 1) * n;
        fft_apply(h, h->qF + (size_t)s * n, dst, phi);
        mul_c(dst, h->exp_mW + (size_t)(s + 1) * n, n);
    }
    for (int s = N - 1; s > 0; --s) {
        const double* phi = h->PHI + (size_t)(h->bond_off[sp] + s - 1) * n;
        cd* dst = h->qB + (size_t)(s - 1) * n;
        fft_apply(h, h->qB + (size_t)s * n, dst, phi);
        mul_c(dst, h->exp_mW + (size_t)(s - 1) * n, n);
    }
    return mean_c(h->qF + (size_t)(N - 1) * n, n);
}

/* accumulatePolymerDensityByChainDensityKernel (common.h:560-580) */
static void accumulate_density(oracle_state* h, cd* rho, int s, double chain_density, cd Q, double weight)
{
    if (weight == 0.0) return;
    const int n = h->size;
    const cd factor = cscale(cinv(Q), chain_density * weight);
    const cd* qF = h->qF + (size_t)s * n;
    const cd* qB = h->qB + (size_t)s * n;
    const cd* eW = h->exp_W + (size_t)s * n;
    for (int i = 0; i < n; ++i) rho[i] = cadd(rho[i], cmul(cmul(cmul(qF[i], qB[i]), eW[i]), factor));
}

static void solve_and_compute_densities(oracle_state* h, const cd* omega, const cd* psi, cd* Q)
{
    const int n = h->size;
    const oracle_config* c = &h->c;
    for (int al = 0; al < c->M; ++al) fill_c(h->rho_type + (size_t)al * n, mk(0, 0), n);
    fill_c(h->rho_c_poly, mk(0, 0), n);
    fill_c(h->rho_c_ion, mk(0, 0), n);
    fill_c(h->rho_c, mk(0, 0), n);
    build_smoothed_sources(h, omega, psi);
    for (int sp = 0; sp < h->n_species; ++sp) {
        const cd Qs = solve_chain_species_prepared(h, sp);
        Q[sp] = Qs;
        const double chain_density = h->num_chains[sp] / h->volume;
        for (int s = 0; s < h->N[sp]; ++s) {
            const int off = h->seg_off[sp] + s;
            accumulate_density(h, h->rho_type + (size_t)h->seg_type[off] * n, s, chain_density, Qs, 1.0);
            if (h->elec) accumulate_density(h, h->rho_c_poly, s, chain_density, Qs, h->seg_charge[off]);
        }
    }
    fill_c(h->rho_p, mk(0, 0), n);
    for (int al = 0; al < c->M; ++al) {
        cd* ra = h->rho_type + (size_t)al * n;
        fft_apply(h, ra, ra, h->Gamma);
        add_c(h->rho_p, ra, n);
    }
    if (h->elec) {
        fft_apply(h, h->rho_c_poly, h->rho_c_poly, h->Gamma);
        add_c(h->rho_c, h->rho_c_poly, n);
    }
}

/* ---- ions: ion.cu:54-72, common.h:1104-1130 ---- */
static cd ion_partition_function(oracle_state* h, cd* smoothed, cd* boltz, const cd* psi, const double* kernel, double z)
{
    const int n = h->size;
    fft_apply(h, psi, smoothed, kernel);
    for (int i = 0; i < n; ++i) boltz[i] = cexp_(mk(z * smoothed[i].y, -z * smoothed[i].x));
    return mean_c(boltz, n);
}

static void ion_compute_densities(oracle_state* h, const cd* psi)
{
    const int n = h->size;
    for (int j = 0; j < h->c.n_ions; ++j) {
        const double* kernel = h->ion_kernels + (size_t)j * n;
        cd* rho = h->ion_rho + (size_t)j * n;
        const double nd = h->ions[j].count / h->volume;
        if (!h->elec) {
            fill_c(rho, mk(nd, 0.0), n);
            continue;
        }
        const cd Q = ion_partition_function(h, h->ion_psi, h->ion_boltzmann, psi, kernel, h->ions[j].valence);
        const cd factor = cscale(cinv(Q), nd);
        for (int i = 0; i < n; ++i) rho[i] = cmul(h->ion_boltzmann[i], factor);
        fft_apply(h, rho, h->ion_charge, kernel);
        scale_real_const(h->ion_charge, h->ions[j].valence, n);
        add_c(h->rho_c_ion, h->ion_charge, n);
        add_c(h->rho_c, h->ion_charge, n);
    }
}

static void compute_densities(oracle_state* h, const cd* omega, const cd* psi, cd* Q)
{
    solve_and_compute_densities(h, omega, psi, Q);
    ion_compute_densities(h, psi);
}

/* ---- CL update: complexLangevin.cu:272-368 ---- */
static void compute_drifts(oracle_state* h, const cd* omega, cd* drift)
{
    const int n = h->size;
    const oracle_config* c = &h->c;
    for (int a = 0; a < c->n_modes; ++a) {
        cd* u = drift + (size_t)a * n;
        fill_c(u, mk(0, 0), n);
        add_scaled_c(u, omega + (size_t)a * n, h->mode_coeff[a], n);
        for (int al = 0; al < c->M; ++al) {
            const cd coeff = cscale(h->mode_gamma[a], h->mode_O[a * c->M + al]);
            add_scaled_cc(u, h->rho_type + (size_t)al * n, coeff, n);
        }
    }
}

static void remove_psi_zero_mode(oracle_state* h, cd* f)
{
    if (h->elec) remove_complex_mean(f, h->size);
    else fill_c(f, mk(0, 0), h->size);
}

static void compute_psi_drift(oracle_state* h, const cd* psi, const cd* rho_source, cd* drift)
{
    const int n = h->size;
    if (!h->elec) {
        fill_c(drift, mk(0, 0), n);
        return;
    }
    fft_apply(h, psi, drift, h->k2);
    scale_real_const(drift, 1.0 / (4.0 * PI * h->c.lB), n);
    add_i_times(drift, rho_source, n);
    remove_psi_zero_mode(h, drift);
}

static void predictor_step(oracle_state* h)
{
    const int n = h->size;
    const oracle_config* c = &h->c;
    compute_psi_drift(h, h->psi, h->rho_c_old, h->dpsi);
    for (int a = 0; a < c->n_modes; ++a) {
        cd* pred = h->omega_bar + (size_t)a * n;
        copy_c(pred, h->omega + (size_t)a * n, n);
        add_scaled_c(pred, h->drift + (size_t)a * n, -c->dt * h->mode_lambda[a], n);
        add_scaled_real(pred, h->eta_omega + (size_t)a * n, 1.0, n);
    }
    copy_c(h->psi_bar, h->psi, n);
    if (h->elec) add_scaled_c(h->psi_bar, h->dpsi, -c->dt * c->lambda_psi, n);
    else fill_c(h->psi_bar, mk(0, 0), n);
    if (h->elec) add_scaled_real(h->psi_bar, h->etaPsi, 1.0, n);
    remove_psi_zero_mode(h, h->psi_bar);
}

static void corrector_step(oracle_state* h)
{
    const int n = h->size;
    const oracle_config* c = &h->c;
    for (int a = 0; a < c->n_modes; ++a) {
        cd* w = h->omega + (size_t)a * n;
        const double lam = h->mode_lambda[a];
        add_scaled_c(w, h->drift + (size_t)a * n, -0.5 * c->dt * lam, n);
        add_scaled_c(w, h->drift_bar + (size_t)a * n, -0.5 * c->dt * lam, n);
        add_scaled_real(w, h->eta_omega + (size_t)a * n, 1.0, n);
    }
    if (h->elec) {
        add_scaled_c(h->psi, h->dpsi, -0.5 * c->dt * c->lambda_psi, n);
        add_scaled_c(h->psi, h->dpsi_bar, -0.5 * c->dt * c->lambda_psi, n);
        add_scaled_real(h->psi, h->etaPsi, 1.0, n);
    }
    remove_psi_zero_mode(h, h->psi);
}

/* ---- observables: observable.cu:53-317, stress.cu:161-321 ---- */
static cd mean_product(oracle_state* h, cd* scratch, const cd* a, const cd* b)
{
    copy_c(scratch, a, h->size);
    mul_c(scratch, b, h->size);
    return cscale(sum_c(scratch, h->size), 1.0 / (double)h->size);
}

static double total_ion_count(oracle_state* h)
{
    double t = 0.0;
    for (int j = 0; j < h->c.n_ions; ++j) t += h->ions[j].count;
    return t;
}

static double total_chains(oracle_state* h)
{
    double t = 0.0;
    for (int sp = 0; sp < h->n_species; ++sp) t += h->num_chains[sp];
    return t;
}

static cd stress_ideal(oracle_state* h, int cc)
{
    const double delta = cc < 3 ? 1.0 : 0.0;
    const double ideal = (total_chains(h) + total_ion_count(h)) / h->volume;
    return mk((ideal + h->c.self_pressure) * delta + h->mode_term[cc], 0.0);
}

static cd stress_electrostatic(oracle_state* h, const cd* psi, int cc)
{
    if (!h->elec) return mk(0, 0);
    const double delta = cc < 3 ? 1.0 : 0.0;
    fft_apply(h, psi, h->s_a, h->k2);
    const cd g2 = mean_product(h, h->s_b, psi, h->s_a);
    fft_apply(h, psi, h->s_a, h->kab + (size_t)cc * h->size);
    const cd gab = mean_product(h, h->s_b, psi, h->s_a);
    const cd bracket = csub(gab, cscale(g2, delta / 3.0));
    return cscale(bracket, 1.0 / (4.0 * PI * h->c.lB));
}

static cd stress_connectivity(oracle_state* h, int sp, cd Q, int cc)
{
    const int n = h->size;
    cd total = mk(0, 0);
    for (int s = 0; s < h->N[sp] - 1; ++s) {
        copy_c(h->s_a, h->exp_W + (size_t)s * n, n);
        mul_c(h->s_a, h->qB + (size_t)s * n, n);
        fft_apply(h, h->s_a, h->s_b, h->minus_kab + (size_t)cc * n);
        copy_c(h->s_c, h->qF + (size_t)s * n, n);
        mul_c(h->s_c, h->s_b, n);
        const cd avg = cscale(sum_c(h->s_c, n), 1.0 / (double)n);
        const double b = h->seg_bond[h->seg_off[sp] + s];
        total = cadd(total, cscale(avg, b * b / 3.0));
    }
    const cd pref = cscale(cinv(Q), -h->num_chains[sp] / h->volume);
    return cmul(pref, total);
}

static cd stress_polymer_field(oracle_state* h, int sp, cd Q, int cc)
{
    const int n = h->size;
    const double a2 = h->c.a * h->c.a;
    const int diag = cc < 3;
    cd total = mk(0, 0);
    if (h->elec) fft_apply(h, h->psi_s, h->s_dpsi, h->minus_kab + (size_t)cc * n);
    else fill_c(h->s_dpsi, mk(0, 0), n);
    for (int s = 0; s < h->N[sp]; ++s) {
        const int off = h->seg_off[sp] + s;
        const cd* Wa = h->W_type_s + (size_t)h->seg_type[off] * n;
        fft_apply(h, Wa, h->s_dfield, h->minus_kab + (size_t)cc * n);
        fill_c(h->s_b, mk(0, 0), n);
        add_scaled_c(h->s_b, h->s_dfield, a2, n);
        if (diag) add_scaled_c(h->s_b, Wa, 0.5, n);
        if (h->elec) {
            add_scaled_cc(h->s_b, h->s_dpsi, mk(0.0, h->seg_charge[off] * a2), n);
            if (diag) add_scaled_cc(h->s_b, h->psi_s, mk(0.0, h->seg_charge[off] / 6.0), n);
        }
        copy_c(h->s_a, h->qF + (size_t)s * n, n);
        mul_c(h->s_a, h->qB + (size_t)s * n, n);
        mul_c(h->s_a, h->exp_W + (size_t)s * n, n);
        copy_c(h->s_c, h->s_a, n);
        mul_c(h->s_c, h->s_b, n);
        total = cadd(total, cscale(sum_c(h->s_c, n), 1.0 / (double)n));
    }
    const cd pref = cscale(cinv(Q), h->num_chains[sp] / h->volume);
    return cmul(pref, total);
}

static cd stress_ion_field(oracle_state* h, const cd* psi, int cc)
{
    if (!h->elec) return mk(0, 0);
    const int n = h->size;
    const int diag = cc < 3;
    cd total = mk(0, 0);
    for (int j = 0; j < h->c.n_ions; ++j) {
        const double* kernel = h->ion_kernels + (size_t)j * n;
        const cd Qj = ion_partition_function(h, h->ion_psi, h->ion_boltzmann, psi, kernel, h->ions[j].valence);
        fft_apply(h, h->ion_psi, h->s_a, h->minus_kab + (size_t)cc * n);
        const double a2 = h->ions[j].smear * h->ions[j].smear;
        scale_real_const(h->s_a, a2, n);
        if (diag) add_scaled_c(h->s_a, h->ion_psi, 1.0 / 6.0, n);
        copy_c(h->s_b, h->ion_boltzmann, n);
        mul_c(h->s_b, h->s_a, n);
        const cd avg = cscale(sum_c(h->s_b, n), 1.0 / (double)n);
        cd pref = cscale(cinv(Qj), h->ions[j].count * h->ions[j].valence / h->volume);
        pref = cmul(mk(0.0, 1.0), pref);
        total = cadd(total, cmul(pref, avg));
    }
    return total;
}

static void iso_trace_block(oracle_state* h, cd* out, const cd* field, double s2, double local)
{
    fft_apply(h, field, out, h->k2);
    scale_real_const(out, -s2 / 3.0, h->size);
    add_scaled_c(out, field, local, h->size);
}

static cd iso_polymer_field(oracle_state* h, int sp, cd Q)
{
    const int n = h->size;
    const double a2 = h->c.a * h->c.a;
    cd total = mk(0, 0);
    for (int s = 0; s < h->N[sp]; ++s) {
        const int off = h->seg_off[sp] + s;
        iso_trace_block(h, h->iso_b, h->W_type_s + (size_t)h->seg_type[off] * n, a2, 0.5);
        if (h->elec) {
            iso_trace_block(h, h->iso_c, h->psi_s, a2, 1.0 / 6.0);
            add_scaled_cc(h->iso_b, h->iso_c, mk(0.0, h->seg_charge[off]), n);
        }
        copy_c(h->iso_a, h->qF + (size_t)s * n, n);
        mul_c(h->iso_a, h->qB + (size_t)s * n, n);
        mul_c(h->iso_a, h->exp_W + (size_t)s * n, n);
        mul_c(h->iso_a, h->iso_b, n);
        total = cadd(total, cscale(sum_c(h->iso_a, n), 1.0 / (double)n));
    }
    return cmul(cscale(cinv(Q), h->num_chains[sp] / h->volume), total);
}

static cd iso_connectivity(oracle_state* h, int sp, cd Q)
{
    const int n = h->size;
    cd total = mk(0, 0);
    for (int s = 0; s < h->N[sp] - 1; ++s) {
        copy_c(h->iso_a, h->exp_W + (size_t)s * n, n);
        mul_c(h->iso_a, h->qB + (size_t)s * n, n);
        fft_apply(h, h->iso_a, h->iso_b, h->k2);
        copy_c(h->iso_c, h->qF + (size_t)s * n, n);
        mul_c(h->iso_c, h->iso_b, n);
        const cd avg = cscale(sum_c(h->iso_c, n), 1.0 / (double)n);
        const double b = h->seg_bond[h->seg_off[sp] + s];
        total = cadd(total, cscale(avg, b * b / 9.0));
    }
    return cmul(cscale(cinv(Q), h->num_chains[sp] / h->volume), total);
}

static cd iso_ion_field(oracle_state* h, const cd* psi)
{
    if (!h->elec) return mk(0, 0);
    const int n = h->size;
    cd total = mk(0, 0);
    for (int j = 0; j < h->c.n_ions; ++j) {
        const double* kernel = h->ion_kernels + (size_t)j * n;
        const cd Qj = ion_partition_function(h, h->ion_psi, h->ion_boltzmann, psi, kernel, h->ions[j].valence);
        const double a2 = h->ions[j].smear * h->ions[j].smear;
        iso_trace_block(h, h->iso_b, h->ion_psi, a2, 1.0 / 6.0);
        copy_c(h->iso_c, h->ion_boltzmann, n);
        mul_c(h->iso_c, h->iso_b, n);
        const cd avg = cscale(sum_c(h->iso_c, n), 1.0 / (double)n);
        cd pref = cscale(cinv(Qj), h->ions[j].count * h->ions[j].valence / h->volume);
        pref = cmul(mk(0.0, 1.0), pref);
        total = cadd(total, cmul(pref, avg));
    }
    return total;
}

int oracle_measure(oracle_state* h, int which, const double* Qd, double* out)
{
    const oracle_config* c = &h->c;
    const int n = h->size;
    const cd* omega = which ? h->omega_bar : h->omega;
    const cd* psi = which ? h->psi_bar : h->psi;
    const cd* Q = (const cd*)Qd;
    const int S = h->n_species, J = c->n_ions;
    cd* rec = (cd*)out;
    int k = 0;
    /* chemical operators: observable.cu:69-87, 111-118 */
    cd* chem = rec;
    for (int sp = 0; sp < S; ++sp) rec[k++] = cneglog(Q[sp]);
    for (int j = 0; j < J; ++j) {
        if (!h->elec) { rec[k++] = mk(0, 0); continue; }
        rec[k++] = cneglog(ion_partition_function(h, h->obs_a, h->obs_b, psi, h->ion_kernels + (size_t)j * n, h->ions[j].valence));
    }
    /* self: observable.cu:89-100 */
    for (int sp = 0; sp < S; ++sp) {
        double zz = 0.0;
        for (int s = 0; s < h->N[sp]; ++s) zz += h->seg_charge[h->seg_off[sp] + s] * h->seg_charge[h->seg_off[sp] + s];
        rec[k++] = mk(-c->lB * zz / (2.0 * sqrt(PI) * c->a), 0.0);
    }
    for (int j = 0; j < J; ++j)
        rec[k++] = mk(-c->lB * h->ions[j].valence * h->ions[j].valence / (2.0 * sqrt(PI) * h->ions[j].smear), 0.0);
    /* ideal: observable.cu:120-127 */
    for (int sp = 0; sp < S; ++sp) rec[k++] = mk(log(h->num_chains[sp] / h->volume), 0.0);
    for (int j = 0; j < J; ++j) rec[k++] = mk(log(h->ions[j].count / h->volume), 0.0);
    /* mean-field Hamiltonian density: observable.cu:141-182 */
    cd H = mk(0, 0);
    for (int a = 0; a < c->n_modes; ++a) {
        copy_c(h->obs_a, omega + (size_t)a * n, n);
        mul_c(h->obs_a, omega + (size_t)a * n, n);
        H = cadd(H, cscale(sum_c(h->obs_a, n), 0.5 * h->mode_coeff[a] / (double)n));
    }
    if (h->elec) {
        fft_apply(h, psi, h->obs_a, h->k2);
        copy_c(h->obs_b, psi, n);
        mul_c(h->obs_b, h->obs_a, n);
        H = cadd(H, cscale(sum_c(h->obs_b, n), 1.0 / (8.0 * PI * c->lB * (double)n)));
    }
    for (int sp = 0; sp < S; ++sp) H = cadd(H, cscale(chem[sp], h->num_chains[sp] / h->volume));
    for (int j = 0; j < J; ++j) H = cadd(H, cscale(chem[S + j], h->ions[j].count / h->volume));
    rec[k++] = H;
    /* stress tensor: stress.cu:161-196 */
    int active[6], na = 0;
    for (int cc = 0; cc < 6; ++cc) if (c->stress_mask & (1 << cc)) active[na++] = cc;
    if (na > 0) {
        cd* vals = rec + k;
        for (int i = 0; i < na; ++i) {
            vals[i] = stress_ideal(h, active[i]);
            if (h->elec) vals[i] = cadd(vals[i], stress_electrostatic(h, psi, active[i]));
        }
        build_smoothed_sources(h, omega, psi);
        for (int sp = 0; sp < S; ++sp) {
            (void)solve_chain_species_prepared(h, sp);
            for (int i = 0; i < na; ++i) {
                vals[i] = cadd(vals[i], stress_connectivity(h, sp, Q[sp], active[i]));
                vals[i] = cadd(vals[i], stress_polymer_field(h, sp, Q[sp], active[i]));
            }
        }
        if (h->elec)
            for (int i = 0; i < na; ++i) vals[i] = cadd(vals[i], stress_ion_field(h, psi, active[i]));
        k += na;
    }
    /* isotropic pressure: observable.cu:297-317 */
    if (c->isotropic_pressure) {
        const double ideal = (total_chains(h) + total_ion_count(h)) / h->volume;
        cd v = mk(ideal + c->self_pressure, 0.0);
        build_smoothed_sources(h, omega, psi);
        for (int sp = 0; sp < S; ++sp) {
            (void)solve_chain_species_prepared(h, sp);
            v = cadd(v, iso_polymer_field(h, sp, Q[sp]));
            v = cadd(v, iso_connectivity(h, sp, Q[sp]));
        }
        v = cadd(v, iso_ion_field(h, psi));
        rec[k++] = v;
    }
    return k;
}

void oracle_set_fields(oracle_state* h, const double* omega, const double* psi)
{
    const size_t n = (size_t)h->size;
    if (h->c.n_modes > 0) memcpy(h->omega, omega, sizeof(cd) * n * (size_t)h->c.n_modes);
    memcpy(h->psi, psi, sizeof(cd) * n);
    remove_psi_zero_mode(h, h->psi);
}

void oracle_compute_densities(oracle_state* h, int which, double* Q_out)
{
    compute_densities(h, which ? h->omega_bar : h->omega, which ? h->psi_bar : h->psi, (cd*)Q_out);
}

/* complexLangevin::run_step (complexLangevin.cu:669-698) with injected noise. */
int oracle_step(oracle_state* h, const double* eta, double* Q_bar_out, double* record_out, double* drift_max_out)
{
    const int n = h->size;
    const oracle_config* c = &h->c;
    cd* Q = (cd*)calloc((size_t)h->n_species + 1, sizeof(cd));
    compute_densities(h, h->omega, h->psi, Q);
    copy_c(h->rho_c_old, h->rho_c, n);
    const size_t nm = (size_t)c->n_modes;
    if (eta) {
        memcpy(h->eta_omega, eta, sizeof(double) * nm * (size_t)n);
        memcpy(h->etaPsi, eta + nm * (size_t)n, sizeof(double) * (size_t)n);
    } else {
        memset(h->eta_omega, 0, sizeof(double) * (nm ? nm : 1) * (size_t)n);
        memset(h->etaPsi, 0, sizeof(double) * (size_t)n);
    }
    if (h->elec) remove_real_mean(h->etaPsi, n);
    compute_drifts(h, h->omega, h->drift);
    predictor_step(h);
    compute_densities(h, h->omega_bar, h->psi_bar, Q);
    if (Q_bar_out) memcpy(Q_bar_out, Q, sizeof(cd) * (size_t)h->n_species);
    compute_psi_drift(h, h->psi_bar, h->rho_c, h->dpsi_bar);
    int k = 0;
    if (record_out) k = oracle_measure(h, 1, (const double*)Q, record_out);
    compute_drifts(h, h->omega_bar, h->drift_bar);
    if (drift_max_out) {
        for (int a = 0; a < c->n_modes; ++a) {
            copy_c(h->obs_a, h->drift + (size_t)a * n, n);
            add_c(h->obs_a, h->drift_bar + (size_t)a * n, n);
            drift_max_out[a] = max_complex_magnitude(h->obs_a, 0.5 * h->mode_lambda[a], n);
        }
        copy_c(h->obs_a, h->dpsi, n);
        add_c(h->obs_a, h->dpsi_bar, n);
        drift_max_out[c->n_modes] = max_complex_magnitude(h->obs_a, 0.5 * c->lambda_psi, n);
    }
    corrector_step(h);
    free(Q);
    return k;
}

long long oracle_get(oracle_state* h, const char* name, double* out)
{
    const size_t n = (size_t)h->size;
    const size_t nm = (size_t)h->c.n_modes, M = (size_t)h->c.M, J = (size_t)h->c.n_ions, Nm = (size_t)h->Nmax;
    struct { const char* name; const void* p; size_t doubles; } t[] = {
        {"omega", h->omega, 2 * nm * n}, {"psi", h->psi, 2 * n}, {"omega_bar", h->omega_bar, 2 * nm * n},
        {"psi_bar", h->psi_bar, 2 * n}, {"omega_s", h->omega_s, 2 * nm * n}, {"psi_s", h->psi_s, 2 * n},
        {"W_type_s", h->W_type_s, 2 * M * n}, {"rho_type", h->rho_type, 2 * M * n}, {"rho_p", h->rho_p, 2 * n},
        {"rho_c", h->rho_c, 2 * n}, {"rho_c_poly", h->rho_c_poly, 2 * n}, {"rho_c_ion", h->rho_c_ion, 2 * n},
        {"rho_c_old", h->rho_c_old, 2 * n}, {"ion_rho", h->ion_rho, 2 * J * n}, {"drift", h->drift, 2 * nm * n},
        {"drift_bar", h->drift_bar, 2 * nm * n}, {"dpsi", h->dpsi, 2 * n}, {"dpsi_bar", h->dpsi_bar, 2 * n},
        {"qF", h->qF, 2 * Nm * n}, {"qB", h->qB, 2 * Nm * n}, {"k2", h->k2, n}, {"Gamma", h->Gamma, n},
    };
    for (size_t i = 0; i < sizeof(t) / sizeof(t[0]); ++i) {
        if (strcmp(t[i].name, name) == 0) {
            if (out && t[i].doubles) memcpy(out, t[i].p, sizeof(double) * t[i].doubles);
            return (long long)t[i].doubles;
        }
    }
    return -1;
}
