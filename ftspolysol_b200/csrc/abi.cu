// C ABI of the engine (include/ftsp.h): configuration checks and the
// extern "C" entry points.  Every entry point catches C++ exceptions and
// CUDA errors and turns them into status codes; nothing calls exit().
#include "engine.cuh"

#include <mutex>

namespace ftsp {

HostCfg make_cfg(const ftsp_config* in)
{
    HostCfg c{};
    c.m1 = in->m1; c.m2 = in->m2; c.m3 = in->m3;
    if (c.m1 <= 0 || c.m2 <= 0 || c.m3 <= 0) throw std::runtime_error("invalid mesh");
    c.V = (size_t)c.m1 * c.m2 * c.m3;
    c.L[0] = in->L1; c.L[1] = in->L2; c.L[2] = in->L3;
    c.volume = in->L1 * in->L2 * in->L3;
    c.dV = in->dV; c.a = in->a; c.lB = in->lB; c.dt = in->dt; c.lpsi = in->lambda_psi;
    c.elec = in->lB > 0.0;
    c.M = in->M; c.nm = in->n_modes;
    if (c.M < 1 || c.M > MAXM) throw std::runtime_error("monomer type count out of range (1..8)");
    if (c.nm < 0 || c.nm > MAXMODE) throw std::runtime_error("active mode count out of range (0..8)");
    for (int a = 0; a < c.nm; ++a) {
        c.coeff.push_back(in->mode_coeff[a]);
        c.lambda.push_back(in->mode_lambda[a]);
        c.gamma.push_back(make_double2(in->mode_gamma[2 * a], in->mode_gamma[2 * a + 1]));
        for (int al = 0; al < c.M; ++al) c.O.push_back(in->mode_O[a * c.M + al]);
    }
    if (in->n_species < 1 || in->n_species > MAXSP) throw std::runtime_error("polymer species count out of range (1..16)");
    if (in->n_ions < 0 || in->n_ions > MAXION) throw std::runtime_error("ion species count out of range (0..16)");
    int off = 0;
    for (int s = 0; s < in->n_species; ++s) {
        Species sp{};
        sp.nc = in->num_chains[s];
        sp.N = in->N[s];
        if (sp.N < 1) throw std::runtime_error("species with N < 1");
        for (int t = 0; t < sp.N; ++t) {
            const int ty = in->seg_type[off + t];
            if (ty < 0 || ty >= c.M) throw std::runtime_error("segment monomer type out of range");
            sp.type.push_back(ty);
            sp.charge.push_back(in->seg_charge[off + t]);
            sp.bond.push_back(in->seg_bond[off + t]);
        }
        off += sp.N;
        for (int t = 0; t < sp.N; ++t) {
            const double z = c.elec ? sp.charge[t] : 0.0;
            int k = -1;
            for (size_t q = 0; q < c.cls.size(); ++q)
                if (c.cls[q].type == sp.type[t] && c.cls[q].z == z) k = (int)q;
            if (k < 0) {
                c.cls.push_back(Cls{sp.type[t], z});
                k = (int)c.cls.size() - 1;
            }
            sp.cls.push_back(k);
        }
        for (int t = 0; t + 1 < sp.N; ++t) {
            int k = -1;
            for (size_t q = 0; q < c.bond_lengths.size(); ++q)
                if (c.bond_lengths[q] == sp.bond[t]) k = (int)q;
            if (k < 0) {
                c.bond_lengths.push_back(sp.bond[t]);
                k = (int)c.bond_lengths.size() - 1;
            }
            sp.bcls.push_back(k);
        }
        c.sp.push_back(sp);
    }
    for (int j = 0; j < in->n_ions; ++j) c.ions.push_back(Ion{in->ion_valence[j], in->ion_count[j], in->ion_smear[j]});
    c.self_pressure = in->self_pressure;
    c.stress_mask = in->stress_mask & 63;
    c.iso = in->isotropic_pressure ? 1 : 0;
    c.noise = in->noise != 0;
    c.seed = in->seed;
    c.precision = in->precision;
    c.scheme = in->scheme;
    c.device = in->device;
    c.restart_interval = in->restart_interval > 0 ? in->restart_interval : 0;
    c.max_restarts = in->max_restarts > 0 ? in->max_restarts : 20;
    c.autotune = in->autotune != 0 ? 1 : 0;
    if (c.record_len() > 128) throw std::runtime_error("observable record too long");
    return c;
}

}  // namespace ftsp

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
struct ftsp_handle {
    std::unique_ptr<ftsp::EngineBase> eng;
    std::string err;
};

static thread_local std::string g_create_error;

namespace ftsp {
// Error text of handle-less calls, read back with ftsp_last_error(NULL).
void set_thread_error(const std::string& s) { g_create_error = s; }
}  // namespace ftsp

#define FTSP_GUARD(h, body)                                      \
    do {                                                         \
        if (!(h) || !(h)->eng) return FTSP_ERROR;                \
        try {                                                    \
            body;                                                \
        } catch (const std::exception& e_) {                     \
            (h)->err = e_.what();                                \
            return FTSP_ERROR;                                   \
        }                                                        \
    } while (0)

extern "C" {

int ftsp_create(const ftsp_config* cfg, ftsp_handle** out)
{
    if (!cfg || !out) return FTSP_ERROR;
    *out = nullptr;
    try {
        ftsp::HostCfg c = ftsp::make_cfg(cfg);
        auto* h = new ftsp_handle();
        if (c.precision == FTSP_FP32) h->eng.reset(ftsp::make_engine_f32(c));
        else h->eng.reset(ftsp::make_engine_f64(c));
        *out = h;
        return FTSP_OK;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        return FTSP_ERROR;
    }
}

int ftsp_destroy(ftsp_handle* h)
{
    if (!h) return FTSP_ERROR;
    try {
        h->eng.reset();
    } catch (...) {
    }
    delete h;
    return FTSP_OK;
}

const char* ftsp_last_error(const ftsp_handle* h)
{
    if (!h) return g_create_error.c_str();
    return h->err.c_str();
}

int ftsp_set_stream(ftsp_handle* h, void* s)
{
    FTSP_GUARD(h, {
        h->eng->stream = static_cast<cudaStream_t>(s);
        h->eng->drop_step_graph();
    });
    return FTSP_OK;
}

int ftsp_set_fields(ftsp_handle* h, const double* omega, const double* psi)
{
    if (!psi) return FTSP_ERROR;
    FTSP_GUARD(h, h->eng->set_fields(omega, psi));
    return FTSP_OK;
}

int ftsp_set_fields_async(ftsp_handle* h, const double* omega, const double* psi)
{
    if (!psi) return FTSP_ERROR;
    FTSP_GUARD(h, h->eng->set_fields_async(omega, psi));
    return FTSP_OK;
}

int ftsp_get_field(ftsp_handle* h, const char* name, double* out, long long* count)
{
    long long n = -1;
    FTSP_GUARD(h, n = h->eng->get_field(name ? name : "", out));
    if (count) *count = n;
    if (n < 0) {
        h->err = std::string("unknown field ") + (name ? name : "");
        return FTSP_ERROR;
    }
    return FTSP_OK;
}

int ftsp_compute_densities(ftsp_handle* h, int which, double* Q_out)
{
    FTSP_GUARD(h, h->eng->compute_densities(which ? 1 : 0, Q_out));
    for (size_t s = 0; s < h->eng->c.sp.size(); ++s)
        if (Q_out && !(std::isfinite(Q_out[2 * s]) && std::isfinite(Q_out[2 * s + 1]))) return FTSP_NONFINITE;
    return FTSP_OK;
}

int ftsp_record_length(const ftsp_handle* h)
{
    if (!h || !h->eng) return -1;
    return h->eng->c.record_len();
}

int ftsp_measure(ftsp_handle* h, int which, double* record)
{
    FTSP_GUARD(h, h->eng->measure(which ? 1 : 0, record));
    if (record)
        for (int i = 0; i < 2 * h->eng->c.record_len(); ++i)
            if (!std::isfinite(record[i])) return FTSP_NONFINITE;
    return FTSP_OK;
}

int ftsp_set_noise(ftsp_handle* h, const double* eta)
{
    if (!eta) return FTSP_ERROR;
    FTSP_GUARD(h, h->eng->set_noise(eta));
    return FTSP_OK;
}

int ftsp_set_seed(ftsp_handle* h, unsigned long long seed)
{
    FTSP_GUARD(h, {
        h->eng->c.seed = seed;
        h->eng->drop_step_graph();
    });
    return FTSP_OK;
}

int ftsp_step(ftsp_handle* h, double* Q_bar, double* record, double* drift_max)
{
    int st = FTSP_ERROR;
    FTSP_GUARD(h, st = h->eng->step(Q_bar, record, drift_max, true));
    return st;
}

int ftsp_step_async(ftsp_handle* h)
{
    FTSP_GUARD(h, h->eng->step(nullptr, nullptr, nullptr, false));
    return FTSP_OK;
}

int ftsp_read_status(ftsp_handle* h, double* record, double* drift_max)
{
    int st = FTSP_ERROR;
    FTSP_GUARD(h, st = h->eng->read_status(record, drift_max));
    return st;
}

int ftsp_tune_info_get(ftsp_handle* h, ftsp_tune_info* info)
{
    if (!info) return FTSP_ERROR;
    FTSP_GUARD(h, h->eng->tune_info(info));
    return FTSP_OK;
}

int ftsp_set_adaptive(ftsp_handle* h, double u_ref)
{
    FTSP_GUARD(h, h->eng->set_adaptive(u_ref));
    return FTSP_OK;
}

int ftsp_set_step_graph(ftsp_handle* h, int on)
{
    FTSP_GUARD(h, {
        h->eng->step_graph = on != 0;
        h->eng->drop_step_graph();
    });
    return FTSP_OK;
}

int ftsp_set_chain_symmetry(ftsp_handle* h, int on, int* n_species)
{
    FTSP_GUARD(h, {
        h->eng->set_chain_symmetry(on != 0);
        if (n_species) *n_species = h->eng->chain_symmetric_species();
    });
    return FTSP_OK;
}

int ftsp_step_info(ftsp_handle* h, double* dt_eff, double* umax)
{
    FTSP_GUARD(h, h->eng->step_info(dt_eff, umax));
    return FTSP_OK;
}

int ftsp_set_dt(ftsp_handle* h, double dt)
{
    FTSP_GUARD(h, h->eng->set_dt(dt));
    return FTSP_OK;
}

int ftsp_learn_configure(ftsp_handle* h, const ftsp_learn_config* cfg)
{
    if (!cfg) return FTSP_ERROR;
    FTSP_GUARD(h, h->eng->learn_configure(*cfg));
    return FTSP_OK;
}

int ftsp_learn_collect(ftsp_handle* h, int on)
{
    FTSP_GUARD(h, h->eng->learn_collect(on != 0));
    return FTSP_OK;
}

int ftsp_learn_reset(ftsp_handle* h)
{
    FTSP_GUARD(h, h->eng->learn_reset());
    return FTSP_OK;
}

int ftsp_learn_train(ftsp_handle* h, int iterations, double* loss)
{
    double l = 0.0;
    FTSP_GUARD(h, l = h->eng->learn_train(iterations));
    if (loss) *loss = l;
    return FTSP_OK;
}

int ftsp_learn_use(ftsp_handle* h, int on)
{
    FTSP_GUARD(h, h->eng->learn_use(on != 0));
    return FTSP_OK;
}

int ftsp_learn_get_stats(ftsp_handle* h, ftsp_learn_stats* st)
{
    if (!st) return FTSP_ERROR;
    FTSP_GUARD(h, h->eng->learn_stats(st));
    return FTSP_OK;
}

int ftsp_learn_get_weights(ftsp_handle* h, float* out, int* n)
{
    if (!n) return FTSP_ERROR;
    FTSP_GUARD(h, *n = h->eng->learn_weights(out, out ? *n : 0, false));
    return FTSP_OK;
}

int ftsp_learn_set_weights(ftsp_handle* h, const float* w, int n)
{
    if (!w) return FTSP_ERROR;
    FTSP_GUARD(h, h->eng->learn_weights(const_cast<float*>(w), n, true));
    return FTSP_OK;
}

int ftsp_learn_grad(ftsp_handle* h, const float* x, const float* t, const float* m, int n, double* loss, float* grad)
{
    if (!x || !t || !m || !grad) return FTSP_ERROR;
    double l = 0.0;
    FTSP_GUARD(h, l = h->eng->learn_grad(x, t, m, n, grad));
    if (loss) *loss = l;
    return FTSP_OK;
}

int ftsp_state_views(ftsp_handle* h, ftsp_views* v)
{
    if (!v) return FTSP_ERROR;
    FTSP_GUARD(h, h->eng->views(v));
    return FTSP_OK;
}

int ftsp_propagate_chain(ftsp_handle* h, const double* w, int N, double bond_length, double* q_end, double* Q)
{
    if (!w || !q_end) return FTSP_ERROR;
    FTSP_GUARD(h, h->eng->propagate_chain(reinterpret_cast<const double2*>(w), N, bond_length,
                                          reinterpret_cast<double2*>(q_end), Q));
    if (Q && !(std::isfinite(Q[0]) && std::isfinite(Q[1]))) return FTSP_NONFINITE;
    return FTSP_OK;
}

int ftsp_average_start(ftsp_handle* h, int skip, long long samples, int blocks)
{
    FTSP_GUARD(h, h->eng->average_start(skip, samples, blocks));
    return FTSP_OK;
}

int ftsp_average_read(ftsp_handle* h, double* mean, double* std_error, long long* count)
{
    long long n = 0;
    FTSP_GUARD(h, n = h->eng->average_read(mean, std_error));
    if (count) *count = n;
    return FTSP_OK;
}

int ftsp_rollback_info(ftsp_handle* h, long long* restarts, int* exhausted)
{
    FTSP_GUARD(h, {
        const long long r = h->eng->restarts();
        if (restarts) *restarts = r;
        if (exhausted) *exhausted = h->eng->restarts_exhausted() ? 1 : 0;
    });
    return FTSP_OK;
}

long long ftsp_restart_count(ftsp_handle* h)
{
    if (!h || !h->eng) return -1;
    try {
        return h->eng->restarts();
    } catch (const std::exception& e_) {
        h->err = e_.what();
        return -1;
    }
}

int ftsp_profile_enable(ftsp_handle* h, int on)
{
    FTSP_GUARD(h, {
        h->eng->prof_reset();
        h->eng->profiling = on != 0;
    });
    return FTSP_OK;
}

int ftsp_profile_read(ftsp_handle* h, ftsp_kernel_stat* out, int max_entries, int* count)
{
    FTSP_GUARD(h, {
        h->eng->prof_collect();
        const int n = (int)h->eng->prof.size();
        if (count) *count = n;
        for (int i = 0; i < n && out && i < max_entries; ++i) {
            const auto& p = h->eng->prof[i];
            std::snprintf(out[i].name, sizeof(out[i].name), "%s", p.first.c_str());
            out[i].ms = p.second.ms;
            out[i].launches = p.second.launches;
            out[i].bytes = p.second.bytes;
        }
    });
    return FTSP_OK;
}

long long ftsp_last_launch_count(const ftsp_handle* h)
{
    if (!h || !h->eng) return -1;
    return h->eng->launches;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Replica batches: the steps of many independent systems captured into one
// CUDA graph, each system on its own stream branch (fork/join through
// events), so kernels of different replicas run concurrently and a whole
// batch step costs one graph launch on the host.
// ---------------------------------------------------------------------------
struct ftsp_batch {
    std::vector<ftsp_handle*> hs;
    std::vector<cudaStream_t> saved;   // the handles' streams before the batch took them
    std::vector<cudaStream_t> rs;      // one branch stream per replica
    std::vector<cudaEvent_t> ev;
    cudaEvent_t fork = nullptr;
    cudaStream_t main = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int steps_per_graph = 1;
    int device = 0;
    long long launches = 0;            // kernels of one graph
    std::string err;

    void release()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        for (size_t i = 0; i < hs.size() && i < saved.size(); ++i)
            if (hs[i] && hs[i]->eng) hs[i]->eng->stream = saved[i];
        for (auto e : ev) cudaEventDestroy(e);
        for (auto s : rs) cudaStreamDestroy(s);
        ev.clear();
        rs.clear();
        if (fork) cudaEventDestroy(fork);
        if (main) cudaStreamDestroy(main);
        fork = nullptr;
        main = nullptr;
    }
};

namespace {
void batch_check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace

extern "C" {

int ftsp_batch_create(ftsp_handle* const* handles, int n, int steps_per_graph, ftsp_batch** out)
{
    if (!out || !handles || n < 1 || steps_per_graph < 1) {
        g_create_error = "ftsp_batch_create: bad argument";
        return FTSP_ERROR;
    }
    *out = nullptr;
    auto* b = new ftsp_batch();
    try {
        for (int i = 0; i < n; ++i) {
            if (!handles[i] || !handles[i]->eng) throw std::runtime_error("ftsp_batch_create: null handle");
            b->hs.push_back(handles[i]);
        }
        b->device = b->hs[0]->eng->c.device;
        for (auto* h : b->hs)
            if (h->eng->c.device != b->device) throw std::runtime_error("ftsp_batch_create: handles on different devices");
        b->steps_per_graph = steps_per_graph;
        batch_check(cudaSetDevice(b->device), "cudaSetDevice");
        batch_check(cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking), "cudaStreamCreate");
        batch_check(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "cudaEventCreate");
        for (int i = 0; i < n; ++i) {
            cudaStream_t s;
            cudaEvent_t e;
            batch_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
            b->rs.push_back(s);
            batch_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
            b->ev.push_back(e);
        }
        // finish whatever the handles queued on their own streams
        for (auto* h : b->hs) h->eng->install_pending_fields();   // before the capture
        for (auto* h : b->hs) batch_check(cudaStreamSynchronize(h->eng->stream), "cudaStreamSynchronize");
        for (int i = 0; i < n; ++i) {
            b->saved.push_back(b->hs[i]->eng->stream);
            b->hs[i]->eng->stream = b->rs[i];
        }
        batch_check(cudaStreamBeginCapture(b->main, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        try {
            for (int k = 0; k < steps_per_graph; ++k) {
                batch_check(cudaEventRecord(b->fork, b->main), "cudaEventRecord");
                for (int i = 0; i < n; ++i) {
                    batch_check(cudaStreamWaitEvent(b->rs[i], b->fork, 0), "cudaStreamWaitEvent");
                    b->hs[i]->eng->step(nullptr, nullptr, nullptr, false);
                    b->launches += b->hs[i]->eng->launches;
                    batch_check(cudaEventRecord(b->ev[i], b->rs[i]), "cudaEventRecord");
                    batch_check(cudaStreamWaitEvent(b->main, b->ev[i], 0), "cudaStreamWaitEvent");
                }
            }
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(b->main, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        batch_check(cudaStreamEndCapture(b->main, &b->graph), "cudaStreamEndCapture");
        batch_check(cudaGraphInstantiate(&b->exec, b->graph, 0), "cudaGraphInstantiate");
        *out = b;
        return FTSP_OK;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        b->release();
        delete b;
        return FTSP_ERROR;
    }
}

int ftsp_batch_step(ftsp_batch* b, int launches)
{
    if (!b || !b->exec) return FTSP_ERROR;
    for (int i = 0; i < launches; ++i) {
        const cudaError_t e = cudaGraphLaunch(b->exec, b->main);
        if (e != cudaSuccess) {
            b->err = std::string("cudaGraphLaunch: ") + cudaGetErrorString(e);
            return FTSP_ERROR;
        }
    }
    return FTSP_OK;
}

int ftsp_batch_sync(ftsp_batch* b)
{
    if (!b) return FTSP_ERROR;
    const cudaError_t e = cudaStreamSynchronize(b->main);
    if (e != cudaSuccess) {
        b->err = std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e);
        return FTSP_ERROR;
    }
    return FTSP_OK;
}

void* ftsp_batch_stream(ftsp_batch* b) { return b ? static_cast<void*>(b->main) : nullptr; }

long long ftsp_batch_launch_count(const ftsp_batch* b) { return b ? b->launches : -1; }

const char* ftsp_batch_last_error(const ftsp_batch* b) { return b ? b->err.c_str() : g_create_error.c_str(); }

void ftsp_batch_destroy(ftsp_batch* b)
{
    if (!b) return;
    if (b->main) cudaStreamSynchronize(b->main);
    b->release();
    delete b;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Chain propagation without any device allocation.
//
// For callers that cannot call cudaMalloc: code inside a framework whose
// caching allocator owns the device memory (e.g. a PyTorch process that has
// reserved the pool), and real-time loops that must not block on the
// driver's allocator.  It computes exactly what ftsp_propagate_chain
// computes, but all of its scratch lives in the single file-scope array
// below, so no call allocates or frees device memory.  The call is
// synchronous: it copies its tables from host memory into the array, and
// copies Q back to the host and waits for the stream before returning.
//
// Limits: at most NOALLOC_MAX_POINTS grid points (64^3) and NOALLOC_MAX_EXTENT
// points along any axis; complex128 only.  The array (about 8.3 MiB) is part
// of the library image, so every GPU that loads libftsp.so holds it until the
// process exits.  Every call on a device shares all of it, the tables
// included: calls whose work overlaps on the GPU (different host threads on
// different streams) race on it and must be serialised by the caller.  Each
// call writes every part of the scratch it later reads (the exp(-w) table,
// the intermediate field, the reduction partials, the FFT and bond tables),
// so no region has to start at zero and nothing carries over from the
// previous call.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t NOALLOC_MAX_POINTS = 262144;   // 64^3
constexpr int NOALLOC_MAX_EXTENT = 256;
constexpr size_t NA_FIELD = NOALLOC_MAX_POINTS * sizeof(double2);      // 4 MiB
constexpr size_t NA_PARTIALS_N = 16384;
constexpr size_t NA_PARTIALS = NA_PARTIALS_N * sizeof(double2);       // 256 KiB
constexpr size_t NA_TABLES = 64 * 1024;
constexpr size_t NA_BYTES = 2 * NA_FIELD + NA_PARTIALS + NA_TABLES;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

std::mutex g_noalloc_mutex;
constexpr int NA_MAX_DEVICES = 128;
unsigned char* g_noalloc_base[NA_MAX_DEVICES] = {};

// Small tables copied into the scratch at every call.
struct NoallocTables {
    ftsp::FftPlan1 plans[3];                 // x, y, z
    double2 tw[3][NOALLOC_MAX_EXTENT];       // exp(-2 pi i j / m_d)
    double phi[3 * NOALLOC_MAX_EXTENT];      // separable exp(-b^2 k_d^2 / 6)
    double qsum[2];                          // sum of q_N (combine output)
};
static_assert(sizeof(NoallocTables) <= NA_TABLES, "noalloc tables do not fit their region");

}  // namespace

namespace ftsp {
void set_thread_error(const std::string& s);
}

extern "C" int ftsp_propagate_chain_noalloc(int m1, int m2, int m3, double L1, double L2, double L3,
                                            const double* w, int N, double bond_length, double* q_end, double* Q,
                                            void* cuda_stream)
{
    using namespace ftsp;
    try {
        if (!w || !q_end || !Q) throw std::runtime_error("ftsp_propagate_chain_noalloc: null argument");
        if (m1 < 1 || m2 < 1 || m3 < 1) throw std::runtime_error("ftsp_propagate_chain_noalloc: invalid mesh");
        if (m1 > NOALLOC_MAX_EXTENT || m2 > NOALLOC_MAX_EXTENT || m3 > NOALLOC_MAX_EXTENT)
            throw std::runtime_error("ftsp_propagate_chain_noalloc: an extent exceeds the limit of " +
                                     std::to_string(NOALLOC_MAX_EXTENT));
        const size_t V = (size_t)m1 * m2 * m3;
        if (V > NOALLOC_MAX_POINTS)
            throw std::runtime_error("ftsp_propagate_chain_noalloc: " + std::to_string(V) +
                                     " grid points exceed the limit of " + std::to_string(NOALLOC_MAX_POINTS) +
                                     " (64^3); use ftsp_propagate_chain for larger grids");
        if (N < 1) throw std::runtime_error("ftsp_propagate_chain_noalloc: N must be >= 1");
        if (!(bond_length > 0.0)) throw std::runtime_error("ftsp_propagate_chain_noalloc: bond length must be positive");
        if (!(L1 > 0.0 && L2 > 0.0 && L3 > 0.0)) throw std::runtime_error("ftsp_propagate_chain_noalloc: box lengths must be positive");
        cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);

        // one-time set-up per device: the device address of the scratch array
        int dev = 0;
        FTSP_CUDA(cudaGetDevice(&dev));
        if (dev < 0 || dev >= NA_MAX_DEVICES) throw std::runtime_error("ftsp_propagate_chain_noalloc: device ordinal out of range");
        unsigned char* base = nullptr;
        {
            std::lock_guard<std::mutex> lock(g_noalloc_mutex);
            if (!g_noalloc_base[dev]) {
                void* ptr = nullptr;
                const cudaError_t err = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
                if (err != cudaSuccess)
                    throw std::runtime_error(std::string("ftsp_propagate_chain_noalloc: cudaGetSymbolAddress failed: ") +
                                             cudaGetErrorString(err));
                g_noalloc_base[dev] = static_cast<unsigned char*>(ptr);
            }
            base = g_noalloc_base[dev];
        }
        double2* Eb = reinterpret_cast<double2*>(base);
        double2* Gb = reinterpret_cast<double2*>(base + NA_FIELD);
        double2* partials = reinterpret_cast<double2*>(base + 2 * NA_FIELD);
        NoallocTables* dtab = reinterpret_cast<NoallocTables*>(base + 2 * NA_FIELD + NA_PARTIALS);

        // host tables: plans, twiddles, bond factors
        NoallocTables ht{};
        const int ms[3] = {m1, m2, m3};
        const double Ls[3] = {L1, L2, L3};
        for (int d = 0; d < 3; ++d) {
            ht.plans[d] = make_plan(ms[d], 3);   // complex128: radix <= 8
            for (int j = 0; j < ms[d]; ++j) {
                const long double ang = -2.0L * 3.141592653589793238462643383279502884L * j / ms[d];
                ht.tw[d][j] = make_double2((double)cosl(ang), (double)sinl(ang));
            }
        }
        int off = 0;
        for (int d = 0; d < 3; ++d)
            for (int i = 0; i < ms[d]; ++i) {
                const double k = wave_number(i, ms[d], Ls[d]);
                ht.phi[off++] = std::exp(-bond_length * bond_length * k * k / 6.0);
            }
        FTSP_CUDA(cudaMemcpyAsync(dtab, &ht, sizeof(ht), cudaMemcpyHostToDevice, stream));

        // launch geometry of the runtime-plan passes (complex128)
        int dev_smem = 0;
        FTSP_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        constexpr int EP = 16, EL = 8;
        auto round32 = [](int t) { return std::max(32, (t + 31) / 32 * 32); };
        PlaneGeom pg{};
        pg.m1 = m1; pg.m2 = m2; pg.m3 = m3; pg.P = m3 + 1;
        pg.py = &dtab->plans[1];
        pg.pz = &dtab->plans[2];
        pg.fm2 = make_fastdiv(m2);
        pg.fm3 = make_fastdiv(m3);
        const size_t plane_smem = std::max(sizeof(double2) * ((size_t)m2 * pg.P + m2 + m3), (size_t)4096);
        const int plane_threads = round32((m2 * m3 + EP - 1) / EP);
        const bool plane_ok = plane_smem <= (size_t)dev_smem && plane_threads <= 512;
        int W = 1;
        const int wmax = std::max(1, std::min(16, (EL * 256) / std::max(m1, m2)));
        for (int cand = 1; cand <= std::min(m3, wmax); ++cand)
            if (m3 % cand == 0) W = cand;
        LineGeom gx{m1, m2, m3, m1, W, 0, W, &dtab->plans[0], make_fastdiv(W), make_fastdiv(1), make_fastdiv(m2), make_fastdiv(m3)};
        LineGeom gy{m1, m2, m3, m2, W, 0, W, &dtab->plans[1], make_fastdiv(W), make_fastdiv(1), make_fastdiv(m2), make_fastdiv(m3)};
        int B = std::max(1, 2048 / m3);
        while ((m1 * m2) % B) --B;
        LineGeom gz{m1, m2, m3, m3, 0, B, m3 + 1, &dtab->plans[2], make_fastdiv(1), make_fastdiv(B), make_fastdiv(m2), make_fastdiv(m3)};
        const int x_threads = round32((m1 * W + EL - 1) / EL);
        const int y_threads = round32((m2 * W + EL - 1) / EL);
        const int z_threads = round32((B * m3 + EL - 1) / EL);
        const size_t x_smem = std::max(sizeof(double2) * ((size_t)m1 * W + m1), (size_t)4096);
        const size_t y_smem = std::max(sizeof(double2) * ((size_t)m2 * W + m2), (size_t)4096);
        const size_t z_smem = std::max(sizeof(double2) * ((size_t)B * (m3 + 1) + m3), (size_t)4096);
        if (x_threads > 256 || y_threads > 256 || z_threads > 256) throw std::runtime_error("ftsp_propagate_chain_noalloc: mesh too large for the line passes");
        const int parts = plane_ok ? m1 : m1 * m2 / B;
        if ((size_t)parts > NA_PARTIALS_N) throw std::runtime_error("ftsp_propagate_chain_noalloc: too many reduction partials");
        const double2* tw1 = dtab->tw[0];
        const double2* tw2 = dtab->tw[1];
        const double2* tw3 = dtab->tw[2];
        auto smem_attr = [&](auto kernel, size_t bytes) {
            if (bytes > 48 * 1024) FTSP_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
        };
        // real-space pass of one segment (plane, or y / z-line / y)
        auto seg = [&](auto s1c, auto s2c, const double2* src, double2* dst, const auto& op) {
            constexpr int S1 = decltype(s1c)::value, S2 = decltype(s2c)::value;
            using Op = std::decay_t<decltype(op)>;
            if (plane_ok) {
                auto k = k_plane<double, EP, S1, S2, Op>;
                smem_attr(k, plane_smem);
                k<<<dim3(m1, 1), plane_threads, plane_smem, stream>>>(pg, src, dst, V, tw2, tw3, op);
                return;
            }
            if (S1 != 0) {
                auto k = k_strided<double, EL, 1, 0, S1, OpLoadOne<double>>;
                smem_attr(k, y_smem);
                k<<<dim3(m1 * (m3 / W), 1), y_threads, y_smem, stream>>>(gy, nullptr, const_cast<double2*>(src), V, tw2, OpLoadOne<double>{src});
            }
            auto kz = k_zline<double, EL, S1, S2, Op>;
            smem_attr(kz, z_smem);
            kz<<<dim3(m1 * m2 / B, 1), z_threads, z_smem, stream>>>(gz, src, dst, V, tw3, op);
            if (S2 != 0) {
                auto k = k_strided<double, EL, 1, 0, S2, OpLoadOne<double>>;
                smem_attr(k, y_smem);
                k<<<dim3(m1 * (m3 / W), 1), y_threads, y_smem, stream>>>(gy, nullptr, dst, V, tw2, OpLoadOne<double>{dst});
            }
        };
        OpBond<double, true, false> ob{};
        ob.phix = dtab->phi;
        ob.phiy = dtab->phi + m1;
        ob.phiz = dtab->phi + m1 + m2;
        ob.invV = 1.0 / (double)V;
        auto kb = k_strided<double, EL, 0, -1, +1, OpBond<double, true, false>>;
        smem_attr(kb, x_smem);

        const double2* wp = reinterpret_cast<const double2*>(w);
        double2* qe = reinterpret_cast<double2*>(q_end);
        {
            const int blocks = (int)std::min<size_t>((V + 255) / 256, 148 * 16);
            k_foreach<<<std::max(1, blocks), 256, 0, stream>>>(V, [=] __device__(size_t i) {
                const double2 x = wp[i];
                Eb[i] = cexpT(-x.x, -x.y);
            });
        }
        using I0 = std::integral_constant<int, 0>;
        using Ip = std::integral_constant<int, +1>;
        using Im = std::integral_constant<int, -1>;
        if (N == 1) {
            OpProp<double, FWD_SINGLE> op{};
            op.E = Eb; op.qstore = qe; op.partial = partials;
            seg(I0{}, I0{}, nullptr, nullptr, op);
        } else {
            OpProp<double, FWD_START> op0{};
            op0.E = Eb; op0.qstore = qe;
            seg(I0{}, Im{}, nullptr, Gb, op0);
            for (int b = 0; b < N - 1; ++b) {
                kb<<<dim3(m2 * (m3 / W), 1), x_threads, x_smem, stream>>>(gx, Gb, Gb, V, tw1, ob);
                if (b + 1 < N - 1) {
                    OpProp<double, FWD_MID> op{};
                    op.E = Eb; op.qstore = qe;
                    seg(Ip{}, Im{}, Gb, Gb, op);
                } else {
                    OpProp<double, FWD_LAST> op{};
                    op.E = Eb; op.qstore = qe; op.partial = partials;
                    seg(Ip{}, I0{}, Gb, nullptr, op);
                }
            }
        }
        k_combine<false><<<2, 32, 0, stream>>>(reinterpret_cast<const double*>(partials), parts, 2, dtab->qsum);
        FTSP_CUDA(cudaGetLastError());
        double qs[2] = {0.0, 0.0};
        FTSP_CUDA(cudaMemcpyAsync(qs, dtab->qsum, sizeof(qs), cudaMemcpyDeviceToHost, stream));
        FTSP_CUDA(cudaStreamSynchronize(stream));
        Q[0] = qs[0] / (double)V;
        Q[1] = qs[1] / (double)V;
        if (!(std::isfinite(Q[0]) && std::isfinite(Q[1]))) return FTSP_NONFINITE;
        return FTSP_OK;
    } catch (const std::exception& e) {
        ftsp::set_thread_error(e.what());
        return FTSP_ERROR;
    }
}
