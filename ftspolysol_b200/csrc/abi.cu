// C ABI of the engine (include/ftsp.h): configuration checks and the
// extern "C" entry points.  Every entry point catches C++ exceptions and
// CUDA errors and turns them into status codes; nothing calls exit().
#include "engine.cuh"

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
    FTSP_GUARD(h, h->eng->stream = static_cast<cudaStream_t>(s));
    return FTSP_OK;
}

int ftsp_set_fields(ftsp_handle* h, const double* omega, const double* psi)
{
    if (!psi) return FTSP_ERROR;
    FTSP_GUARD(h, h->eng->set_fields(omega, psi));
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
    FTSP_GUARD(h, h->eng->c.seed = seed);
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
