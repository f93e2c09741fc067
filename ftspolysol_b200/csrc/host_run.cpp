// The reference program on the engine: command line, setup, the step loop
// with its output files and non-finite restarts, final outputs
// (main.cu:9-93, complexLangevin.cu:191-230 and 345-698).
//
// One ftsp_step call does what run_step does between its finite checks
// (densities, noise, drifts, predictor, densities at the predictor,
// observables, corrector); the loop around it reproduces the reference's
// bookkeeping: observables every max(1, Nss) steps and their average over
// the Ns steps after Nss, drift maxima after N_stat, tmp checkpoints every
// Ntmp steps (written as .new files and renamed), restarts from the last
// checkpoint on a non-finite value, at most max_nan_restarts times, step
// outputs after Nso, and the final fields and densities.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <memory>
#include <string>
#include <vector>

#include "ftsp.h"
#include "ftsp_host.h"
#include "host_io.h"
#include "host_model.h"

struct ftsp_model {
    ftsp::host::Model m;
};

namespace ftsp {
void set_thread_error(const std::string& s);
}

namespace ftsp {
namespace host {
namespace {

constexpr int STEP_W = 10;   // step column width (complexLangevin.cu:13-17)
constexpr int VALUE_W = 22;
constexpr int VALUE_P = 10;

std::string clean(std::string n)
{
    for (char& c : n)
        if (!std::isalnum((unsigned char)c) && c != '_' && c != '-') c = '_';
    return n;
}

// Column labels of the observables file (complexLangevin.cu:19-62).
std::vector<std::string> observable_labels(const Model& m)
{
    const Param& p = m.p;
    std::vector<std::string> L;
    auto poly = [&](const char* suf) {
        for (int i = 0; i < p.species_count; ++i) {
            if (p.species_count == 1) L.push_back(std::string("mu_poly_") + suf);
            else {
                const std::string name = i < (int)p.polymer_species.size() ? p.polymer_species[(size_t)i].name : "P" + std::to_string(i);
                L.push_back("mu_poly" + std::to_string(i) + "_" + clean(name) + "_" + suf);
            }
        }
    };
    auto ion = [&](const char* suf) {
        for (size_t j = 0; j < m.ions.size(); ++j) L.push_back("mu_ion" + std::to_string(j) + "_" + m.ions[j].name + "_" + suf);
    };
    poly("ex"); poly("id"); poly("self");
    ion("ex"); ion("id"); ion("self");
    L.push_back("Hmf_density_real");
    L.push_back("Hmf_density_imag");
    if (p.stress) {
        static const char* names[6] = {"stress_xx", "stress_yy", "stress_zz", "stress_xy", "stress_xz", "stress_yz"};
        for (int c = 0; c < 6; ++c)
            if (p.comp[c]) L.push_back(names[c]);
        if (p.isotropic_pressure) L.push_back("pressure_iso");
    }
    return L;
}

// Engine record (chemical[S+J], chemical_self[S+J], chemical_ideal[S+J], H,
// stress...) -> file columns (complexLangevin.cu:72-92): polymer ex, id,
// self, ion ex, id, self, Re H, Im H, Re stress...
std::vector<double> observable_values(const Model& m, const std::vector<double>& rec)
{
    const int S = (int)m.species.size(), J = (int)m.ions.size(), C = S + J;
    auto re = [&](int i) { return rec[(size_t)2 * i]; };
    std::vector<double> v;
    for (int i = 0; i < S; ++i) v.push_back(re(i));
    for (int i = 0; i < S; ++i) v.push_back(re(2 * C + i));
    for (int i = 0; i < S; ++i) v.push_back(re(C + i));
    for (int j = 0; j < J; ++j) v.push_back(re(S + j));
    for (int j = 0; j < J; ++j) v.push_back(re(2 * C + S + j));
    for (int j = 0; j < J; ++j) v.push_back(re(C + S + j));
    v.push_back(rec[(size_t)2 * 3 * C]);
    v.push_back(rec[(size_t)2 * 3 * C + 1]);
    const int R = (int)rec.size() / 2;
    for (int k = 3 * C + 1; k < R; ++k) v.push_back(re(k));
    return v;
}

bool finite_all(const std::vector<double>& v)
{
    for (double x : v)
        if (!std::isfinite(x)) return false;
    return true;
}

void error(const std::string& s) { std::fprintf(stderr, "error: %s\n", s.c_str()); }

struct Runner {
    Model& m;
    Param& p;
    ftsp_handle* h = nullptr;
    bool screenprint = false;
    std::vector<std::string> labels;
    std::vector<int> widths;
    FILE* obs = nullptr;
    FILE* drift = nullptr;
    std::vector<double> obs_sum;
    long long obs_count = 0;
    double obs_wsum = 0.0;     // sum of the step weights (adaptive step)
    bool adaptive = false;
    bool ck_valid = false;
    int ck_step = -1;
    int restarts = 0;
    size_t V;

    Runner(Model& mm, ftsp_handle* hh, bool sp) : m(mm), p(mm.p), h(hh), screenprint(sp), V((size_t)mm.size())
    {
        labels = observable_labels(m);
        for (const std::string& l : labels) widths.push_back(std::max(VALUE_W, (int)l.size()));
    }
    ~Runner()
    {
        if (obs) std::fclose(obs);
        if (drift) std::fclose(drift);
    }

    bool engine(int rc, const char* what)
    {
        if (rc == FTSP_OK) return true;
        error(std::string(what) + ": " + ftsp_last_error(h));
        return false;
    }

    void write_labels(FILE* fp, const char* first)
    {
        std::fprintf(fp, "#%*s", STEP_W - 1, first);
        for (size_t i = 0; i < labels.size(); ++i) std::fprintf(fp, " %*s", widths[i], labels[i].c_str());
    }
    void write_values(FILE* fp, const std::vector<double>& v)
    {
        for (size_t i = 0; i < v.size(); ++i) std::fprintf(fp, " % *.*e", i < widths.size() ? widths[i] : VALUE_W, VALUE_P, v[i]);
    }
    void obs_header()
    {
        std::fprintf(obs, "# observables Nss=%d Ns=%d\n", p.Nss, p.Ns);
        write_labels(obs, "step");
        std::fprintf(obs, "\n");
        std::fflush(obs);
    }
    bool drift_enabled() const { return p.N_stat >= 0 && !p.drift_max_file.empty(); }
    void drift_header()
    {
        std::fprintf(drift, "#%*s", STEP_W - 1, "step");
        for (int a = 0; a < m.n_modes(); ++a) {
            const std::string l = "u_omega" + std::to_string(a) + "_max";
            std::fprintf(drift, " %*s", VALUE_W, l.c_str());
        }
        std::fprintf(drift, " %*s\n", VALUE_W, "u_psi_max");
        std::fflush(drift);
    }

    bool open_outputs()
    {
        if (!p.observable_file.empty()) {
            obs = std::fopen(p.observable_file.c_str(), "w");
            if (!obs) return error("cannot open " + p.observable_file), false;
            obs_sum.assign(labels.size(), 0.0);
            obs_count = 0;
            obs_wsum = 0.0;
            obs_header();
        }
        if (drift_enabled()) {
            drift = std::fopen(p.drift_max_file.c_str(), "w");
            if (!drift) return error("cannot open " + p.drift_max_file), false;
            drift_header();
        }
        return true;
    }

    bool fetch(const char* name, std::vector<double>& out)
    {
        long long n = 0;
        if (!engine(ftsp_get_field(h, name, nullptr, &n), "get_field")) return false;
        out.assign((size_t)n, 0.0);
        return n == 0 || engine(ftsp_get_field(h, name, out.data(), &n), "get_field");
    }

    // Returns 1 ok, 0 non-finite fields, -1 I/O failure.
    int write_checkpoint(int step)
    {
        std::vector<double> om, ps;
        if (!fetch("omega", om) || !fetch("psi", ps)) return -1;
        if (!finite_all(om) || !finite_all(ps)) {
            std::fprintf(stderr, "error: non-finite value at step %d in checkpoint fields\n", step);
            return 0;
        }
        const std::string no = p.tmp_omega_file + ".new", np = p.tmp_psi_file + ".new";
        std::string err;
        if (!write_omega(m, no, om, err)) return error(err), -1;
        if (!write_fields(np, p, ps.data(), 1, V, err)) {
            std::remove(no.c_str());
            return error(err), -1;
        }
        if (std::rename(no.c_str(), p.tmp_omega_file.c_str()) != 0) {
            error("cannot replace " + p.tmp_omega_file + " with " + no + ": " + std::strerror(errno));
            std::remove(no.c_str());
            std::remove(np.c_str());
            return -1;
        }
        if (std::rename(np.c_str(), p.tmp_psi_file.c_str()) != 0) {
            error("cannot replace " + p.tmp_psi_file + " with " + np + ": " + std::strerror(errno));
            std::remove(np.c_str());
            return -1;
        }
        ck_valid = true;
        ck_step = step;
        return 1;
    }

    // complexLangevin.cu:600-649
    bool restart(int failed)
    {
        if (p.Ntmp <= 0 || !ck_valid || ck_step < 0) return error("non-finite value encountered before a valid checkpoint was written"), false;
        if (restarts >= p.max_nan_restarts) return error("maximum non-finite restarts exceeded"), false;
        ++restarts;
        std::vector<double> om, ps;
        std::string err;
        if (!read_omega_exact(m, p.tmp_omega_file, om, err) || !read_complex_exact(m, p.tmp_psi_file, ps, err)) return error(err), false;
        if (!finite_all(om) || !finite_all(ps)) {
            error("checkpoint restart has non-finite value at step " + std::to_string(failed));
            return false;
        }
        if (!engine(ftsp_set_fields(h, om.empty() ? nullptr : om.data(), ps.data()), "set_fields")) return false;
        if (obs) {
            std::fclose(obs);
            obs = nullptr;
        }
        obs_sum.clear();
        obs_count = 0;
        obs_wsum = 0.0;
        if (!p.observable_file.empty()) {
            obs = std::fopen(p.observable_file.c_str(), "w");
            if (!obs) return error("cannot open " + p.observable_file), false;
            obs_sum.assign(labels.size(), 0.0);
            obs_header();
            std::fprintf(obs, "# restarted after non-finite value at step %d from checkpoint step %d; previous observable records discarded\n",
                         failed, ck_step);
            std::fflush(obs);
        }
        if (drift) {
            std::fclose(drift);
            drift = nullptr;
        }
        if (drift_enabled()) {
            drift = std::fopen(p.drift_max_file.c_str(), "w");
            if (!drift) return error("cannot open " + p.drift_max_file), false;
            drift_header();
            std::fprintf(drift, "# restarted after non-finite value at step %d from checkpoint step %d; previous drift statistics discarded\n",
                         failed, ck_step);
            std::fflush(drift);
        }
        return true;
    }

    bool step_outputs_enabled() const
    {
        return p.Nso >= 0 && (!p.step_omega_file.empty() || !p.step_psi_file.empty() || !p.step_rho_type_file.empty() ||
                              !p.step_rhop_file.empty() || !p.step_rhoc_file.empty() || !p.step_rhoc_poly_file.empty() ||
                              !p.step_rhoc_ion_file.empty() || !p.step_ion_density_prefix.empty());
    }

    // complexLangevin.cu:510-561.  Returns 1 ok, 0 non-finite, -1 failure.
    int step_outputs(int step)
    {
        if (!step_outputs_enabled()) return 1;
        const int first = p.Nso > 1 ? p.Nso : 1;
        if (step < first) return 1;
        const int index = step - first + 1;
        const bool want_density = !p.step_rho_type_file.empty() || !p.step_rhop_file.empty() || !p.step_rhoc_file.empty() ||
                                  !p.step_rhoc_poly_file.empty() || !p.step_rhoc_ion_file.empty() || !p.step_ion_density_prefix.empty();
        if (want_density) {
            std::vector<double> Q(2 * m.species.size());
            if (!engine(ftsp_compute_densities(h, 0, Q.data()), "compute_densities")) return -1;
            if (!finite_all(Q)) {
                std::fprintf(stderr, "error: non-finite value at step %d in Q(step output)\n", step);
                return 0;
            }
        }
        struct Out {
            const std::string* pattern;
            const char* field;
            int kind;   // 0 omega, 1 single complex, 2 rho_type, 3 ions
        } outs[] = {{&p.step_omega_file, "omega", 0},       {&p.step_psi_file, "psi", 1},
                    {&p.step_rho_type_file, "rho_type", 2}, {&p.step_rhop_file, "rho_p", 1},
                    {&p.step_rhoc_file, "rho_c", 1},        {&p.step_rhoc_poly_file, "rho_c_poly", 1},
                    {&p.step_rhoc_ion_file, "rho_c_ion", 1}, {&p.step_ion_density_prefix, "ion_rho", 3}};
        std::vector<std::vector<double>> data(8);
        for (int i = 0; i < 8; ++i) {
            if (outs[i].pattern->empty()) continue;
            if (outs[i].kind == 3 && m.ions.empty()) continue;
            if (!fetch(outs[i].field, data[(size_t)i])) return -1;
            if (!finite_all(data[(size_t)i])) {
                std::fprintf(stderr, "error: non-finite value at step %d in step-output %s\n", step, outs[i].field);
                return 0;
            }
        }
        bool ok = true;
        std::string err;
        for (int i = 0; i < 8; ++i) {
            if (outs[i].pattern->empty()) continue;
            const std::string f = step_filename(*outs[i].pattern, index);
            const std::vector<double>& d = data[(size_t)i];
            switch (outs[i].kind) {
            case 0: ok = write_omega(m, f, d, err) && ok; break;
            case 1: ok = write_fields(f, p, d.data(), 1, V, err) && ok; break;
            case 2: ok = write_fields(f, p, d.data(), p.monomer_type_count, V, err) && ok; break;
            default: ok = write_ion_densities(m, f, d, err) && ok; break;
            }
        }
        if (!ok) error(err);
        return ok ? 1 : -1;
    }

    // Returns 1 ok, 0 non-finite, -1 failure.
    int one_step(int step)
    {
        const int S = (int)m.species.size();
        const int R = ftsp_record_length(h);
        std::vector<double> Qb(2 * (size_t)S), rec(2 * (size_t)std::max(0, R)), dmax((size_t)m.n_modes() + 1);
        const int rc = ftsp_step(h, Qb.data(), rec.data(), dmax.data());
        if (rc == FTSP_NONFINITE) {
            std::fprintf(stderr, "error: non-finite value at step %d\n", step);
            return 0;
        }
        if (!engine(rc, "step")) return -1;
        const std::vector<double> v = observable_values(m, rec);
        if (!finite_all(v) || !finite_all(dmax)) {
            std::fprintf(stderr, "error: non-finite value at step %d in observables\n", step);
            return 0;
        }
        // accumulate (complexLangevin.cu:424-441); with the adaptive step each
        // record is weighted by its step dt_eff / dt (time average)
        double wgt = 1.0;
        if (adaptive) {
            double dt_eff = p.dt;
            if (!engine(ftsp_step_info(h, &dt_eff, nullptr), "step_info")) return -1;
            wgt = p.dt > 0.0 ? dt_eff / p.dt : 1.0;
        }
        if (step > p.Nss && obs_count < p.Ns && !obs_sum.empty()) {
            obs_wsum += wgt;
            for (size_t c = 0; c < v.size(); ++c) {
                obs_sum[c] += wgt * v[c];
                if (!std::isfinite(obs_sum[c])) {
                    std::fprintf(stderr, "error: non-finite value at step %d in %s_sum\n", step, labels[c].c_str());
                    return -1;
                }
            }
            ++obs_count;
        }
        if (obs && step % std::max(1, p.Nss) == 0) {
            std::fprintf(obs, "%*d", STEP_W, step);
            write_values(obs, v);
            std::fprintf(obs, "\n");
            std::fflush(obs);
        }
        if (screenprint) {
            for (double x : v) std::printf("% 13.4e", x);
            std::printf("\n");
        }
        if (drift && step > p.N_stat) {
            std::fprintf(drift, "%*d", STEP_W, step);
            for (double x : dmax) std::fprintf(drift, " % *.*e", VALUE_W, VALUE_P, x);
            std::fprintf(drift, "\n");
            std::fflush(drift);
        }
        return step_outputs(step);
    }

    bool run()
    {
        if (!open_outputs()) return false;
        if (p.Ntmp > 0 && write_checkpoint(0) != 1) return false;
        int step = 0;
        while (step < p.Nt) {
            const int next = step + 1;
            const int st = one_step(next);
            if (st < 0) return false;
            if (st == 0) {
                if (!restart(next)) return false;
                step = ck_step;
                continue;
            }
            step = next;
            if (p.Ntmp > 0 && step % p.Ntmp == 0) {
                const int c = write_checkpoint(step);
                if (c < 0) return false;
                if (c == 0) {
                    if (!restart(step)) return false;
                    step = ck_step;
                    continue;
                }
            }
        }
        // ensemble average (complexLangevin.cu:443-467)
        if (obs) {
            std::fprintf(obs, "\n# ensemble_average Nss=%d Ns=%d count=%lld\n", p.Nss, p.Ns, obs_count);
            if (obs_count == 0) {
                std::fprintf(obs, "# no_observables\n");
            } else {
                std::vector<double> avg;
                for (double s : obs_sum) avg.push_back(adaptive ? s / obs_wsum : s / (double)obs_count);
                write_labels(obs, "stat");
                std::fprintf(obs, "\n");
                std::fprintf(obs, "%*s", STEP_W, "average");
                write_values(obs, avg);
                std::fprintf(obs, "\n");
            }
            std::fflush(obs);
        }
        return true;
    }

    // Final densities and files (main.cu:76-89, fieldIO.cu:710-726).
    bool finish()
    {
        std::vector<double> Q(2 * m.species.size());
        if (!engine(ftsp_compute_densities(h, 0, Q.data()), "compute_densities")) return false;
        if (!finite_all(Q)) return error("non-finite value in Q(final)"), false;
        std::vector<double> om, ps, rt, rp, rc, rcp, rci, ir;
        if (!fetch("omega", om) || !fetch("psi", ps) || !fetch("rho_type", rt) || !fetch("rho_p", rp) || !fetch("rho_c", rc) ||
            !fetch("rho_c_poly", rcp) || !fetch("rho_c_ion", rci))
            return false;
        if (!m.ions.empty() && !fetch("ion_rho", ir)) return false;
        const std::pair<const char*, std::vector<double>*> all[] = {{"omega", &om},          {"psi", &ps},   {"rho_type", &rt},
                                                                    {"rho_p", &rp},          {"rho_c", &rc}, {"rho_c_poly", &rcp},
                                                                    {"rho_c_ion", &rci},     {"ion_rho", &ir}};
        for (const auto& f : all)
            if (!finite_all(*f.second)) return error(std::string("non-finite value in output ") + f.first), false;
        std::string err;
        const bool ok = write_omega(m, p.omega_file, om, err) && write_fields(p.psi_file, p, ps.data(), 1, V, err) &&
                        write_fields(p.rho_type_file, p, rt.data(), p.monomer_type_count, V, err) &&
                        write_fields(p.rhop_file, p, rp.data(), 1, V, err) && write_fields(p.rhoc_file, p, rc.data(), 1, V, err) &&
                        write_fields(p.rhoc_poly_file, p, rcp.data(), 1, V, err) &&
                        write_fields(p.rhoc_ion_file, p, rci.data(), 1, V, err) && write_ion_densities(m, p.ion_density_prefix, ir, err);
        if (!ok) error(err);
        return ok;
    }
};

void print_setup(const Options& o, const Model& m, const RunPaths& r)
{
    const Param& p = m.p;
    std::printf("parameter file = %s\n", o.param_file.c_str());
    if (!r.run.empty()) std::printf("run directory = %s\n", r.run.c_str());
    std::printf("omega input file = %s\n", r.input_omega.c_str());
    if (m.elec()) std::printf("psi input file = %s\n", r.input_psi.c_str());
    else std::printf("psi input file = ignored (electrostatics disabled)\n");
    std::printf("omega output file = %s\n", p.omega_file.c_str());
    std::printf("psi output file = %s\n", p.psi_file.c_str());
    if (p.Ntmp > 0) {
        std::printf("tmp omega checkpoint file = %s\n", p.tmp_omega_file.c_str());
        std::printf("tmp psi checkpoint file = %s\n", p.tmp_psi_file.c_str());
    }
    std::printf("observable file = %s\n", p.observable_file.c_str());
    std::printf("sequence file = %s\n", p.sequence_file.c_str());
    std::printf("monomer types (M = %d):", p.monomer_type_count);
    for (const std::string& n : p.monomer_names) std::printf(" %s", n.c_str());
    std::printf("\n");
    for (size_t l = 0; l < m.modes.eig.size(); ++l) std::printf("mode %zu eigenvalue = % .10e\n", l, m.modes.eig[l]);
    for (size_t k = 0; k < m.species.size(); ++k)
        std::printf("polymer species %zu: name=%s n=%lld N=%zu\n", k, m.species[k].name.c_str(), m.species[k].num_chains,
                    m.species[k].type.size());
    std::printf("m1 m2 m3 = %d %d %d\n", p.m1, p.m2, p.m3);
    std::printf("L1 L2 L3 = % 13.4e % 13.4e % 13.4e\n", p.L1, p.L2, p.L3);
    std::printf("reduced density total_segments/V = % 13.4e\n", p.rho0);
    std::printf("short_range_self_pressure = % 13.4e\n", m.self_pressure);
    std::printf("lB = % 13.4e%s\n", p.lB, m.elec() ? "" : " (electrostatics disabled)");
    std::printf("dt = % 13.4e\nlambdaPsi = % 13.4e\nNt = %d\nNss = %d\nNs = %d\nNtmp = %d\nNso = %d\n", p.dt, p.lambdaPsi, p.Nt, p.Nss,
                p.Ns, p.Ntmp, p.Nso);
    std::printf("noise = %s\n", p.noise ? "on" : "off");
    for (size_t j = 0; j < m.ions.size(); ++j)
        std::printf("ion[%zu] %s z=% 13.4e n=%lld smearing=% 13.4e density=% 13.4e\n", j, m.ions[j].name.c_str(), m.ions[j].valence,
                    m.ions[j].count, m.ions[j].smearing, (double)m.ions[j].count / m.volume());
    std::printf("engine = %s, %s\n", o.precision == FTSP_FP32 ? "complex64" : "complex128",
                o.scheme == FTSP_SCHEME_SI ? "semi-implicit" : "predictor-corrector");
}

int run_main(int argc, char** argv)
{
    const auto t0 = std::chrono::steady_clock::now();
    Options o;
    std::string err;
    const int pa = parse_args(argc, argv, o, err);
    if (pa == 1) {
        usage(argc > 0 ? argv[0] : "ftsp_main");
        return 0;
    }
    if (pa < 0) {
        error(err);
        usage(argc > 0 ? argv[0] : "ftsp_main");
        return 1;
    }
    Model m;
    if (!load_model(o.param_file, o.sequence_override ? o.sequence_file : std::string(), m, err)) return error(err), 1;
    RunPaths r;
    if (!prepare_run(o, m.p, r, err)) return error(err), 1;
    if (o.screenprint) print_setup(o, m, r);
    std::vector<double> omega, psi;
    if (!read_omega_input(m, r, omega, o.screenprint, err)) return error(err), 1;
    if (m.elec()) {
        if (!read_psi_input(m, r, psi, o.screenprint, err)) return error(err), 1;
    } else {
        psi.assign(2 * (size_t)m.size(), 0.0);
    }
    if (!finite_all(omega) || !finite_all(psi)) return error("non-finite value in input fields"), 1;

    ftsp_config cfg;
    fill_config(m, cfg);
    cfg.precision = o.precision;
    cfg.scheme = o.scheme;
    cfg.device = o.device;
    cfg.restart_interval = 0;
    cfg.autotune = o.autotune;
    if (o.seed_set) cfg.seed = o.seed;
    else {
        // a fresh seed per run, like the reference's clock-derived curand seeds
        timespec ts;
        clock_gettime(CLOCK_REALTIME, &ts);
        cfg.seed = (unsigned long long)ts.tv_nsec ^ ((unsigned long long)ts.tv_sec << 30);
    }
    ftsp_handle* hraw = nullptr;
    if (ftsp_create(&cfg, &hraw) != FTSP_OK) return error(std::string("engine: ") + ftsp_last_error(nullptr)), 1;
    std::unique_ptr<ftsp_handle, int (*)(ftsp_handle*)> h(hraw, ftsp_destroy);
    if (ftsp_set_fields(h.get(), omega.empty() ? nullptr : omega.data(), psi.data()) != FTSP_OK)
        return error(std::string("engine: ") + ftsp_last_error(h.get())), 1;
    if (o.adaptive > 0.0 && ftsp_set_adaptive(h.get(), o.adaptive) != FTSP_OK)
        return error(std::string("engine: ") + ftsp_last_error(h.get())), 1;
    bool ok;
    {
        Runner run(m, h.get(), o.screenprint);
        run.adaptive = o.adaptive > 0.0;
        ok = run.run() && run.finish();
    }
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("total time = % .4e s\n", sec);
    std::fflush(stdout);
    return ok ? 0 : 1;
}

}  // namespace
}  // namespace host
}  // namespace ftsp

extern "C" {

int ftsp_model_load(const char* param_file, const char* sequence_file, ftsp_model** out)
{
    if (!param_file || !out) {
        ftsp::set_thread_error("ftsp_model_load: null argument");
        return FTSP_ERROR;
    }
    *out = nullptr;
    try {
        std::unique_ptr<ftsp_model> m(new ftsp_model());
        std::string err;
        if (!ftsp::host::load_model(param_file, sequence_file ? sequence_file : "", m->m, err)) {
            ftsp::set_thread_error(err);
            return FTSP_ERROR;
        }
        *out = m.release();
        return FTSP_OK;
    } catch (const std::exception& e) {
        ftsp::set_thread_error(e.what());
        return FTSP_ERROR;
    }
}

void ftsp_model_free(ftsp_model* m) { delete m; }

int ftsp_model_config(ftsp_model* m, ftsp_config* cfg)
{
    if (!m || !cfg) {
        ftsp::set_thread_error("ftsp_model_config: null argument");
        return FTSP_ERROR;
    }
    ftsp::host::fill_config(m->m, *cfg);
    return FTSP_OK;
}

int ftsp_model_get_info(const ftsp_model* mm, ftsp_model_info* info)
{
    if (!mm || !info) {
        ftsp::set_thread_error("ftsp_model_get_info: null argument");
        return FTSP_ERROR;
    }
    const ftsp::host::Model& m = mm->m;
    const ftsp::host::Param& p = m.p;
    std::memset(info, 0, sizeof(*info));
    info->m1 = p.m1; info->m2 = p.m2; info->m3 = p.m3;
    info->M = p.monomer_type_count;
    info->n_modes = m.n_modes();
    info->n_species = (int)m.species.size();
    info->n_ions = (int)m.ions.size();
    info->Nt = p.Nt; info->Nss = p.Nss; info->Ns = p.Ns; info->Ntmp = p.Ntmp; info->Nso = p.Nso; info->N_stat = p.N_stat;
    info->max_nan_restarts = p.max_nan_restarts;
    info->noise = p.noise ? 1 : 0;
    info->legacy_ab = m.legacy_ab() ? 1 : 0;
    info->rho0 = p.rho0;
    info->volume = m.volume();
    info->self_pressure = m.self_pressure;
    info->eigen_tol_abs = m.modes.tol_abs;
    info->total_segments = p.total_segments;
    return FTSP_OK;
}

int ftsp_model_modes(const ftsp_model* mm, double* eig, double* O)
{
    if (!mm) {
        ftsp::set_thread_error("ftsp_model_modes: null argument");
        return FTSP_ERROR;
    }
    const ftsp::host::Modes& md = mm->m.modes;
    if (eig) std::copy(md.eig.begin(), md.eig.end(), eig);
    if (O) std::copy(md.O.begin(), md.O.end(), O);
    return FTSP_OK;
}

int ftsp_model_read_fields(const ftsp_model* mm, const char* omega_file, const char* psi_file, double* omega, double* psi)
{
    if (!mm || !omega || !psi) {
        ftsp::set_thread_error("ftsp_model_read_fields: null argument");
        return FTSP_ERROR;
    }
    try {
        const ftsp::host::Model& m = mm->m;
        ftsp::host::RunPaths r;
        r.input_omega = omega_file ? omega_file : m.p.omega_file;
        r.input_psi = psi_file ? psi_file : m.p.psi_file;
        r.zero_missing_default_omega = !omega_file && r.input_omega == "omega.rf";
        std::vector<double> om, ps;
        std::string err;
        if (!ftsp::host::read_omega_input(m, r, om, false, err)) {
            ftsp::set_thread_error(err);
            return FTSP_ERROR;
        }
        if (m.elec()) {
            if (!ftsp::host::read_psi_input(m, r, ps, false, err)) {
                ftsp::set_thread_error(err);
                return FTSP_ERROR;
            }
        } else {
            ps.assign(2 * (size_t)m.size(), 0.0);
        }
        std::copy(om.begin(), om.end(), omega);
        std::copy(ps.begin(), ps.end(), psi);
        return FTSP_OK;
    } catch (const std::exception& e) {
        ftsp::set_thread_error(e.what());
        return FTSP_ERROR;
    }
}

int ftsp_model_write_omega(const ftsp_model* mm, const char* file, const double* omega)
{
    if (!mm || !file || (!omega && mm->m.n_modes() > 0)) {
        ftsp::set_thread_error("ftsp_model_write_omega: null argument");
        return FTSP_ERROR;
    }
    const size_t n = 2 * (size_t)mm->m.n_modes() * (size_t)mm->m.size();
    std::vector<double> om(omega, omega + n);
    std::string err;
    if (!ftsp::host::write_omega(mm->m, file, om, err)) {
        ftsp::set_thread_error(err);
        return FTSP_ERROR;
    }
    return FTSP_OK;
}

int ftsp_model_write_fields(const ftsp_model* mm, const char* file, int count, const double* fields)
{
    if (!mm || !file || count < 0 || (!fields && count > 0)) {
        ftsp::set_thread_error("ftsp_model_write_fields: bad argument");
        return FTSP_ERROR;
    }
    std::string err;
    if (!ftsp::host::write_fields(file, mm->m.p, fields, count, (size_t)mm->m.size(), err)) {
        ftsp::set_thread_error(err);
        return FTSP_ERROR;
    }
    return FTSP_OK;
}

int ftsp_main(int argc, char** argv)
{
    try {
        return ftsp::host::run_main(argc, argv);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
}

}  // extern "C"
