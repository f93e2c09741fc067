// Host-side model setup (see host_model.h for the reference routines it
// follows).  Error texts follow the reference's "error: ..." messages
// (errHandle.cu:3-63) but are returned, never printed-and-exited.
#include "host_model.h"

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <numeric>
#include <sstream>

namespace ftsp {
namespace host {

namespace {

constexpr double PI_ = 3.141592653589793238462643383279502884;

struct Fail {
    std::string msg;
};
[[noreturn]] void fail(const std::string& m) { throw Fail{m}; }

std::string open_error(const std::string& path)
{
    std::string t = "cannot open " + path;
    if (errno) t += ": " + std::string(std::strerror(errno));
    return t;
}

bool is_sep(char c) { return std::isspace(static_cast<unsigned char>(c)) || c == ',' || c == ';' || c == '[' || c == ']'; }

bool parse_bool(const std::string& v, bool& out)
{
    std::string t = unquote(v);
    for (char& c : t) c = (char)std::tolower((unsigned char)c);
    if (t == "true" || t == "1" || t == "yes" || t == "on") return out = true, true;
    if (t == "false" || t == "0" || t == "no" || t == "off") return out = false, true;
    return false;
}
bool parse_real(const std::string& v, double& out)
{
    const std::string t = unquote(v);
    char* end = nullptr;
    out = std::strtod(t.c_str(), &end);
    return end != t.c_str() && *end == '\0';
}
bool parse_int64(const std::string& v, long long& out)
{
    const std::string t = unquote(v);
    char* end = nullptr;
    out = std::strtoll(t.c_str(), &end, 10);
    return end != t.c_str() && *end == '\0';
}
bool parse_int(const std::string& v, int& out)
{
    long long x = 0;
    if (!parse_int64(v, x)) return false;
    out = (int)x;
    return (long long)out == x;
}

int bracket_delta(const std::string& t)
{
    int d = 0;
    bool q = false;
    char qc = 0;
    for (size_t i = 0; i < t.size(); ++i) {
        const char c = t[i];
        if ((c == '"' || c == '\'') && (i == 0 || t[i - 1] != '\\')) {
            if (!q) { q = true; qc = c; }
            else if (qc == c) q = false;
            continue;
        }
        if (q) continue;
        if (c == '[') ++d;
        else if (c == ']') --d;
    }
    return d;
}

std::vector<std::string> bracket_tokens(std::string v)
{
    for (char& c : v)
        if (c == '[' || c == ']' || c == ',' || c == ';') c = ' ';
    std::istringstream in(v);
    std::vector<std::string> out;
    std::string tok;
    while (in >> tok) out.push_back(unquote(tok));
    return out;
}

bool parse_real_list(const std::string& v, std::vector<double>& out)
{
    out.clear();
    for (const std::string& t : bracket_tokens(v)) {
        char* end = nullptr;
        const double x = std::strtod(t.c_str(), &end);
        if (end == t.c_str() || *end != '\0' || !std::isfinite(x)) return false;
        out.push_back(x);
    }
    return !out.empty();
}

bool polymer_section_index(const std::string& sec, int& idx)
{
    const std::string pre = "polymer.";
    if (sec.size() <= pre.size() || sec.compare(0, pre.size(), pre) != 0) return false;
    const std::string t = sec.substr(pre.size());
    char* end = nullptr;
    const long v = std::strtol(t.c_str(), &end, 10);
    if (end == t.c_str() || *end != '\0' || v < 0 || v > std::numeric_limits<int>::max()) return false;
    idx = (int)v;
    return true;
}

std::string default_name(int i) { return i >= 0 && i < 26 ? std::string(1, (char)('A' + i)) : "T" + std::to_string(i); }

PolymerInput& polymer_input(Param& p, int idx)
{
    if ((int)p.polymer_species.size() <= idx) p.polymer_species.resize((size_t)idx + 1);
    p.polymer_species[(size_t)idx].section_seen = true;
    return p.polymer_species[(size_t)idx];
}

// One key of one section (the table of param.cu:205-334).
void apply(Param& p, const std::string& sec, const std::string& key, const std::string& v)
{
    bool ok = true;
    int pidx = -1;
    auto unknown = [&]() { fail("unknown parameter " + (sec.empty() ? key : "[" + sec + "] " + key)); };
    auto str = [&](std::string& out) { out = unquote(v); };
    if (sec == "grid") {
        if (key == "m1") ok = parse_int(v, p.m1);
        else if (key == "m2") ok = parse_int(v, p.m2);
        else if (key == "m3") ok = parse_int(v, p.m3);
        else if (key == "a") ok = parse_real(v, p.a);
        else if (key == "dL") ok = parse_real(v, p.dL);
        else unknown();
    } else if (sec == "monomers") {
        if (key == "M" || key == "m" || key == "count") ok = p.monomer_count_set = parse_int(v, p.monomer_type_count);
        else if (key == "names" || key == "types") {
            p.monomer_names = bracket_tokens(v);
            ok = p.monomer_names_set = !p.monomer_names.empty();
        } else unknown();
    } else if (sec == "polymer") {
        if (key == "species_count") ok = p.species_count_set = parse_int(v, p.species_count);
        else if (key == "sequence_file") str(p.sequence_file);
        else unknown();
    } else if (polymer_section_index(sec, pidx)) {
        PolymerInput& s = polymer_input(p, pidx);
        if (key == "name") { str(s.name); s.name_set = true; }
        else if (key == "num_chains") ok = s.num_chains_set = parse_int64(v, s.num_chains);
        else if (key == "N") ok = s.N_set = parse_int(v, s.N);
        else unknown();
    } else if (sec == "interactions") {
        if (key == "chi" || key == "chi_matrix") ok = p.chi_matrix_set = parse_real_list(v, p.chi_matrix);
        else if (key == "xi" || key == "v") ok = parse_real(v, p.xi);
        else if (key == "lB") ok = parse_real(v, p.lB);
        else if (key == "eigen_tol_rel" || key == "interaction_eigen_tol_rel") ok = parse_real(v, p.eigen_tol_rel);
        else unknown();
    } else if (sec == "dynamics") {
        if (key == "dt") ok = parse_real(v, p.dt);
        else if (key == "lambda_omega" || key == "lambda_w" || key == "lambda") ok = parse_real_list(v, p.lambda_omega_input);
        else if (key == "lambdaPsi") ok = parse_real(v, p.lambdaPsi);
        else if (key == "Nt") ok = parse_int(v, p.Nt);
        else if (key == "Nss") ok = parse_int(v, p.Nss);
        else if (key == "Ns") ok = parse_int(v, p.Ns);
        else if (key == "Ntmp" || key == "ntmp") ok = parse_int(v, p.Ntmp);
        else if (key == "Nso" || key == "nso") ok = parse_int(v, p.Nso);
        else if (key == "N_stat" || key == "n_stat" || key == "Nstat" || key == "nstat") ok = parse_int(v, p.N_stat);
        else if (key == "max_nan_restarts") ok = parse_int(v, p.max_nan_restarts);
        else if (key == "noise") ok = parse_bool(v, p.noise);
        else unknown();
    } else if (sec == "ions") {
        if (key == "enabled") ok = parse_bool(v, p.ions_enabled);
        else if (key == "default_smearing_length") ok = parse_real(v, p.default_smearing_length);
        else unknown();
    } else if (sec == "ions.counterions") {
        if (key == "enabled") ok = parse_bool(v, p.ci_enabled);
        else if (key == "number") {
            const std::string t = unquote(v);
            if (t == "auto_neutralize") p.ci_auto = true;
            else {
                ok = parse_int64(t, p.ci_number);
                p.ci_auto = false;
            }
        } else if (key == "valence") ok = parse_real(v, p.ci_valence);
        else if (key == "name") str(p.ci_name);
        else if (key == "smearing_length") ok = parse_real(v, p.ci_smearing);
        else unknown();
    } else if (sec == "ions.salt") {
        if (key == "enabled") ok = parse_bool(v, p.salt_enabled);
        else if (key == "num_salt") ok = parse_int64(v, p.num_salt);
        else if (key == "cation_name") str(p.cation_name);
        else if (key == "cation_valence") ok = parse_real(v, p.cation_valence);
        else if (key == "cation_stoich") ok = parse_int(v, p.cation_stoich);
        else if (key == "anion_name") str(p.anion_name);
        else if (key == "anion_valence") ok = parse_real(v, p.anion_valence);
        else if (key == "anion_stoich") ok = parse_int(v, p.anion_stoich);
        else if (key == "smearing_length") ok = parse_real(v, p.salt_smearing);
        else if (key == "combine_identical_species") ok = parse_bool(v, p.combine_identical);
        else unknown();
    } else if (sec == "structure_factor") {
        // accepted and ignored, as the reference does (param.cu:272-288)
        bool b;
        int i;
        double r;
        if (key == "enabled" || key == "desmear" || key == "particle_center" || key == "skip_zero") ok = parse_bool(v, b);
        else if (key == "file" || key == "output_file") ok = true;
        else if (key == "interval") ok = parse_int(v, i);
        else if (key == "kmax" || key == "shell_width" || key == "bin_width" || key == "dk" || key == "shell_tolerance" ||
                 key == "k_tolerance") ok = parse_real(v, r);
        else unknown();
    } else if (sec == "observables") {
        static const char* comps[6] = {"component_xx", "component_yy", "component_zz", "component_xy", "component_xz", "component_yz"};
        bool done = false;
        if (key == "stress") ok = parse_bool(v, p.stress), done = true;
        for (int c = 0; c < 6 && !done; ++c)
            if (key == comps[c]) ok = parse_bool(v, p.comp[c]), done = true;
        if (!done) {
            if (key == "isotropic_pressure" || key == "pressure" || key == "pressure_iso" || key == "p_iso" ||
                key == "pressure_trace" || key == "p_trace") ok = parse_bool(v, p.isotropic_pressure);
            else unknown();
        }
    } else if (sec == "output") {
        bool b;
        double r;
        if (key == "Nso" || key == "nso") ok = parse_int(v, p.Nso);
        else if (key == "N_stat" || key == "n_stat" || key == "Nstat" || key == "nstat") ok = parse_int(v, p.N_stat);
        else if (key == "omega_file" || key == "w_file") str(p.omega_file);
        else if (key == "psi_file") str(p.psi_file);
        else if (key == "tmp_omega_file" || key == "tmp_w_file") str(p.tmp_omega_file);
        else if (key == "tmp_psi_file") str(p.tmp_psi_file);
        else if (key == "rho_type_file") str(p.rho_type_file);
        else if (key == "rhop_file") str(p.rhop_file);
        else if (key == "rhoc_file") str(p.rhoc_file);
        else if (key == "rhoc_poly_file") str(p.rhoc_poly_file);
        else if (key == "rhoc_ion_file") str(p.rhoc_ion_file);
        else if (key == "ion_density_prefix") str(p.ion_density_prefix);
        else if (key == "step_omega_file" || key == "step_w_file") str(p.step_omega_file);
        else if (key == "step_psi_file") str(p.step_psi_file);
        else if (key == "step_rho_type_file") str(p.step_rho_type_file);
        else if (key == "step_rhop_file") str(p.step_rhop_file);
        else if (key == "step_rhoc_file") str(p.step_rhoc_file);
        else if (key == "step_rhoc_poly_file") str(p.step_rhoc_poly_file);
        else if (key == "step_rhoc_ion_file") str(p.step_rhoc_ion_file);
        else if (key == "step_ion_density_prefix") str(p.step_ion_density_prefix);
        else if (key == "observable_file") str(p.observable_file);
        else if (key == "drift_max_file") str(p.drift_max_file);
        else if (key == "order_param" || key == "order_param_file") ok = true;
        else if (key == "order_param_kc" || key == "order_kc") ok = parse_real(v, r);
        else if (key == "order_param_enabled" || key == "order_parameter_enabled") ok = parse_bool(v, b);
        else unknown();
    } else {
        unknown();
    }
    if (!ok) fail("cannot parse [" + sec + "] " + key);
}

void read_param(const std::string& file, Param& p)
{
    errno = 0;
    FILE* fp = std::fopen(file.c_str(), "r");
    if (!fp) fail(open_error(file));
    std::string sec;
    char line[4096];
    int lineno = 0;
    try {
        while (std::fgets(line, sizeof(line), fp)) {
            ++lineno;
            const std::string t = trim(strip_comment(line));
            if (t.empty()) continue;
            if (t.front() == '[' && t.back() == ']') {
                sec = trim(t.substr(1, t.size() - 2));
                continue;
            }
            const size_t eq = t.find('=');
            if (eq == std::string::npos) fail("bad line " + std::to_string(lineno) + " in " + file);
            const std::string key = trim(t.substr(0, eq));
            std::string value = trim(t.substr(eq + 1));
            int bal = bracket_delta(value);
            while (bal > 0 && std::fgets(line, sizeof(line), fp)) {
                ++lineno;
                const std::string extra = trim(strip_comment(line));
                if (!extra.empty()) {
                    value += " " + extra;
                    bal += bracket_delta(extra);
                }
            }
            if (bal != 0) fail(file + ": unbalanced brackets while reading [" + sec + "] " + key);
            apply(p, sec, key, value);
        }
    } catch (...) {
        std::fclose(fp);
        throw;
    }
    std::fclose(fp);
}

void recompute_polymer(Param& p)
{
    const int ns = std::max(0, p.species_count);
    if ((int)p.polymer_species.size() < ns) p.polymer_species.resize((size_t)ns);
    p.Nmax = 0;
    p.total_chains = p.total_segments = 0;
    p.total_type_segments.assign((size_t)std::max(0, p.monomer_type_count), 0);
    for (int i = 0; i < ns; ++i) {
        PolymerInput& s = p.polymer_species[(size_t)i];
        if ((int)s.type_counts.size() != std::max(0, p.monomer_type_count)) s.type_counts.assign((size_t)std::max(0, p.monomer_type_count), 0);
        p.Nmax = std::max(p.Nmax, s.N);
        p.total_chains += s.num_chains;
        p.total_segments += s.num_chains * (long long)s.N;
        for (int a = 0; a < p.monomer_type_count; ++a) p.total_type_segments[(size_t)a] += s.num_chains * (long long)s.type_counts[(size_t)a];
    }
    const double V = p.L1 * p.L2 * p.L3;
    if (V > 0.0 && p.total_segments > 0) p.rho0 = (double)p.total_segments / V;
}

// Cyclic Jacobi eigen-decomposition of a real symmetric matrix (textbook
// rotations); eigenvectors in the columns of `vec` (row-major n x n).
void jacobi(const std::vector<double>& in, int n, std::vector<double>& eig, std::vector<double>& vec)
{
    std::vector<double> a = in;
    vec.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) vec[(size_t)i * n + i] = 1.0;
    if (n == 1) {
        eig.assign(1, a[0]);
        return;
    }
    auto frob = [](const std::vector<double>& x) {
        long double s = 0.0L;
        for (double v : x) s += (long double)v * v;
        return std::sqrt((double)s);
    };
    auto offdiag = [&](const std::vector<double>& x) {
        long double s = 0.0L;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                if (i != j) s += (long double)x[(size_t)i * n + j] * x[(size_t)i * n + j];
        return std::sqrt((double)s);
    };
    const double scale = std::max(1.0, frob(in));
    const double tol = 1.0e-14 * scale;
    const int max_sweeps = std::max(50, 100 * n * n);
    bool converged = false;
    for (int sweep = 0; sweep < max_sweeps; ++sweep) {
        if (offdiag(a) <= tol) {
            converged = true;
            break;
        }
        bool rotated = false;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = a[(size_t)p * n + q];
                if (std::abs(apq) <= std::numeric_limits<double>::epsilon() * scale) continue;
                const double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q];
                const double tau = (aqq - app) / (2.0 * apq);
                const double t = tau >= 0.0 ? 1.0 / (tau + std::sqrt(1.0 + tau * tau)) : -1.0 / (-tau + std::sqrt(1.0 + tau * tau));
                const double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
                for (int k = 0; k < n; ++k) {
                    if (k == p || k == q) continue;
                    const double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
                    const double nkp = c * akp - s * akq, nkq = s * akp + c * akq;
                    a[(size_t)k * n + p] = a[(size_t)p * n + k] = nkp;
                    a[(size_t)k * n + q] = a[(size_t)q * n + k] = nkq;
                }
                a[(size_t)p * n + p] = c * c * app - 2.0 * s * c * apq + s * s * aqq;
                a[(size_t)q * n + q] = s * s * app + 2.0 * s * c * apq + c * c * aqq;
                a[(size_t)p * n + q] = a[(size_t)q * n + p] = 0.0;
                for (int k = 0; k < n; ++k) {
                    const double vkp = vec[(size_t)k * n + p], vkq = vec[(size_t)k * n + q];
                    vec[(size_t)k * n + p] = c * vkp - s * vkq;
                    vec[(size_t)k * n + q] = s * vkp + c * vkq;
                }
                rotated = true;
            }
        if (!rotated) {
            converged = true;
            break;
        }
    }
    if (!converged && offdiag(a) > 1.0e-10 * scale) fail("Jacobi diagonalization of interaction matrix did not converge");
    eig.resize((size_t)n);
    for (int i = 0; i < n; ++i) eig[(size_t)i] = a[(size_t)i * n + i];
}

void build_modes(Param& p, Modes& md)
{
    const int M = p.monomer_type_count;
    if (M <= 0) fail("invalid [monomers] M");
    if ((int)p.monomer_names.size() != M) fail("invalid [monomers] names length must equal M");
    for (int i = 0; i < M; ++i) {
        if (p.monomer_names[(size_t)i].empty()) fail("invalid empty monomer name");
        for (int j = i + 1; j < M; ++j)
            if (p.monomer_names[(size_t)i] == p.monomer_names[(size_t)j]) fail("invalid duplicate monomer name " + p.monomer_names[(size_t)i]);
    }
    if (!std::isfinite(p.xi) || p.xi < 0.0) fail("invalid xi");
    if (!std::isfinite(p.eigen_tol_rel) || p.eigen_tol_rel < 0.0) fail("invalid eigen_tol_rel");
    if ((int)p.chi_matrix.size() != M * M) fail("invalid [interactions] chi matrix size must be M*M");
    std::vector<double> chi = p.chi_matrix;
    double mx = 0.0;
    for (double x : chi) {
        if (!std::isfinite(x)) fail("invalid chi matrix entry");
        mx = std::max(mx, std::abs(x));
    }
    const double sym = 1.0e-12 * std::max(1.0, mx);
    for (int a = 0; a < M; ++a) {
        if (std::abs(chi[(size_t)a * M + a]) > sym) fail("invalid chi diagonal entries must be zero");
        chi[(size_t)a * M + a] = 0.0;
        for (int b = a + 1; b < M; ++b) {
            const double ab = chi[(size_t)a * M + b], ba = chi[(size_t)b * M + a];
            if (std::abs(ab - ba) > sym) fail("invalid chi matrix must be symmetric");
            chi[(size_t)a * M + b] = chi[(size_t)b * M + a] = 0.5 * (ab + ba);
        }
    }
    md.M = M;
    md.K.assign((size_t)M * M, 0.0);
    for (int a = 0; a < M; ++a)
        for (int b = 0; b < M; ++b) md.K[(size_t)a * M + b] = a == b ? p.xi : p.xi + chi[(size_t)a * M + b];
    std::vector<double> raw, vec;
    jacobi(md.K, M, raw, vec);
    std::vector<int> order((size_t)M);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int x, int y) {
        if (raw[(size_t)x] != raw[(size_t)y]) return raw[(size_t)x] > raw[(size_t)y];
        return x < y;
    });
    md.eig.assign((size_t)M, 0.0);
    md.O.assign((size_t)M * M, 0.0);
    for (int l = 0; l < M; ++l) {
        const int r = order[(size_t)l];
        md.eig[(size_t)l] = raw[(size_t)r];
        for (int a = 0; a < M; ++a) md.O[(size_t)l * M + a] = vec[(size_t)a * M + r];
        int piv = 0;
        double pa = std::abs(md.O[(size_t)l * M]);
        for (int a = 1; a < M; ++a)
            if (std::abs(md.O[(size_t)l * M + a]) > pa) pa = std::abs(md.O[(size_t)l * M + a]), piv = a;
        if (md.O[(size_t)l * M + piv] < 0.0)
            for (int a = 0; a < M; ++a) md.O[(size_t)l * M + a] *= -1.0;
    }
    double maxd = 0.0;
    for (double d : md.eig) maxd = std::max(maxd, std::abs(d));
    md.tol_abs = p.eigen_tol_rel * std::max(1.0, maxd);
    md.active.clear();
    for (int l = 0; l < M; ++l)
        if (std::abs(md.eig[(size_t)l]) > md.tol_abs) md.active.push_back(l);
    // reconstruction and orthogonality checks (interactionMode.cu:265-298)
    std::vector<double> res((size_t)M * M), orth((size_t)M * M);
    long double kn = 0.0L, rn = 0.0L, on = 0.0L;
    for (int a = 0; a < M; ++a)
        for (int b = 0; b < M; ++b) {
            double v = 0.0;
            for (int l = 0; l < M; ++l) v += md.O[(size_t)l * M + a] * md.eig[(size_t)l] * md.O[(size_t)l * M + b];
            const double r = md.K[(size_t)a * M + b] - v;
            rn += (long double)r * r;
            kn += (long double)md.K[(size_t)a * M + b] * md.K[(size_t)a * M + b];
        }
    for (int l = 0; l < M; ++l)
        for (int m = 0; m < M; ++m) {
            double dot = 0.0;
            for (int a = 0; a < M; ++a) dot += md.O[(size_t)l * M + a] * md.O[(size_t)m * M + a];
            const double o = dot - (l == m ? 1.0 : 0.0);
            on += (long double)o * o;
        }
    md.recon_err = std::sqrt((double)rn) / std::max(1.0, std::sqrt((double)kn));
    md.orth_err = std::sqrt((double)on);
    if (md.recon_err > 1.0e-10) fail("interaction eigenmode reconstruction check failed");
    if (md.orth_err > 1.0e-10) fail("interaction eigenvector orthogonality check failed");
}

// ---- sequence file (polymer.cu:219-273) ----
bool parse_charge(const std::string& t, size_t& i, double& q)
{
    const char c = t[i];
    if (c == '+' || c == '-') {
        const double sg = c == '+' ? 1.0 : -1.0;
        ++i;
        if (i >= t.size() || is_sep(t[i]) || t[i] == '+' || t[i] == '-') {
            q = sg;
            return true;
        }
        const char* b = t.c_str() + i;
        char* e = nullptr;
        const double mag = std::strtod(b, &e);
        if (e == b) return false;
        q = sg * mag;
        i = (size_t)(e - t.c_str());
        return true;
    }
    const char* b = t.c_str() + i;
    char* e = nullptr;
    q = std::strtod(b, &e);
    if (e == b) return false;
    i = (size_t)(e - t.c_str());
    return true;
}

std::vector<double> parse_reals(const std::string& t)
{
    std::vector<double> out;
    size_t i = 0;
    while (true) {
        while (i < t.size() && is_sep(t[i])) ++i;
        if (i >= t.size()) break;
        double q = 0.0;
        if (!parse_charge(t, i, q)) fail("cannot parse sequence real value");
        out.push_back(q);
    }
    return out;
}

void read_sequence(const std::string& file, Param& p, std::vector<Species>& out)
{
    errno = 0;
    FILE* fp = std::fopen(file.c_str(), "r");
    if (!fp) fail(open_error(file));
    struct Block {
        bool present = false;
        std::string monomers, charges, bonds;
    };
    std::vector<Block> blocks((size_t)std::max(1, p.species_count));
    int cur = -1;
    char line[4096];
    int lineno = 0;
    try {
        while (std::fgets(line, sizeof(line), fp)) {
            ++lineno;
            const std::string t = trim(strip_comment(line));
            if (t.empty()) continue;
            if (t.front() == '[' && t.back() == ']') {
                const std::string sec = trim(t.substr(1, t.size() - 2));
                int idx = -1;
                if (!polymer_section_index(sec, idx)) fail("unknown sequence section [" + sec + "]");
                if (idx < 0 || idx >= p.species_count) fail("invalid sequence polymer species index");
                cur = idx;
                blocks[(size_t)cur].present = true;
                continue;
            }
            if (cur < 0) fail("bad line " + std::to_string(lineno) + " in " + file);
            const size_t eq = t.find('=');
            if (eq == std::string::npos) fail("bad line " + std::to_string(lineno) + " in " + file);
            std::string key = trim(t.substr(0, eq));
            const std::string value = trim(t.substr(eq + 1));
            for (char& c : key) c = (char)std::tolower((unsigned char)c);
            if (key.empty()) fail("bad line " + std::to_string(lineno) + " in " + file);
            Block& b = blocks[(size_t)cur];
            std::string* dst = key == "monomers" ? &b.monomers : key == "charges" ? &b.charges : key == "bonds" ? &b.bonds : nullptr;
            if (!dst) fail("unknown sequence key " + key);
            if (!dst->empty()) *dst += ' ';
            *dst += value;
        }
    } catch (...) {
        std::fclose(fp);
        throw;
    }
    std::fclose(fp);
    out.assign((size_t)p.species_count, Species{});
    bool single_char = true;
    for (const std::string& n : p.monomer_names) single_char &= n.size() == 1;
    for (int k = 0; k < p.species_count; ++k) {
        const Block& b = blocks[(size_t)k];
        if (!b.present) fail("missing [polymer." + std::to_string(k) + "] sequence block");
        if (b.monomers.empty()) fail("missing monomers for polymer." + std::to_string(k));
        if (b.charges.empty()) fail("missing charges for polymer." + std::to_string(k));
        const PolymerInput& in = p.polymer_species[(size_t)k];
        // monomer labels
        std::string clean = b.monomers;
        for (char& c : clean)
            if (is_sep(c)) c = ' ';
        std::istringstream is(clean);
        std::vector<std::string> toks;
        std::string tk;
        while (is >> tk) toks.push_back(unquote(tk));
        if (toks.size() == 1 && toks[0].size() > 1 && single_char) {
            const std::string compact = toks[0];
            toks.clear();
            for (char c : compact) toks.push_back(std::string(1, c));
        }
        std::vector<int> types;
        for (const std::string& s : toks) {
            const auto it = std::find(p.monomer_names.begin(), p.monomer_names.end(), s);
            if (it == p.monomer_names.end()) fail("invalid unknown monomer label in sequence: " + s);
            types.push_back((int)(it - p.monomer_names.begin()));
        }
        if (types.empty()) fail("sequence has no monomer line");
        const std::vector<double> charges = parse_reals(b.charges);
        const std::vector<double> bonds = b.bonds.empty() ? std::vector<double>() : parse_reals(b.bonds);
        if (in.name.empty()) fail("polymer species name is required before reading sequence");
        if (in.num_chains <= 0) fail("num_chains must be positive for " + in.name);
        const int N = in.N;
        if (N <= 0) fail("N must be positive for " + in.name);
        if ((int)types.size() != N) fail("sequence length mismatch for " + in.name);
        if ((int)charges.size() != N) fail("charge sequence length mismatch for " + in.name);
        if (!bonds.empty() && (int)bonds.size() != std::max(0, N - 1)) fail("bond sequence length must be N-1 for " + in.name);
        Species& sp = out[(size_t)k];
        sp.name = in.name;
        sp.num_chains = in.num_chains;
        for (int s = 0; s < N; ++s) {
            const double bl = (s < N - 1 && !bonds.empty()) ? bonds[(size_t)s] : 1.0;
            if (bl <= 0.0) fail("invalid sequence bond length");
            sp.type.push_back(types[(size_t)s]);
            sp.charge.push_back(charges[(size_t)s]);
            sp.bond.push_back(bl);
        }
    }
    // update the counts the param file did not know (polymer.cu:275-292)
    for (int k = 0; k < p.species_count; ++k) {
        PolymerInput& in = p.polymer_species[(size_t)k];
        in.N = (int)out[(size_t)k].type.size();
        in.type_counts.assign((size_t)p.monomer_type_count, 0);
        for (int t : out[(size_t)k].type) ++in.type_counts[(size_t)t];
    }
    recompute_polymer(p);
}

std::string clean_name(std::string n)
{
    for (char& c : n)
        if (!std::isalnum((unsigned char)c) && c != '_' && c != '-') c = '_';
    return n.empty() ? "ion" : n;
}

void build_ions(const Param& p, double polymer_charge, std::vector<Ion>& out)
{
    out.clear();
    const bool elec = p.lB > 0.0;
    auto append = [&](const std::string& name, double z, long long n, double sm) {
        if (n == 0) return;
        if (p.combine_identical)
            for (Ion& s : out)
                if (std::fabs(s.valence - z) <= 1.0e-12 && std::fabs(s.smearing - sm) <= 1.0e-12) {
                    s.count += n;
                    return;
                }
        out.push_back(Ion{clean_name(name), z, n, sm});
    };
    if (p.ions_enabled && p.ci_enabled) {
        if (elec && p.ci_valence == 0.0) fail("invalid counterion valence");
        long long n = p.ci_number;
        if (p.ci_auto) {
            if (elec) {
                const double need = -polymer_charge / p.ci_valence;
                if (need < -1.0e-10) fail("invalid counterion sign");
                const double r = std::round(need);
                if (std::fabs(need - r) > 1.0e-8 * std::max(1.0, std::fabs(need))) fail("invalid counterion number");
                n = (long long)r;
            } else {
                n = 0;
            }
        }
        if (n < 0 || p.ci_smearing <= 0.0) fail("invalid counterion");
        append(p.ci_name, p.ci_valence, n, p.ci_smearing);
    }
    if (p.ions_enabled && p.salt_enabled) {
        if (p.num_salt < 0 || p.cation_stoich < 0 || p.anion_stoich < 0) fail("invalid salt counts");
        if (p.salt_smearing <= 0.0) fail("invalid salt");
        if (elec) {
            if (p.cation_valence == 0.0 || p.anion_valence == 0.0) fail("invalid salt");
            if (std::fabs(p.cation_stoich * p.cation_valence + p.anion_stoich * p.anion_valence) > 1.0e-10) fail("salt is not neutral");
        }
        append(p.cation_name, p.cation_valence, p.num_salt * (long long)p.cation_stoich, p.salt_smearing);
        append(p.anion_name, p.anion_valence, p.num_salt * (long long)p.anion_stoich, p.salt_smearing);
    }
    double total = polymer_charge, scale = std::fabs(polymer_charge);
    for (const Ion& s : out) {
        if (s.count < 0 || (elec && s.valence == 0.0) || s.smearing <= 0.0) fail("invalid ion species");
        total += s.valence * (double)s.count;
        scale += std::fabs(s.valence * (double)s.count);
    }
    if (elec && std::fabs(total) > 1.0e-8 * std::max(1.0, scale)) fail("electroneutrality failed");
}

bool valid_template(const std::string& t)
{
    const size_t f = t.find("%d");
    if (f == std::string::npos || t.find("%d", f + 2) != std::string::npos) return false;
    const size_t slash = t.find_last_of("/\\");
    return slash == std::string::npos || f > slash;
}

void validate(const Model& m)
{
    const Param& p = m.p;
    std::string e;
    auto bad = [&](const std::string& s) {
        if (e.empty()) e = s;
    };
    if (!p.species_count_set) bad("invalid [polymer] species_count is required");
    if (p.species_count <= 0) bad("invalid polymer species_count");
    if (p.sequence_file.empty()) bad("invalid [polymer] sequence_file is required");
    if ((int)p.polymer_species.size() > std::max(0, p.species_count)) bad("invalid polymer species section index exceeds species_count");
    for (int i = 0; i < p.species_count && i < (int)p.polymer_species.size(); ++i) {
        const PolymerInput& s = p.polymer_species[(size_t)i];
        const std::string pre = "[polymer." + std::to_string(i) + "]";
        if (!s.section_seen) bad("invalid " + pre + " section is required");
        if (!s.name_set) bad("invalid " + pre + " name is required");
        if (!s.N_set) bad("invalid " + pre + " N is required");
        if (!s.num_chains_set) bad("invalid " + pre + " num_chains is required");
        if (s.N <= 0) bad("invalid " + pre + " N");
        if (s.num_chains <= 0) bad("invalid " + pre + " num_chains");
    }
    if (p.m1 <= 0 || p.m2 <= 0 || p.m3 <= 0) bad("invalid mesh");
    const long long ms = (long long)p.m1 * p.m2 * p.m3;
    if (ms <= 0 || ms > 2147483647LL) bad("invalid mesh size");
    if (p.a <= 0.0 || p.dL <= 0.0 || p.lB < 0.0) bad("invalid a, dL, or lB");
    if (p.dt < 0.0 || p.lambdaPsi < 0.0) bad("invalid dt or lambdaPsi");
    if (p.Nss < 0 || p.Ns < 0 || p.Ntmp < 0 || p.Nso < -1 || p.N_stat < -1) bad("invalid sampling/checkpoint/step-output/drift-stat intervals");
    if (p.N_stat >= 0 && p.drift_max_file.empty()) bad("invalid drift_max_file");
    const bool any = p.comp[0] || p.comp[1] || p.comp[2] || p.comp[3] || p.comp[4] || p.comp[5];
    if (p.stress && !(any || p.isotropic_pressure)) bad("invalid stress observable requires at least one component_* = true or isotropic_pressure = true");
    if (!p.stress && (any || p.isotropic_pressure)) bad("invalid stress components or isotropic_pressure require [observables] stress = true");
    for (const std::string* t : {&p.step_omega_file, &p.step_psi_file, &p.step_rho_type_file, &p.step_rhop_file, &p.step_rhoc_file,
                                 &p.step_rhoc_poly_file, &p.step_rhoc_ion_file, &p.step_ion_density_prefix})
        if (!t->empty() && !valid_template(*t)) bad("invalid step output template (use exactly one %d in the file name)");
    if (p.max_nan_restarts < 0) bad("invalid max_nan_restarts");
    if (p.rho0 <= 0.0) bad("invalid rho0");
    if (p.xi < 0.0) bad("invalid xi");
    if (p.default_smearing_length <= 0.0) bad("invalid default_smearing_length");
    if (p.ci_smearing <= 0.0) bad("invalid counterion smearing_length");
    if (p.salt_smearing <= 0.0) bad("invalid salt smearing_length");
    if ((int)p.lambda_omega.size() != m.n_modes()) bad("invalid lambda_omega count");
    if (!e.empty()) fail(e);
}

}  // namespace

std::string trim(const std::string& s)
{
    size_t f = 0, l = s.size();
    while (f < l && std::isspace((unsigned char)s[f])) ++f;
    while (l > f && std::isspace((unsigned char)s[l - 1])) --l;
    return s.substr(f, l - f);
}

std::string strip_comment(const std::string& s)
{
    bool q = false;
    char qc = 0;
    for (size_t i = 0; i < s.size(); ++i) {
        const char c = s[i];
        if ((c == '"' || c == '\'') && (i == 0 || s[i - 1] != '\\')) {
            if (!q) { q = true; qc = c; }
            else if (qc == c) q = false;
        }
        if (c == '#' && !q) return s.substr(0, i);
    }
    return s;
}

std::string unquote(std::string v)
{
    v = trim(v);
    if (v.size() >= 2 && ((v.front() == '"' && v.back() == '"') || (v.front() == '\'' && v.back() == '\'')))
        v = v.substr(1, v.size() - 2);
    return v;
}

bool load_model(const std::string& param_file, const std::string& sequence_override, Model& m, std::string& err)
{
    try {
        m = Model{};
        Param& p = m.p;
        read_param(param_file, p);
        if (!sequence_override.empty()) p.sequence_file = sequence_override;
        // derive (param.cu:342-359)
        if (p.species_count > 0 && (int)p.polymer_species.size() < p.species_count) p.polymer_species.resize((size_t)p.species_count);
        p.L1 = p.dL * p.m1;
        p.L2 = p.dL * p.m2;
        p.L3 = p.dL * p.m3;
        p.dV = p.dL * p.dL * p.dL;
        if (p.Ns <= 0) p.Ns = p.Nt;
        if (p.default_smearing_length == -1.0) p.default_smearing_length = p.a;
        if (p.ci_smearing == -1.0) p.ci_smearing = p.default_smearing_length;
        if (p.salt_smearing == -1.0) p.salt_smearing = p.default_smearing_length;
        recompute_polymer(p);
        // interactions (param.cu:361-385)
        if (!p.monomer_count_set && p.monomer_names_set) p.monomer_type_count = (int)p.monomer_names.size();
        else if (!p.monomer_count_set && !p.monomer_names_set && p.chi_matrix_set) {
            const int r = (int)(std::sqrt((double)p.chi_matrix.size()) + 0.5);
            if (r > 0 && (size_t)r * r == p.chi_matrix.size()) p.monomer_type_count = r;
        } else if (!p.monomer_count_set && !p.monomer_names_set) p.monomer_type_count = 2;
        if (p.monomer_type_count <= 0) fail("invalid [monomers] M");
        if (p.monomer_names_set) {
            if ((int)p.monomer_names.size() != p.monomer_type_count) fail("invalid [monomers] names length must equal M");
        } else {
            p.monomer_names.clear();
            for (int i = 0; i < p.monomer_type_count; ++i) p.monomer_names.push_back(default_name(i));
        }
        const size_t mm = (size_t)p.monomer_type_count * p.monomer_type_count;
        if (!p.chi_matrix_set) p.chi_matrix.assign(mm, 0.0);
        build_modes(p, m.modes);
        // mobilities (param.cu:387-410)
        const int n = m.n_modes();
        p.lambda_omega.clear();
        if (n > 0) {
            if (p.lambda_omega_input.empty()) p.lambda_omega.assign((size_t)n, 0.0);
            else if (p.lambda_omega_input.size() == 1) p.lambda_omega.assign((size_t)n, p.lambda_omega_input[0]);
            else if ((int)p.lambda_omega_input.size() == n) p.lambda_omega = p.lambda_omega_input;
            else fail("invalid lambda_omega length must be 1 or the number of active interaction modes");
            for (double x : p.lambda_omega)
                if (!std::isfinite(x) || x < 0.0) fail("invalid lambda_omega");
        }
        recompute_polymer(p);
        // sequence (polymer.cu:185-194), then validation and ions
        if (p.sequence_file.empty()) fail("[polymer] sequence_file is required");
        read_sequence(p.sequence_file, p, m.species);
        validate(m);
        double qpoly = 0.0;
        for (const Species& s : m.species) {
            double q = 0.0;
            for (double z : s.charge) q += z;
            qpoly += (double)s.num_chains * q;
        }
        build_ions(p, qpoly, m.ions);
        // short-range self pressure (param.cu:130-147)
        m.self_pressure = 0.0;
        if (p.a > 0.0 && p.total_segments > 0) {
            const int M = p.monomer_type_count;
            long double wd = 0.0L;
            for (int a = 0; a < M && a < (int)p.total_type_segments.size(); ++a)
                wd += (long double)p.total_type_segments[(size_t)a] * (long double)m.modes.K[(size_t)a * M + a];
            const long double mean = wd / (long double)p.total_segments;
            const long double den = 16.0L * (long double)PI_ * std::sqrt((long double)PI_) * (long double)p.a * p.a * p.a;
            m.self_pressure = (double)(mean / den);
        }
        return true;
    } catch (const Fail& f) {
        err = f.msg;
        return false;
    }
}

void fill_config(Model& m, ftsp_config& c)
{
    const Param& p = m.p;
    std::memset(&c, 0, sizeof(c));
    c.max_restarts = p.max_nan_restarts;
    c.m1 = p.m1;
    c.m2 = p.m2;
    c.m3 = p.m3;
    c.L1 = p.L1;
    c.L2 = p.L2;
    c.L3 = p.L3;
    c.dV = p.dV;
    c.a = p.a;
    c.lB = p.lB;
    c.dt = p.dt;
    c.lambda_psi = p.lambdaPsi;
    c.M = p.monomer_type_count;
    const int nm = m.n_modes();
    c.n_modes = nm;
    m.c_coeff.clear(); m.c_gamma.clear(); m.c_O.clear(); m.c_lambda.clear();
    for (int a = 0; a < nm; ++a) {
        const double d = m.mode_eig(a);
        m.c_coeff.push_back(p.rho0 / std::abs(d));
        m.c_gamma.push_back(d > 0.0 ? 0.0 : 1.0);
        m.c_gamma.push_back(d > 0.0 ? 1.0 : 0.0);
        for (int al = 0; al < c.M; ++al) m.c_O.push_back(m.modes.O[(size_t)m.modes.active[a] * c.M + al]);
        m.c_lambda.push_back(p.lambda_omega[(size_t)a]);
    }
    m.c_chains.clear(); m.c_N.clear(); m.c_type.clear(); m.c_charge.clear(); m.c_bond.clear();
    for (const Species& s : m.species) {
        m.c_chains.push_back((double)s.num_chains);
        m.c_N.push_back((int)s.type.size());
        m.c_type.insert(m.c_type.end(), s.type.begin(), s.type.end());
        m.c_charge.insert(m.c_charge.end(), s.charge.begin(), s.charge.end());
        m.c_bond.insert(m.c_bond.end(), s.bond.begin(), s.bond.end());
    }
    m.c_ival.clear(); m.c_icount.clear(); m.c_ismear.clear();
    for (const Ion& i : m.ions) {
        m.c_ival.push_back(i.valence);
        m.c_icount.push_back((double)i.count);
        m.c_ismear.push_back(i.smearing);
    }
    auto ptr = [](std::vector<double>& v) -> const double* { return v.empty() ? nullptr : v.data(); };
    c.mode_coeff = ptr(m.c_coeff);
    c.mode_gamma = ptr(m.c_gamma);
    c.mode_O = ptr(m.c_O);
    c.mode_lambda = ptr(m.c_lambda);
    c.n_species = (int)m.species.size();
    c.num_chains = ptr(m.c_chains);
    c.N = m.c_N.data();
    c.seg_type = m.c_type.data();
    c.seg_charge = ptr(m.c_charge);
    c.seg_bond = ptr(m.c_bond);
    c.n_ions = (int)m.ions.size();
    c.ion_valence = ptr(m.c_ival);
    c.ion_count = ptr(m.c_icount);
    c.ion_smear = ptr(m.c_ismear);
    c.self_pressure = m.self_pressure;
    int mask = 0;
    if (p.stress)
        for (int k = 0; k < 6; ++k)
            if (p.comp[k]) mask |= 1 << k;
    c.stress_mask = mask;
    c.isotropic_pressure = p.stress && p.isotropic_pressure ? 1 : 0;
    c.noise = p.noise ? 1 : 0;
}

}  // namespace host
}  // namespace ftsp
