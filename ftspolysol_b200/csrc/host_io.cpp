// Field files and run-directory layout (see host_io.h for the reference
// routines each function follows).
#include "host_io.h"

#include <sys/stat.h>
#include <sys/types.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace ftsp {
namespace host {

namespace {

size_t grid(int a, int b, int c) { return (size_t)a * (size_t)b * (size_t)c; }

std::string open_error(const std::string& path)
{
    std::string t = "cannot open " + path;
    if (errno) t += ": " + std::string(std::strerror(errno));
    return t;
}

// Strips a '#' comment and leading blanks; false for an empty line
// (common.h:229-236).
bool content(char* line, char*& ptr)
{
    if (char* h = std::strchr(line, '#')) *h = '\0';
    ptr = line;
    while (std::isspace((unsigned char)*ptr)) ++ptr;
    return *ptr != '\0';
}

bool mesh_header(const char* s, int& a, int& b, int& c)
{
    char extra = 0;
    return std::sscanf(s, "%d %d %d %c", &a, &b, &c, &extra) == 3 && a > 0 && b > 0 && c > 0;
}

bool box_header(const char* s)
{
    double a = 0, b = 0, c = 0;
    char extra = 0;
    return std::sscanf(s, "%lf %lf %lf %c", &a, &b, &c, &extra) == 3 && a > 0.0 && b > 0.0 && c > 0.0;
}

bool path_is_dir(const std::string& p)
{
    struct stat st;
    return stat(p.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

bool make_directory(const std::string& p, std::string& err)
{
    if (p.empty()) return false;
    if (path_is_dir(p)) return true;
    if (mkdir(p.c_str(), 0775) == 0) return true;
    if (errno == EEXIST && path_is_dir(p)) return true;
    err = "cannot create " + p;
    return false;
}

bool copy_file(const std::string& src, const std::string& dst, std::string& err)
{
    errno = 0;
    FILE* in = std::fopen(src.c_str(), "rb");
    if (!in) return err = open_error(src), false;
    std::vector<char> data;
    char buf[65536];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), in)) > 0) data.insert(data.end(), buf, buf + got);
    const bool rd_err = std::ferror(in) != 0;
    std::fclose(in);
    if (rd_err) return err = "cannot read " + src, false;
    errno = 0;
    FILE* out = std::fopen(dst.c_str(), "wb");
    if (!out) return err = open_error(dst), false;
    if (!data.empty() && std::fwrite(data.data(), 1, data.size(), out) != data.size()) {
        std::fclose(out);
        return err = "cannot write " + dst, false;
    }
    if (std::fclose(out) != 0) return err = "cannot close " + dst, false;
    return true;
}

std::string directory_path(const std::string& path)
{
    const size_t pos = path.find_last_of("/\\");
    if (pos == std::string::npos) return std::string();
    return pos == 0 ? path.substr(0, 1) : path.substr(0, pos);
}

// Folder named after a template's stem: "snap_%d.rf" -> "snap"
// (fieldIO.cu:162-174).
std::string template_folder(const std::string& pattern)
{
    const std::string base = basename_path(pattern);
    const size_t pos = base.find("%d");
    std::string name = pos == std::string::npos ? base : base.substr(0, pos);
    while (!name.empty() && (name.back() == '_' || name.back() == '-' || name.back() == '.')) name.pop_back();
    return name.empty() ? "step_fields" : name;
}

bool prepare_template(std::string& pattern, std::string& err)
{
    if (pattern.empty() || !valid_step_template(pattern)) return true;
    const std::string base = basename_path(pattern), parent = directory_path(pattern);
    const std::string folder = template_folder(base);
    const std::string full = (!parent.empty() && basename_path(parent) == folder) ? parent : join_path(parent, folder);
    if (!make_directories(full, err)) return false;
    pattern = join_path(full, base);
    return true;
}

std::string run_output(const std::string& run, const std::string& name)
{
    return run.empty() ? name : join_path(run, basename_path(name));
}

bool valid_run_id(const std::string& id)
{
    if (id.empty() || id == "." || id == "..") return false;
    for (char c : id)
        if (c == '/' || c == '\\') return false;
    return true;
}

// Index of the first active mode with a positive (density-like) or negative
// (composition-like) eigenvalue (fieldIO.cu:368-376).
int active_by_sign(const Model& m, bool positive)
{
    for (int a = 0; a < m.n_modes(); ++a) {
        const double d = m.mode_eig(a);
        if (positive ? d > 0.0 : d < 0.0) return a;
    }
    return -1;
}

bool legacy_to_active(const Model& m, const FieldTable& t, std::vector<double>& omega, std::string& err)
{
    const int nf = m.n_modes();
    const size_t V = (size_t)m.size();
    omega.assign((size_t)std::max(0, nf) * V * 2, 0.0);
    if (nf <= 0) return true;
    if (t.field_count != 1 && t.field_count != 2) {
        err = "legacy A/B omega file must contain either one complex field or two complex fields";
        return false;
    }
    if (t.rows() != V) {
        err = "legacy A/B omega field: rows " + std::to_string(t.rows()) + ", expected " + std::to_string(V);
        return false;
    }
    const int comp = active_by_sign(m, false), dens = active_by_sign(m, true);
    if (comp >= 0) std::copy(t.fields.begin(), t.fields.begin() + 2 * V, omega.begin() + (ptrdiff_t)(2 * V * comp));
    if (t.field_count == 2 && dens >= 0)
        std::copy(t.fields.begin() + 2 * V, t.fields.begin() + 4 * V, omega.begin() + (ptrdiff_t)(2 * V * dens));
    return true;
}

bool resize_table(const FieldTable& in, int m1, int m2, int m3, FieldTable& out, std::string& err)
{
    const size_t src = grid(in.m1, in.m2, in.m3);
    if (in.rows() != src) {
        err = "omega field resize source: rows " + std::to_string(in.rows()) + ", expected " + std::to_string(src);
        return false;
    }
    out = FieldTable{};
    out.m1 = m1; out.m2 = m2; out.m3 = m3;
    out.header = true;
    out.field_count = in.field_count;
    const size_t dst = grid(m1, m2, m3);
    out.fields.assign((size_t)in.field_count * dst * 2, 0.0);
    std::vector<double> r;
    for (int f = 0; f < in.field_count; ++f) {
        trilinear_resize(in.fields.data() + (size_t)f * src * 2, in.m1, in.m2, in.m3, r, m1, m2, m3);
        std::copy(r.begin(), r.end(), out.fields.begin() + (ptrdiff_t)((size_t)f * dst * 2));
    }
    return true;
}

}  // namespace

bool read_field_table(const std::string& file, int m1, int m2, int m3, FieldTable& t, std::string& err)
{
    errno = 0;
    FILE* fp = std::fopen(file.c_str(), "r");
    if (!fp) return err = open_error(file), false;
    t = FieldTable{};
    t.m1 = m1; t.m2 = m2; t.m3 = m3;
    bool first = true, maybe_box = false;
    std::vector<std::vector<double>> rows;
    std::vector<char> line(1 << 16);
    size_t lineno = 0;
    while (std::fgets(line.data(), (int)line.size(), fp)) {
        ++lineno;
        char* ptr = nullptr;
        if (!content(line.data(), ptr)) continue;
        if (first) {
            first = false;
            int a, b, c;
            if (mesh_header(ptr, a, b, c)) {
                t.m1 = a; t.m2 = b; t.m3 = c;
                t.header = true;
                maybe_box = true;
                continue;
            }
        }
        if (maybe_box) {
            maybe_box = false;
            if (box_header(ptr)) continue;
        }
        std::vector<double> v;
        char* s = ptr;
        while (*s) {
            while (std::isspace((unsigned char)*s)) ++s;
            if (!*s) break;
            char* e = nullptr;
            const double x = std::strtod(s, &e);
            if (e == s) {
                std::fclose(fp);
                err = "bad line " + std::to_string(lineno) + " in " + file;
                return false;
            }
            v.push_back(x);
            s = e;
        }
        if (v.empty() || v.size() % 2) {
            std::fclose(fp);
            err = file + ": expected an even number of numeric columns per row";
            return false;
        }
        const int nf = (int)(v.size() / 2);
        if (t.field_count == 0) t.field_count = nf;
        if (nf != t.field_count) {
            std::fclose(fp);
            err = file + ": inconsistent number of field columns";
            return false;
        }
        rows.push_back(std::move(v));
    }
    std::fclose(fp);
    const size_t R = rows.size();
    t.fields.assign((size_t)t.field_count * R * 2, 0.0);
    for (size_t i = 0; i < R; ++i)
        for (int f = 0; f < t.field_count; ++f) {
            t.fields[((size_t)f * R + i) * 2] = rows[i][(size_t)2 * f];
            t.fields[((size_t)f * R + i) * 2 + 1] = rows[i][(size_t)2 * f + 1];
        }
    return true;
}

bool write_fields(const std::string& file, const Param& p, const double* fields, int count, size_t size, std::string& err)
{
    errno = 0;
    FILE* fp = std::fopen(file.c_str(), "w");
    if (!fp) return err = open_error(file), false;
    bool ok = std::fprintf(fp, "%d %d %d\n", p.m1, p.m2, p.m3) > 0 && std::fprintf(fp, "%.17g %.17g %.17g\n", p.L1, p.L2, p.L3) > 0;
    if (!ok) {
        std::fclose(fp);
        err = "cannot write mesh header to " + file;
        return false;
    }
    // One formatted row per point; buffered through a string to keep the
    // 128^3 outputs fast.
    std::string buf;
    buf.reserve(1 << 20);
    char cell[96];
    for (size_t i = 0; i < size && ok; ++i) {
        for (int f = 0; f < count; ++f) {
            const double* z = fields + ((size_t)f * size + i) * 2;
            const int n = std::snprintf(cell, sizeof(cell), "%s%.10f  %.10f", f == 0 ? "" : "  ", z[0], z[1]);
            buf.append(cell, (size_t)n);
        }
        buf.push_back('\n');
        if (buf.size() > (1u << 20) - 256) {
            ok = std::fwrite(buf.data(), 1, buf.size(), fp) == buf.size();
            buf.clear();
        }
    }
    if (ok && !buf.empty()) ok = std::fwrite(buf.data(), 1, buf.size(), fp) == buf.size();
    if (!ok) {
        std::fclose(fp);
        err = "cannot write " + file;
        return false;
    }
    if (std::fclose(fp) != 0) return err = "cannot close " + file, false;
    return true;
}

bool infer_mesh(size_t rows, const Param& p, int& m1, int& m2, int& m3)
{
    const size_t target = grid(p.m1, p.m2, p.m3);
    if (rows == target) {
        m1 = p.m1; m2 = p.m2; m3 = p.m3;
        return true;
    }
    if (rows == 0) return false;
    const double ratio = target > rows ? (double)target / rows : (double)rows / target;
    const int sc = (int)std::llround(std::cbrt(ratio));
    if (sc > 1 && std::fabs((double)sc * sc * sc - ratio) < 1.0e-8) {
        if (target > rows) {
            if (p.m1 % sc == 0 && p.m2 % sc == 0 && p.m3 % sc == 0 && grid(p.m1 / sc, p.m2 / sc, p.m3 / sc) == rows) {
                m1 = p.m1 / sc; m2 = p.m2 / sc; m3 = p.m3 / sc;
                return true;
            }
        } else if (grid(p.m1 * sc, p.m2 * sc, p.m3 * sc) == rows) {
            m1 = p.m1 * sc; m2 = p.m2 * sc; m3 = p.m3 * sc;
            return true;
        }
    }
    const int cube = (int)std::llround(std::cbrt((double)rows));
    if (cube > 0 && grid(cube, cube, cube) == rows) {
        m1 = m2 = m3 = cube;
        return true;
    }
    return false;
}

void trilinear_resize(const double* in, int n1, int n2, int n3, std::vector<double>& out, int m1, int m2, int m3)
{
    const size_t dst = grid(m1, m2, m3);
    if (n1 == m1 && n2 == m2 && n3 == m3) {
        out.assign(in, in + 2 * dst);
        return;
    }
    out.assign(2 * dst, 0.0);
    auto wrap = [](int i, int n) { return (i % n + n) % n; };
    auto at = [&](int x, int y, int z, int c) {
        return in[(((size_t)wrap(x, n1) * n2 + wrap(y, n2)) * n3 + wrap(z, n3)) * 2 + c];
    };
    // interpolation weights along one axis: source cell i0 and fraction t
    auto axis = [](int i, int n, int m, int& i0, int& i1, double& t) {
        const double s = (double)i * n / m;
        i0 = (int)std::floor(s);
        i1 = n == 1 ? 0 : i0 + 1;
        t = n == 1 ? 0.0 : s - i0;
    };
    auto lerp = [](double a, double b, double t) { return a + t * (b - a); };
    for (int x = 0; x < m1; ++x) {
        int x0, x1;
        double tx;
        axis(x, n1, m1, x0, x1, tx);
        for (int y = 0; y < m2; ++y) {
            int y0, y1;
            double ty;
            axis(y, n2, m2, y0, y1, ty);
            for (int z = 0; z < m3; ++z) {
                int z0, z1;
                double tz;
                axis(z, n3, m3, z0, z1, tz);
                for (int c = 0; c < 2; ++c) {
                    // innermost along z, then y, then x: the reference's order
                    const double c00 = lerp(at(x0, y0, z0, c), at(x0, y0, z1, c), tz);
                    const double c01 = lerp(at(x0, y1, z0, c), at(x0, y1, z1, c), tz);
                    const double c10 = lerp(at(x1, y0, z0, c), at(x1, y0, z1, c), tz);
                    const double c11 = lerp(at(x1, y1, z0, c), at(x1, y1, z1, c), tz);
                    out[(((size_t)x * m2 + y) * m3 + z) * 2 + c] = lerp(lerp(c00, c01, ty), lerp(c10, c11, ty), tx);
                }
            }
        }
    }
}

bool valid_step_template(const std::string& pattern)
{
    const size_t f = pattern.find("%d");
    if (f == std::string::npos || pattern.find("%d", f + 2) != std::string::npos) return false;
    const size_t slash = pattern.find_last_of("/\\");
    return slash == std::string::npos || f > slash;
}

std::string step_filename(const std::string& pattern, int step)
{
    const size_t pos = pattern.find("%d");
    if (pos == std::string::npos) return pattern;
    return pattern.substr(0, pos) + std::to_string(step) + pattern.substr(pos + 2);
}

std::string join_path(const std::string& a, const std::string& b)
{
    if (a.empty() || a == ".") return b;
    return a.back() == '/' ? a + b : a + "/" + b;
}

std::string basename_path(const std::string& path)
{
    const size_t pos = path.find_last_of("/\\");
    return pos == std::string::npos ? path : path.substr(pos + 1);
}

bool make_directories(const std::string& path, std::string& err)
{
    if (path.empty()) return false;
    std::string cur;
    size_t i = 0;
    if (path[0] == '/') {
        cur = "/";
        i = 1;
    }
    while (i <= path.size()) {
        const size_t next = path.find('/', i);
        const std::string part = path.substr(i, next == std::string::npos ? std::string::npos : next - i);
        if (!part.empty() && part != ".") {
            if (!cur.empty() && cur.back() != '/') cur += '/';
            cur += part;
            if (!make_directory(cur, err)) return false;
        }
        if (next == std::string::npos) break;
        i = next + 1;
    }
    return path_is_dir(path) || make_directory(path, err);
}

void usage(const char* program)
{
    std::fprintf(stderr,
                 "usage: %s [-p param] [-i id] [-s dir] [--omega omega_file] [--psi psi_file] [--seq sequence_file] "
                 "[--screenprint] [--fp32|--fp64] [--si|--pc] [--seed N] [--device N] [--autotune] [--adaptive U]\n",
                 program);
}

int parse_args(int argc, char** argv, Options& o, std::string& err)
{
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto value = [&](const char* name, std::string& out) {
            if (++i == argc) {
                err = std::string("missing value for ") + name;
                return false;
            }
            out = argv[i];
            return true;
        };
        std::string v;
        if (a == "-p") {
            if (!value("-p", o.param_file)) return -1;
        } else if (a == "--omega") {
            if (!value("--omega", o.omega_file)) return -1;
            o.omega_override = true;
        } else if (a == "-psi" || a == "--psi") {
            if (!value("--psi", o.psi_file)) return -1;
            o.psi_override = true;
        } else if (a == "-i" || a == "--id") {
            if (!value("-i", o.run_id)) return -1;
            o.run_id_set = true;
        } else if (a == "-s" || a == "--dir" || a == "--run-dir") {
            if (!value("-s", o.run_parent)) return -1;
            o.run_parent_set = true;
        } else if (a == "--seq") {
            if (!value("--seq", o.sequence_file)) return -1;
            o.sequence_override = true;
        } else if (a == "-c" || a == "--charge" || a == "--charges" || a == "--sigma") {
            err = "charge files are not used; use --seq";
            return -1;
        } else if (a == "--screenprint") {
            o.screenprint = true;
        } else if (a == "-h" || a == "--help") {
            return 1;
        } else if (a == "--fp32") {
            o.precision = FTSP_FP32;
        } else if (a == "--fp64") {
            o.precision = FTSP_FP64;
        } else if (a == "--autotune") {
            o.autotune = 1;
        } else if (a == "--adaptive") {
            if (!value("--adaptive", v)) return -1;
            char* e = nullptr;
            o.adaptive = std::strtod(v.c_str(), &e);
            if (e == v.c_str() || *e || !(o.adaptive >= 0.0)) {
                err = "cannot parse --adaptive " + v;
                return -1;
            }
        } else if (a == "--si") {
            o.scheme = FTSP_SCHEME_SI;
        } else if (a == "--pc") {
            o.scheme = FTSP_SCHEME_PC;
        } else if (a == "--seed" || a == "--device") {
            if (!value(a.c_str(), v)) return -1;
            char* e = nullptr;
            const unsigned long long x = std::strtoull(v.c_str(), &e, 10);
            if (e == v.c_str() || *e) {
                err = "cannot parse " + a + " " + v;
                return -1;
            }
            if (a == "--seed") o.seed = x, o.seed_set = true;
            else o.device = (int)x;
        } else {
            err = "unknown option " + a;
            return -1;
        }
    }
    return 0;
}

bool prepare_run(const Options& o, Param& p, RunPaths& r, std::string& err)
{
    if (!o.run_id_set) {
        if (o.run_parent_set) return err = "-s requires -i", false;
        r.run.clear();
    } else {
        if (!valid_run_id(o.run_id)) return err = "invalid run id " + o.run_id, false;
        r.run = join_path(o.run_parent, o.run_id);
        if (!make_directories(r.run, err)) return false;
        if (!copy_file(o.param_file, join_path(r.run, o.run_id + ".param"), err)) return false;
        if (!p.sequence_file.empty() && !copy_file(p.sequence_file, join_path(r.run, o.run_id + ".sequence"), err)) return false;
    }
    r.input_omega = o.omega_override ? o.omega_file : p.omega_file;
    r.input_psi = o.psi_override ? o.psi_file : p.psi_file;
    r.zero_missing_default_omega = !o.omega_override && r.input_omega == "omega.rf";
    r.source_mesh_known = false;
    for (std::string* f : {&p.omega_file, &p.psi_file, &p.tmp_omega_file, &p.tmp_psi_file, &p.rho_type_file, &p.rhop_file,
                           &p.rhoc_file, &p.rhoc_poly_file, &p.rhoc_ion_file, &p.ion_density_prefix})
        *f = run_output(r.run, *f);
    for (std::string* f : {&p.step_omega_file, &p.step_psi_file, &p.step_rho_type_file, &p.step_rhop_file, &p.step_rhoc_file,
                           &p.step_rhoc_poly_file, &p.step_rhoc_ion_file, &p.step_ion_density_prefix})
        if (!f->empty()) *f = run_output(r.run, *f);
    if (p.Nso >= 0)
        for (std::string* f : {&p.step_omega_file, &p.step_psi_file, &p.step_rho_type_file, &p.step_rhop_file, &p.step_rhoc_file,
                               &p.step_rhoc_poly_file, &p.step_rhoc_ion_file, &p.step_ion_density_prefix})
            if (!prepare_template(*f, err)) return false;
    p.observable_file = run_output(r.run, p.observable_file);
    p.drift_max_file = run_output(r.run, p.drift_max_file);
    return true;
}

bool read_omega_input(const Model& m, RunPaths& r, std::vector<double>& omega, bool sp, std::string& err)
{
    const Param& p = m.p;
    const int nf = m.n_modes();
    const size_t V = (size_t)m.size();
    omega.assign((size_t)std::max(0, nf) * V * 2, 0.0);
    if (nf <= 0) return true;
    errno = 0;
    FILE* probe = std::fopen(r.input_omega.c_str(), "r");
    if (!probe) {
        if (r.zero_missing_default_omega && errno == ENOENT) {
            if (sp) std::printf("%s not found; initializing omega fields to zero.\n", r.input_omega.c_str());
            return true;
        }
        return err = open_error(r.input_omega), false;
    }
    std::fclose(probe);
    FieldTable t;
    if (!read_field_table(r.input_omega, p.m1, p.m2, p.m3, t, err)) return false;
    if (!m.legacy_ab() && t.field_count != nf) {
        err = r.input_omega + ": expected " + std::to_string(2 * nf) + " numeric columns per row";
        return false;
    }
    size_t expected = grid(t.m1, t.m2, t.m3);
    const size_t rows = t.rows();
    if (!t.header && rows != expected) {
        if (!infer_mesh(rows, p, t.m1, t.m2, t.m3)) {
            err = r.input_omega + ": cannot infer mesh from " + std::to_string(rows) + " rows";
            return false;
        }
        expected = grid(t.m1, t.m2, t.m3);
        if (sp) std::printf("inferred mesh of %s as %d %d %d\n", r.input_omega.c_str(), t.m1, t.m2, t.m3);
    }
    if (rows != expected) {
        err = r.input_omega + ": rows " + std::to_string(rows) + ", expected " + std::to_string(expected);
        return false;
    }
    r.source_mesh_known = true;
    r.source_m1 = t.m1; r.source_m2 = t.m2; r.source_m3 = t.m3;
    FieldTable fin = t;
    if (t.m1 != p.m1 || t.m2 != p.m2 || t.m3 != p.m3) {
        if (sp) std::printf("resizing %s from %d %d %d to %d %d %d\n", r.input_omega.c_str(), t.m1, t.m2, t.m3, p.m1, p.m2, p.m3);
        if (!resize_table(t, p.m1, p.m2, p.m3, fin, err)) return false;
    }
    if (m.legacy_ab()) {
        if (fin.field_count == 1 && sp)
            std::printf("%s has one complex field; reading it as the legacy A/B composition field and setting the legacy density field to zero.\n",
                        r.input_omega.c_str());
        return legacy_to_active(m, fin, omega, err);
    }
    omega.swap(fin.fields);
    return true;
}

bool read_psi_input(const Model& m, const RunPaths& r, std::vector<double>& psi, bool sp, std::string& err)
{
    const Param& p = m.p;
    const size_t V = (size_t)m.size();
    psi.assign(2 * V, 0.0);
    FILE* probe = std::fopen(r.input_psi.c_str(), "r");
    if (!probe) {
        if (sp) std::printf("%s not found; initializing Psi to zero.\n", r.input_psi.c_str());
        return true;
    }
    std::fclose(probe);
    FieldTable t;
    if (!read_field_table(r.input_psi, p.m1, p.m2, p.m3, t, err)) return false;
    if (t.field_count > 1) {
        err = "bad line in " + r.input_psi + ": expected one complex value per row";
        return false;
    }
    size_t expected = grid(t.m1, t.m2, t.m3);
    const size_t rows = t.rows();
    if (rows != expected && !t.header && r.source_mesh_known && rows == grid(r.source_m1, r.source_m2, r.source_m3)) {
        t.m1 = r.source_m1; t.m2 = r.source_m2; t.m3 = r.source_m3;
        expected = rows;
    }
    if (rows != expected && !t.header) {
        if (!infer_mesh(rows, p, t.m1, t.m2, t.m3)) {
            err = r.input_psi + ": cannot infer mesh from " + std::to_string(rows) + " rows";
            return false;
        }
        expected = grid(t.m1, t.m2, t.m3);
        if (sp) std::printf("inferred mesh of %s as %d %d %d\n", r.input_psi.c_str(), t.m1, t.m2, t.m3);
    }
    if (rows != expected) {
        err = r.input_psi + ": rows " + std::to_string(rows) + ", expected " + std::to_string(expected);
        return false;
    }
    if (t.m1 != p.m1 || t.m2 != p.m2 || t.m3 != p.m3) {
        if (sp) std::printf("resizing %s from %d %d %d to %d %d %d\n", r.input_psi.c_str(), t.m1, t.m2, t.m3, p.m1, p.m2, p.m3);
        trilinear_resize(t.fields.data(), t.m1, t.m2, t.m3, psi, p.m1, p.m2, p.m3);
    } else {
        psi.swap(t.fields);
    }
    return true;
}

bool read_omega_exact(const Model& m, const std::string& file, std::vector<double>& omega, std::string& err)
{
    const Param& p = m.p;
    const int nf = m.n_modes();
    const size_t V = (size_t)m.size();
    omega.assign((size_t)std::max(0, nf) * V * 2, 0.0);
    if (nf <= 0) return true;
    FieldTable t;
    if (!read_field_table(file, p.m1, p.m2, p.m3, t, err)) return false;
    if (!m.legacy_ab() && t.field_count != nf) {
        err = file + ": expected " + std::to_string(2 * nf) + " numeric columns per row";
        return false;
    }
    if (t.m1 != p.m1 || t.m2 != p.m2 || t.m3 != p.m3) return err = file + ": checkpoint mesh does not match current mesh", false;
    if (t.rows() != V) return err = file + ": rows " + std::to_string(t.rows()) + ", expected " + std::to_string(V), false;
    if (m.legacy_ab()) return legacy_to_active(m, t, omega, err);
    omega.swap(t.fields);
    return true;
}

bool read_complex_exact(const Model& m, const std::string& file, std::vector<double>& field, std::string& err)
{
    const Param& p = m.p;
    FieldTable t;
    if (!read_field_table(file, p.m1, p.m2, p.m3, t, err)) return false;
    if (t.field_count > 1) return err = "bad line in " + file + ": expected one complex value per row", false;
    if (t.m1 != p.m1 || t.m2 != p.m2 || t.m3 != p.m3) return err = file + ": checkpoint mesh does not match current mesh", false;
    if (t.rows() != (size_t)m.size()) return err = file + ": rows " + std::to_string(t.rows()) + ", expected " + std::to_string(m.size()), false;
    field.swap(t.fields);
    return true;
}

bool write_omega(const Model& m, const std::string& file, const std::vector<double>& omega, std::string& err)
{
    const size_t V = (size_t)m.size();
    const int nf = m.n_modes();
    if (nf <= 0) return write_fields(file, m.p, nullptr, 0, V, err);
    if (m.legacy_ab()) {
        std::vector<double> legacy(4 * V, 0.0);
        const int comp = active_by_sign(m, false), dens = active_by_sign(m, true);
        if (comp >= 0) std::copy(omega.begin() + (ptrdiff_t)(2 * V * comp), omega.begin() + (ptrdiff_t)(2 * V * (comp + 1)), legacy.begin());
        if (dens >= 0) std::copy(omega.begin() + (ptrdiff_t)(2 * V * dens), omega.begin() + (ptrdiff_t)(2 * V * (dens + 1)), legacy.begin() + 2 * V);
        return write_fields(file, m.p, legacy.data(), 2, V, err);
    }
    return write_fields(file, m.p, omega.data(), nf, V, err);
}

bool write_ion_densities(const Model& m, const std::string& prefix, const std::vector<double>& ion_rho, std::string& err)
{
    bool ok = true;
    const size_t V = (size_t)m.size();
    for (size_t j = 0; j < m.ions.size(); ++j) {
        char name[1024];
        std::snprintf(name, sizeof(name), "%s_%zu_%s.rf", prefix.c_str(), j, m.ions[j].name.c_str());
        std::string e;
        if (!write_fields(name, m.p, ion_rho.data() + 2 * V * j, 1, V, e)) {
            ok = false;
            if (err.empty()) err = e;
        }
    }
    return ok;
}

}  // namespace host
}  // namespace ftsp
