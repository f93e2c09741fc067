// Field files and run-directory layout of the reference (fieldIO.cu,
// trilinear.cu, common.h:229-290, 375-460).
//
// A field file holds an optional mesh header "m1 m2 m3", an optional box
// line "L1 L2 L3" right after it, then one row per grid point (x slowest,
// z fastest) with `re im` pairs for every field in the file.  Fields are kept
// here as interleaved complex doubles, field-major.
#pragma once

#include <string>
#include <vector>

#include "host_model.h"

namespace ftsp {
namespace host {

struct FieldTable {
    int m1 = 0, m2 = 0, m3 = 0;
    bool header = false;
    int field_count = 0;
    std::vector<double> fields;   // [field][row][re,im]
    size_t rows() const { return field_count > 0 ? fields.size() / (2 * (size_t)field_count) : 0; }
};

// Readers return false and set `err` (the reference's error text).
bool read_field_table(const std::string& file, int m1, int m2, int m3, FieldTable& t, std::string& err);
bool write_fields(const std::string& file, const Param& p, const double* fields, int count, size_t size, std::string& err);

// Mesh inference for a header-less file (fieldIO.cu:226-258).
bool infer_mesh(size_t rows, const Param& p, int& m1, int& m2, int& m3);
// Periodic trilinear resampling of one complex field (trilinear.cu:13-61).
void trilinear_resize(const double* in, int n1, int n2, int n3, std::vector<double>& out, int m1, int m2, int m3);

// Step output template helpers (common.h:272-288, fieldIO.cu:194-224).
bool valid_step_template(const std::string& pattern);
std::string step_filename(const std::string& pattern, int step);
std::string join_path(const std::string& a, const std::string& b);
std::string basename_path(const std::string& path);
bool make_directories(const std::string& path, std::string& err);

struct Options {
    std::string param_file = "param";
    std::string omega_file, psi_file, sequence_file, run_id, run_parent = ".";
    bool omega_override = false, psi_override = false, sequence_override = false;
    bool run_id_set = false, run_parent_set = false, screenprint = false;
    // engine options (no reference counterpart)
    int precision = 0, scheme = 0, device = 0, autotune = 0;
    double adaptive = 0.0;   // adaptive-step bound u_ref (0: fixed step)
    bool seed_set = false;
    unsigned long long seed = 0;
};

// Command line of the reference (parse.cu:3-45) plus --fp32/--fp64, --si/--pc,
// --seed N and --device N.  Returns 0 to continue, 1 for --help, -1 on error.
int parse_args(int argc, char** argv, Options& o, std::string& err);
void usage(const char* program);

// Run directory, input names and output paths (fieldIO.cu:3-45).
struct RunPaths {
    std::string run, input_omega, input_psi;
    bool zero_missing_default_omega = false;
    bool source_mesh_known = false;
    int source_m1 = 0, source_m2 = 0, source_m3 = 0;
};
bool prepare_run(const Options& o, Param& p, RunPaths& r, std::string& err);

// Initial fields (fieldIO.cu:432-520): omega [n_modes][V] and psi [V].
bool read_omega_input(const Model& m, RunPaths& r, std::vector<double>& omega, bool screenprint, std::string& err);
bool read_psi_input(const Model& m, const RunPaths& r, std::vector<double>& psi, bool screenprint, std::string& err);
// Checkpoint readers: exact mesh required (fieldIO.cu:522-551).
bool read_omega_exact(const Model& m, const std::string& file, std::vector<double>& omega, std::string& err);
bool read_complex_exact(const Model& m, const std::string& file, std::vector<double>& field, std::string& err);
// Omega writer in the file order of the model (legacy A/B or active modes).
bool write_omega(const Model& m, const std::string& file, const std::vector<double>& omega, std::string& err);
bool write_ion_densities(const Model& m, const std::string& prefix, const std::vector<double>& ion_rho, std::string& err);

}  // namespace host
}  // namespace ftsp
