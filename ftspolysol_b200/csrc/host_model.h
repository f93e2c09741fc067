// Host-side model setup: the reference's input-file surface.
//
// Reads the INI-like param file (param.cu:165-334 key table, parse.cu value
// rules), the block sequence file (polymer.cu:219-273), builds the
// interaction modes (interactionMode.cu:9-263), the ion species
// (ion.cu:3-46), the derived quantities (param.cu:342-436) and validates them
// (param.cu:448-501).  The result fills an ftsp_config for the engine.
#pragma once

#include <string>
#include <vector>

#include "ftsp.h"

namespace ftsp {
namespace host {

struct PolymerInput {
    std::string name;
    long long num_chains = 0;
    int N = 0;
    std::vector<int> type_counts;
    bool section_seen = false, name_set = false, num_chains_set = false, N_set = false;
};

struct Param {
    // [grid]
    int m1 = 0, m2 = 0, m3 = 0;
    double a = 0.0, dL = 0.0;
    // [monomers]
    int monomer_type_count = 2;
    bool monomer_count_set = false, monomer_names_set = false;
    std::vector<std::string> monomer_names;
    // [polymer]
    int species_count = 1;
    bool species_count_set = false;
    std::string sequence_file;
    std::vector<PolymerInput> polymer_species;
    // [interactions]
    std::vector<double> chi_matrix;
    bool chi_matrix_set = false;
    double xi = 0.0, lB = 0.0, eigen_tol_rel = 1.0e-12;
    // [dynamics]
    double dt = 0.0, lambdaPsi = 0.0;
    std::vector<double> lambda_omega_input, lambda_omega;
    int Nt = 0, Nss = 0, Ns = 0, Ntmp = 0, Nso = -1, N_stat = -1, max_nan_restarts = 20;
    bool noise = true;
    // [ions]
    bool ions_enabled = false;
    double default_smearing_length = -1.0;
    bool ci_enabled = false, ci_auto = true;
    long long ci_number = 0;
    double ci_valence = 0.0, ci_smearing = -1.0;
    std::string ci_name = "counterion";
    bool salt_enabled = false;
    long long num_salt = 0;
    double cation_valence = 0.0, anion_valence = 0.0, salt_smearing = -1.0;
    int cation_stoich = 1, anion_stoich = 1;
    bool combine_identical = true;
    std::string cation_name = "salt_cation", anion_name = "salt_anion";
    // [observables]
    bool stress = false, comp[6] = {false, false, false, false, false, false}, isotropic_pressure = false;
    // [output]
    std::string omega_file = "omega.rf", psi_file = "psi.rf", tmp_omega_file = "tmp_omega.rf", tmp_psi_file = "tmp_psi.rf";
    std::string rho_type_file = "rho_type.rf", rhop_file = "rhop.rf", rhoc_file = "rhoc.rf";
    std::string rhoc_poly_file = "rhoc_poly.rf", rhoc_ion_file = "rhoc_ion.rf", ion_density_prefix = "rho_ion";
    std::string step_omega_file, step_psi_file, step_rho_type_file, step_rhop_file, step_rhoc_file;
    std::string step_rhoc_poly_file, step_rhoc_ion_file, step_ion_density_prefix;
    std::string observable_file = "observables.dat", drift_max_file = "drift_max.dat";
    // derived
    double L1 = 0.0, L2 = 0.0, L3 = 0.0, dV = 0.0, rho0 = 0.0;
    int Nmax = 0;
    long long total_chains = 0, total_segments = 0;
    std::vector<long long> total_type_segments;
};

struct Species {
    std::string name;
    long long num_chains = 0;
    std::vector<int> type;
    std::vector<double> charge, bond;   // bond[s]: s -> s+1 (last entry 1.0)
};

struct Ion {
    std::string name;
    double valence = 0.0;
    long long count = 0;
    double smearing = 0.0;
};

struct Modes {
    int M = 0;
    std::vector<double> K, eig, O;   // O row-major by mode
    std::vector<int> active;
    double tol_abs = 0.0, recon_err = 0.0, orth_err = 0.0;
};

struct Model {
    Param p;
    std::vector<Species> species;
    std::vector<Ion> ions;
    Modes modes;
    double self_pressure = 0.0;
    bool elec() const { return p.lB > 0.0; }
    int size() const { return p.m1 * p.m2 * p.m3; }
    double volume() const { return p.L1 * p.L2 * p.L3; }
    int n_modes() const { return (int)modes.active.size(); }
    // legacy A/B omega-file order (fieldIO.cu:434-477): two types, no [monomers]/chi given
    bool legacy_ab() const
    {
        return p.monomer_type_count == 2 && !p.monomer_count_set && !p.monomer_names_set && !p.chi_matrix_set;
    }
    double mode_eig(int a) const { return modes.eig[(size_t)modes.active[a]]; }

    // flat arrays backing an ftsp_config
    std::vector<double> c_coeff, c_gamma, c_O, c_lambda, c_chains, c_charge, c_bond, c_ival, c_icount, c_ismear;
    std::vector<int> c_N, c_type;
};

// Parsing helpers (parse.cu).
std::string trim(const std::string& s);
std::string strip_comment(const std::string& s);
std::string unquote(std::string s);

// Loads param + sequence, derives and validates.  Returns false with `err`.
bool load_model(const std::string& param_file, const std::string& sequence_override, Model& m, std::string& err);

// Fills an ftsp_config whose arrays point into `m` (keep `m` alive).
void fill_config(Model& m, ftsp_config& cfg);

}  // namespace host
}  // namespace ftsp
