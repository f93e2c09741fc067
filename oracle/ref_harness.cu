// Test-infrastructure harness around the REFERENCE implementation.
//
// This file is part of the checker, not of the product.  It is compiled
// together with the reference's own, unmodified sources (every FTSPolySol
// *.cu file except main.cu) by oracle/build_ref.sh into oracle/_ref/, and it
// drives the reference's classes exactly as main.cu does (main.cu:9-93):
// param::read -> fieldIO::prepare -> polymerSpecies::setup -> param::validate
// -> ion::build -> spectral::build_kernels -> complexLangevin::initialize.
//
// Modes:
//   golden <case.param> <omega.rf> <psi.rf> <outdir> <steps> [noise.bin]
//       Dumps derived parameters, the densities and observables at the input
//       fields, then `steps` complex-Langevin steps (complexLangevin.cu:669-698)
//       with the noise read from noise.bin (raw eta values, before the psi
//       mean removal of generate_noises, complexLangevin.cu:287-297) or, when
//       no file is given, the reference's own noise path.  Every array is a
//       raw little-endian float64 file listed in <outdir>/manifest.txt.
//   time <case.param> <omega.rf> <psi.rf> <warmup> <steps>
//       Times complexLangevin::run_step with CUDA events and prints one JSON
//       line (steps/s of the reference build on this GPU).
//
// Access to the class internals is obtained by compiling the reference
// headers with `private` mapped to `public`; no reference source is changed.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "common.h"
#include "errHandle.h"
#include "parse.h"
#include "interactionMode.h"

#define private public
#define protected public
#include "param.h"
#include "deviceState.h"
#include "polymer.h"
#include "ion.h"
#include "stress.h"
#include "observable.h"
#include "complexLangevin.h"
#include "fieldIO.h"
#include "spectral.h"
#undef private
#undef protected

namespace {

struct Dumper {
    std::string dir;
    FILE* manifest = nullptr;
    explicit Dumper(const std::string& d) : dir(d)
    {
        manifest = std::fopen((dir + "/manifest.txt").c_str(), "w");
        if (!manifest) {
            std::fprintf(stderr, "harness: cannot open manifest in %s\n", dir.c_str());
            std::exit(2);
        }
    }
    ~Dumper()
    {
        if (manifest) std::fclose(manifest);
    }
    void raw(const std::string& name, const double* data, size_t count, const std::string& shape)
    {
        FILE* fp = std::fopen((dir + "/" + name + ".bin").c_str(), "wb");
        if (!fp) {
            std::fprintf(stderr, "harness: cannot write %s\n", name.c_str());
            std::exit(2);
        }
        if (count) std::fwrite(data, sizeof(double), count, fp);
        std::fclose(fp);
        std::fprintf(manifest, "%s %s\n", name.c_str(), shape.c_str());
        std::fflush(manifest);
    }
    void complex_host(const std::string& name, const std::vector<Complex>& v, size_t fields, size_t size)
    {
        raw(name, reinterpret_cast<const double*>(v.data()), 2 * v.size(),
            std::to_string(fields) + "," + std::to_string(size) + ",2");
    }
    void complex_device(const std::string& name, const Complex* dptr, size_t fields, size_t size)
    {
        std::vector<Complex> h(fields * size);
        if (!h.empty()) CUDA_CHECK(cudaMemcpy(h.data(), dptr, h.size() * sizeof(Complex), cudaMemcpyDeviceToHost));
        complex_host(name, h, fields, size);
    }
    void real_device(const std::string& name, const double* dptr, size_t fields, size_t size)
    {
        std::vector<double> h(fields * size);
        if (!h.empty()) CUDA_CHECK(cudaMemcpy(h.data(), dptr, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
        raw(name, h.data(), h.size(), std::to_string(fields) + "," + std::to_string(size));
    }
    void scalars(const std::string& name, const std::vector<double>& v)
    {
        raw(name, v.data(), v.size(), std::to_string(v.size()));
    }
    void complex_list(const std::string& name, const std::vector<Complex>& v)
    {
        raw(name, reinterpret_cast<const double*>(v.data()), 2 * v.size(), std::to_string(v.size()) + ",2");
    }
};

struct Setup {
    parse::options options;
    param p;
    fieldIO io;
    polymerSpecies poly;
    ion ions;
    std::vector<Complex> omega, psi;
    std::vector<double> Gamma, PHI, k2, ion_kernels;
};

bool setup(Setup& s, const char* param_file, const char* omega_file, const char* psi_file)
{
    s.options.param_file = param_file;
    s.options.omega_file = omega_file;
    s.options.omega_override = true;
    s.options.psi_file = psi_file;
    s.options.psi_override = true;
    if (!s.p.read(param_file)) return false;
    if (!s.io.prepare(s.options, s.p)) return false;
    if (!s.poly.setup(s.p)) return false;
    if (!s.p.validate()) return false;
    if (!s.ions.build(s.p, s.poly.total_polymer_charge())) return false;
    const int size = s.p.size();
    s.omega.assign(static_cast<size_t>(s.p.omega_count()) * size, complex_zero());
    s.psi.assign(size, complex_zero());
    spectral::build_kernels(s.p, s.poly, s.Gamma, s.PHI, s.k2);
    s.ions.build_kernels(s.p, s.k2, s.ion_kernels);
    if (!s.io.read_omega_fields(s.p, s.omega)) return false;
    if (s.p.electrostatics_enabled()) {
        if (!s.io.read_psi_field(s.p, s.psi)) return false;
    }
    return true;
}

std::vector<double> record_values(const observableRecord& r)
{
    // Complex values in the order: chemical[], chemical_self[], chemical_ideal[],
    // hamiltonian_density, stress_values[]  (re, im interleaved).
    std::vector<double> v;
    auto put = [&](const Complex& z) { v.push_back(z.x); v.push_back(z.y); };
    for (const Complex& z : r.chemical) put(z);
    for (const Complex& z : r.chemical_self) put(z);
    for (const Complex& z : r.chemical_ideal) put(z);
    put(r.hamiltonian_density);
    for (const Complex& z : r.stress_values) put(z);
    return v;
}

void dump_derived(Dumper& D, Setup& s)
{
    param& p = s.p;
    std::vector<double> g;
    g.push_back(p.m1); g.push_back(p.m2); g.push_back(p.m3);
    g.push_back(p.L1); g.push_back(p.L2); g.push_back(p.L3);
    g.push_back(p.dV); g.push_back(p.volume()); g.push_back(p.rho0);
    g.push_back(p.a); g.push_back(p.lB); g.push_back(p.dt); g.push_back(p.lambdaPsi);
    g.push_back(p.short_range_self_pressure());
    g.push_back(p.monomer_count()); g.push_back(p.omega_count());
    D.scalars("derived_scalars", g);
    std::vector<double> modes;
    for (int a = 0; a < p.omega_count(); ++a) {
        modes.push_back(p.omega_coefficient(a));
        modes.push_back(p.omega_mobility(a));
        modes.push_back(p.omega_gamma(a).x);
        modes.push_back(p.omega_gamma(a).y);
        modes.push_back(p.modes.active_eigenvalue(a));
        for (int alpha = 0; alpha < p.monomer_count(); ++alpha) modes.push_back(p.omega_O(a, alpha));
    }
    D.scalars("derived_modes", modes);
    std::vector<double> ions;
    for (const IonSpecies& sp : s.ions.all()) {
        ions.push_back(sp.valence);
        ions.push_back(static_cast<double>(sp.count));
        ions.push_back(sp.smearing_length);
    }
    D.scalars("derived_ions", ions);
    std::vector<double> poly;
    for (const polymerSpecies::Species& sp : s.poly.all()) {
        poly.push_back(static_cast<double>(sp.num_chains));
        poly.push_back(sp.N);
        for (int t = 0; t < sp.N; ++t) {
            poly.push_back(sp.monomer_type(t));
            poly.push_back(sp.charge(t));
            poly.push_back(sp.bond_length(t));
        }
    }
    D.scalars("derived_polymers", poly);
}

void dump_densities(Dumper& D, Setup& s, complexLangevin& cl, const std::string& tag, const std::vector<Complex>& Q)
{
    const param& p = s.p;
    const size_t size = static_cast<size_t>(p.size());
    deviceState& d = cl.d;
    D.complex_list(tag + "_Q", Q);
    D.complex_device(tag + "_rho_type", d.rho_type, p.monomer_count(), size);
    D.complex_device(tag + "_rho_p", d.rho_p, 1, size);
    D.complex_device(tag + "_rho_c", d.rho_c, 1, size);
    D.complex_device(tag + "_rho_c_poly", d.rho_c_poly, 1, size);
    D.complex_device(tag + "_rho_c_ion", d.rho_c_ion, 1, size);
    if (!s.ions.empty()) D.complex_device(tag + "_ion_rho", d.ion_rho, s.ions.count(), size);
    D.complex_device(tag + "_W_type_s", d.W_type_s, p.monomer_count(), size);
    D.complex_device(tag + "_psi_s", d.psi_s, 1, size);
}

bool read_noise(const std::string& path, std::vector<double>& out)
{
    std::ifstream in(path, std::ios::binary);
    if (!in) return false;
    in.seekg(0, std::ios::end);
    const size_t bytes = static_cast<size_t>(in.tellg());
    in.seekg(0, std::ios::beg);
    out.resize(bytes / sizeof(double));
    in.read(reinterpret_cast<char*>(out.data()), static_cast<std::streamsize>(out.size() * sizeof(double)));
    return static_cast<bool>(in);
}

// One CL step in the order of complexLangevin::run_step (complexLangevin.cu:669-698),
// with generate_noises replaced by the injected values (plus the same psi-noise
// mean removal) when `eta` is non-null.
bool step_once(Setup& s, complexLangevin& cl, int step, const double* eta, Dumper& D)
{
    param& p = s.p;
    deviceState& d = cl.d;
    const int size = p.size();
    std::vector<Complex> Qp = cl.compute_densities(d.omega, d.psi);
    if (!cl.finite_chain_partitions(Qp, "Q", step)) return false;
    copy_complex(d.rho_c_old, d.rho_c, size);

    if (eta) {
        const size_t nm = static_cast<size_t>(p.omega_count());
        if (nm) copy_to_device(d.eta_omega, eta, nm * size);
        copy_to_device(d.etaPsi, eta + nm * size, static_cast<size_t>(size));
        if (p.electrostatics_enabled()) remove_real_mean(d.etaPsi, size);
    } else {
        cl.generate_noises();
    }
    cl.compute_drifts(d.omega, d.drift);
    cl.predictor_step();

    Qp = cl.compute_densities(d.omega_bar, d.psi_bar);
    if (!cl.finite_chain_partitions(Qp, "Qbar", step)) return false;
    cl.compute_psi_drift(d.psi_bar, d.rho_c, d.dpsi_bar);
    const std::string tag = "step" + std::to_string(step);
    dump_densities(D, s, cl, tag + "_bar", Qp);
    D.complex_device(tag + "_omega_bar", d.omega_bar, p.omega_count(), size);
    D.complex_device(tag + "_psi_bar", d.psi_bar, 1, size);
    D.complex_device(tag + "_dpsi", d.dpsi, 1, size);
    D.complex_device(tag + "_dpsi_bar", d.dpsi_bar, 1, size);
    D.complex_device(tag + "_drift", d.drift, p.omega_count(), size);

    observableRecord record = cl.obs.measure(cl.plan, d, Qp, d.omega_bar, d.psi_bar);
    D.scalars(tag + "_record", record_values(record));

    cl.compute_drifts(d.omega_bar, d.drift_bar);
    D.complex_device(tag + "_drift_bar", d.drift_bar, p.omega_count(), size);
    std::vector<double> dmax;
    for (int a = 0; a < p.omega_count(); ++a) {
        dmax.push_back(cl.corrector_drift_max(d.obs_a, d.drift + static_cast<size_t>(a) * size,
                                              d.drift_bar + static_cast<size_t>(a) * size, p.omega_mobility(a)));
    }
    dmax.push_back(cl.corrector_drift_max(d.obs_a, d.dpsi, d.dpsi_bar, p.lambdaPsi));
    D.scalars(tag + "_drift_max", dmax);
    cl.corrector_step();
    D.complex_device(tag + "_omega", d.omega, p.omega_count(), size);
    D.complex_device(tag + "_psi", d.psi, 1, size);
    return true;
}

int golden(int argc, char** argv)
{
    if (argc < 7) {
        std::fprintf(stderr, "usage: %s golden case.param omega.rf psi.rf outdir steps [noise.bin]\n", argv[0]);
        return 2;
    }
    Setup s;
    if (!setup(s, argv[2], argv[3], argv[4])) return 1;
    const std::string outdir = argv[5];
    const int steps = std::atoi(argv[6]);
    std::vector<double> noise;
    if (argc > 7 && !read_noise(argv[7], noise)) {
        std::fprintf(stderr, "harness: cannot read noise file %s\n", argv[7]);
        return 1;
    }
    const size_t size = static_cast<size_t>(s.p.size());
    const size_t per_step = (static_cast<size_t>(s.p.omega_count()) + 1) * size;
    if (!noise.empty() && noise.size() < per_step * static_cast<size_t>(steps)) {
        std::fprintf(stderr, "harness: noise file too short\n");
        return 1;
    }

    Dumper D(outdir);
    dump_derived(D, s);
    D.complex_host("input_omega", s.omega, s.p.omega_count(), size);
    D.complex_host("input_psi", s.psi, 1, size);
    D.scalars("k2", s.k2);
    D.scalars("Gamma", s.Gamma);

    complexLangevin cl(s.p, s.poly, s.ions);
    if (!cl.initialize(s.omega, s.psi, s.Gamma, s.PHI, s.k2, s.ion_kernels)) return 1;
    D.complex_device("init_psi", cl.d.psi, 1, size);

    // Densities and observables at the input fields.
    std::vector<Complex> Q0 = cl.compute_densities(cl.d.omega, cl.d.psi);
    dump_densities(D, s, cl, "init", Q0);
    const int nmax = std::max(1, s.p.Nmax);
    if (s.poly.count() == 1) {
        D.complex_device("init_qF", cl.d.qF, nmax, size);
        D.complex_device("init_qB", cl.d.qB, nmax, size);
    }
    observableRecord r0 = cl.obs.measure(cl.plan, cl.d, Q0, cl.d.omega, cl.d.psi);
    D.scalars("init_record", record_values(r0));

    for (int step = 1; step <= steps; ++step) {
        const double* eta = noise.empty() ? nullptr : noise.data() + per_step * static_cast<size_t>(step - 1);
        if (!step_once(s, cl, step, eta, D)) return 1;
    }
    std::printf("golden: wrote %d steps to %s\n", steps, outdir.c_str());
    return 0;
}

int timing(int argc, char** argv)
{
    if (argc < 7) {
        std::fprintf(stderr, "usage: %s time case.param omega.rf psi.rf warmup steps\n", argv[0]);
        return 2;
    }
    const auto t0 = std::chrono::steady_clock::now();
    Setup s;
    if (!setup(s, argv[2], argv[3], argv[4])) return 1;
    const int warmup = std::atoi(argv[5]);
    const int steps = std::atoi(argv[6]);
    complexLangevin cl(s.p, s.poly, s.ions);
    if (!cl.initialize(s.omega, s.psi, s.Gamma, s.PHI, s.k2, s.ion_kernels)) return 1;
    const auto t1 = std::chrono::steady_clock::now();
    // A step that ends non-finite is followed by a restore of the input
    // fields (the reference's checkpoint restart, complexLangevin.cu:626-636,
    // taken from memory instead of the checkpoint files) so that the timed
    // sample keeps running; restarts are counted and reported.
    int step = 0;
    int restarts = 0;
    auto restore = [&]() {
        copy_to_device(cl.d.omega, s.omega);
        copy_to_device(cl.d.psi, s.psi);
        cl.remove_psi_zero_mode(cl.d.psi);
        ++restarts;
    };
    for (int i = 0; i < warmup; ++i) {
        const auto st = cl.run_step(false, ++step);
        if (st == complexLangevin::StepStatus::failed) return 1;
        if (st == complexLangevin::StepStatus::nonfinite) restore();
    }
    CUDA_CHECK(cudaDeviceSynchronize());
    cudaEvent_t e0, e1;
    CUDA_CHECK(cudaEventCreate(&e0));
    CUDA_CHECK(cudaEventCreate(&e1));
    const auto w0 = std::chrono::steady_clock::now();
    CUDA_CHECK(cudaEventRecord(e0));
    for (int i = 0; i < steps; ++i) {
        const auto st = cl.run_step(false, ++step);
        if (st == complexLangevin::StepStatus::failed) return 1;
        if (st == complexLangevin::StepStatus::nonfinite) restore();
    }
    CUDA_CHECK(cudaEventRecord(e1));
    CUDA_CHECK(cudaEventSynchronize(e1));
    const auto w1 = std::chrono::steady_clock::now();
    float ms = 0.0f;
    CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
    const double wall = std::chrono::duration<double>(w1 - w0).count();
    const double setup_s = std::chrono::duration<double>(t1 - t0).count();
    std::printf("{\"impl\": \"reference-cuda\", \"grid\": [%d, %d, %d], \"N\": %d, \"steps\": %d, \"warmup\": %d, "
                "\"event_ms_per_step\": %.6f, \"wall_ms_per_step\": %.6f, \"steps_per_s\": %.6f, \"setup_s\": %.3f, "
                "\"restarts\": %d}\n",
                s.p.m1, s.p.m2, s.p.m3, s.p.Nmax, steps, warmup, ms / steps, 1e3 * wall / steps,
                steps / (ms * 1e-3), setup_s, restarts);
    return 0;
}

} // namespace

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s golden|time ...\n", argv[0]);
        return 2;
    }
    if (std::strcmp(argv[1], "golden") == 0) return golden(argc, argv);
    if (std::strcmp(argv[1], "time") == 0) return timing(argc, argv);
    std::fprintf(stderr, "unknown mode %s\n", argv[1]);
    return 2;
}
