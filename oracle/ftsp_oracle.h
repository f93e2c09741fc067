/* FP64 CPU oracle of the FTSPolySol complex-Langevin step -- TEST
 * INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py may load it, and only as the checker; the product
 * path never calls it.
 *
 * It restates, literally and in the same operation order, the reference
 * algorithm: spectral tables (spectral.cu:3-35), chain propagators and
 * densities (polymer.cu:341-478), ion densities (ion.cu:54-72,
 * common.h:1104-1130), drifts and the predictor-corrector update
 * (complexLangevin.cu:272-368, 669-698), chemical potentials and the
 * mean-field Hamiltonian (observable.cu:53-182), the isotropic pressure
 * (observable.cu:184-317) and the k-space stress tensor (stress.cu:106-321),
 * including the re-solves of the chain propagators inside the stress and
 * pressure operators.  The 3-D FFT is an own mixed-radix Stockham transform
 * with cuFFT's conventions (forward sign -1, both directions unnormalised).
 *
 * Parity is pinned against dumps of the reference's own CUDA build
 * (the .npz files of tests/golden, made by tests/golden/make_golden.py).
 */
#ifndef FTSP_ORACLE_H
#define FTSP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_config {
    int m1, m2, m3;
    double L1, L2, L3;
    double dV;
    double a;                    /* bead smearing length (Gamma of the chains) */
    double lB;                   /* Bjerrum length; electrostatics on iff > 0   */
    double dt;
    double lambda_psi;
    int M;                       /* monomer types                               */
    int n_modes;                 /* active interaction modes                    */
    const double* mode_coeff;    /* [n_modes]   rho0/|d_a|                      */
    const double* mode_gamma;    /* [n_modes*2] complex gamma_a (i or 1)        */
    const double* mode_O;        /* [n_modes*M] O_{a alpha}                     */
    const double* mode_lambda;   /* [n_modes]   mobility                        */
    int n_species;
    const double* num_chains;    /* [n_species]                                 */
    const int* N;                /* [n_species] segments per chain              */
    const int* seg_type;         /* concatenated per-segment monomer type       */
    const double* seg_charge;    /* concatenated per-segment valence            */
    const double* seg_bond;      /* concatenated per-segment bond length s->s+1 */
    int n_ions;
    const double* ion_valence;   /* [n_ions] */
    const double* ion_count;     /* [n_ions] */
    const double* ion_smear;     /* [n_ions] */
    double self_pressure;        /* param::short_range_self_pressure            */
    int stress_mask;             /* bit c: component c of XX,YY,ZZ,XY,XZ,YZ     */
    int isotropic_pressure;
} oracle_config;

typedef struct oracle_state oracle_state;

oracle_state* oracle_create(const oracle_config* cfg);
void oracle_destroy(oracle_state* h);
int oracle_threads(void);

/* Loads omega[n_modes*V] and psi[V] (interleaved re,im doubles) and removes
 * the psi zero mode, as complexLangevin::initialize does. */
void oracle_set_fields(oracle_state* h, const double* omega, const double* psi);

/* Densities at (omega, psi) when which == 0, at (omega_bar, psi_bar) when 1.
 * Q_out receives n_species complex values. */
void oracle_compute_densities(oracle_state* h, int which, double* Q_out);

/* Observable record at (omega, psi) (which == 0) or the predictor fields
 * (which == 1), using the Q values passed in.  Record layout (complex,
 * interleaved): chemical[S+J], chemical_self[S+J], chemical_ideal[S+J],
 * hamiltonian, stress components (active, XX..YZ order), pressure.
 * Returns the number of complex values written. */
int oracle_measure(oracle_state* h, int which, const double* Q, double* record_out);

/* One predictor-corrector step.  eta: raw noise [(n_modes+1)*V] doubles
 * (modes, then psi) or NULL for zero noise.  Q_bar_out[n_species*2],
 * record_out (as oracle_measure), drift_max_out[n_modes+1]. */
int oracle_step(oracle_state* h, const double* eta, double* Q_bar_out, double* record_out, double* drift_max_out);

/* Copies a named buffer out (interleaved complex doubles, or doubles for the
 * real tables).  Returns the number of doubles copied, -1 for an unknown
 * name.  Names: omega psi omega_bar psi_bar omega_s psi_s W_type_s rho_type
 * rho_p rho_c rho_c_poly rho_c_ion rho_c_old ion_rho drift drift_bar dpsi
 * dpsi_bar qF qB k2 Gamma. */
long long oracle_get(oracle_state* h, const char* name, double* out);

/* Plain 3-D FFT of one complex field (cuFFT conventions): sign -1 forward,
 * +1 inverse, unnormalised.  For the FFT's own tests. */
void oracle_fft3d(int m1, int m2, int m3, double* data, int sign);

#ifdef __cplusplus
}
#endif
#endif
