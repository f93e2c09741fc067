/* ftsp.h -- C ABI of the B200 complex-Langevin engine (libftsp.so).
 *
 * Drop-in boundary for the step loop of FTSPolySol.  The reference exposes
 * no FFI: its boundary is the C++ class surface that main.cu drives from one
 * host thread.  Each entry point below names the reference interface it
 * replaces (file:line in the FTSPolySol sources).  Plain pointers and sizes
 * only; complex fields are interleaved (re, im) float64 pairs in the
 * reference's row-major (x, y, z) order with z fastest (common.h:54-58), the
 * layout of cufftDoubleComplex.
 *
 * Conventions (replacing errHandle.cu:3-84, which prints and exit()s):
 *   every call returns FTSP_OK (0), FTSP_NONFINITE (1: a non-finite Q, field
 *   or observable, the reference's StepStatus::nonfinite,
 *   complexLangevin.h:31-35), FTSP_ERROR (2) or FTSP_TIMEOUT (3); nothing
 *   calls exit().  ftsp_last_error() gives the message of the last failure.
 *   A handle is used from one host thread at a time; all device work of a
 *   handle runs on one CUDA stream (ftsp_set_stream).
 */
#ifndef FTSP_H
#define FTSP_H

#ifdef __cplusplus
extern "C" {
#endif

#define FTSP_OK 0
#define FTSP_NONFINITE 1
#define FTSP_ERROR 2
#define FTSP_TIMEOUT 3

#define FTSP_FP64 0
#define FTSP_FP32 1

#define FTSP_SCHEME_PC 0   /* the reference's predictor-corrector (complexLangevin.cu:328-368) */
#define FTSP_SCHEME_SI 1   /* semi-implicit PC with the analytic linear-response kernel (no reference counterpart) */

#define FTSP_STRESS_XX 1
#define FTSP_STRESS_YY 2
#define FTSP_STRESS_ZZ 4
#define FTSP_STRESS_XY 8
#define FTSP_STRESS_XZ 16
#define FTSP_STRESS_YZ 32

/* Derived model parameters: what param::derive (param.cu:342-359),
 * interactionMode::build (interactionMode.cu:9-59), polymerSpecies::setup
 * (polymer.cu:185-194) and ion::build (ion.cu:3-46) produce.  Array
 * arguments are copied by ftsp_create. */
typedef struct ftsp_config {
    int m1, m2, m3;              /* mesh                                              */
    double L1, L2, L3;           /* box lengths                                       */
    double dV;                   /* cell volume dL^3                                  */
    double a;                    /* bead smearing length                              */
    double lB;                   /* Bjerrum length; electrostatics on iff lB > 0      */
    double dt;
    double lambda_psi;
    int M;                       /* monomer types                                     */
    int n_modes;                 /* active interaction modes                          */
    const double* mode_coeff;    /* [n_modes]     rho0 / |d_a|                        */
    const double* mode_gamma;    /* [2*n_modes]   complex gamma_a (i or 1)            */
    const double* mode_O;        /* [n_modes*M]   O_{a alpha}                         */
    const double* mode_lambda;   /* [n_modes]     mobilities                          */
    int n_species;
    const double* num_chains;    /* [n_species]                                       */
    const int* N;                /* [n_species]   segments per chain                  */
    const int* seg_type;         /* [sum N]       monomer type of each segment        */
    const double* seg_charge;    /* [sum N]       valence of each segment             */
    const double* seg_bond;      /* [sum N]       bond length s -> s+1 (last unused)  */
    int n_ions;
    const double* ion_valence;   /* [n_ions] */
    const double* ion_count;     /* [n_ions] */
    const double* ion_smear;     /* [n_ions] */
    double self_pressure;        /* param::short_range_self_pressure (param.cu:130-147) */
    int stress_mask;             /* FTSP_STRESS_* bits                                */
    int isotropic_pressure;      /* 1: append the isotropic pressure to the record    */
    int noise;                   /* 1: Langevin noise on (param [dynamics] noise)     */
    unsigned long long seed;     /* counter-based noise seed                          */
    int precision;               /* FTSP_FP64 or FTSP_FP32                            */
    int scheme;                  /* FTSP_SCHEME_PC or FTSP_SCHEME_SI                  */
    int device;                  /* CUDA device ordinal                               */
    int restart_interval;        /* >0: device checkpoint every so many steps and
                                    rollback after a non-finite step (the
                                    reference's Ntmp / max_nan_restarts recovery,
                                    complexLangevin.cu:583-636); 0: off          */
} ftsp_config;

typedef struct ftsp_handle ftsp_handle;

/* Allocates the device state and builds the spectral tables.
 * Replaces deviceState::allocate (deviceState.cu:8-61), spectral::build_kernels
 * (spectral.cu:3-35), ion::build_kernels (ion.cu:48-52) and
 * complexLangevin::initialize (complexLangevin.cu:166-191). */
int ftsp_create(const ftsp_config* cfg, ftsp_handle** out);
int ftsp_destroy(ftsp_handle* h);
const char* ftsp_last_error(const ftsp_handle* h);
int ftsp_set_stream(ftsp_handle* h, void* cuda_stream);

/* Loads omega [n_modes*V] and psi [V] from host memory (interleaved complex
 * float64) and removes the psi zero mode (complexLangevin.cu:182-183). */
int ftsp_set_fields(ftsp_handle* h, const double* omega, const double* psi);

/* Copies a named field to host memory as interleaved complex float64.
 * Names follow deviceState (deviceState.h:6-48): omega psi omega_bar psi_bar
 * drift drift_bar dpsi dpsi_bar rho_type rho_p rho_c rho_c_poly rho_c_ion
 * ion_rho W_type_s psi_s qF.  *count receives the number of doubles. */
int ftsp_get_field(ftsp_handle* h, const char* name, double* out, long long* count);

/* Densities at (omega, psi) (which = 0) or (omega_bar, psi_bar) (which = 1).
 * Q_out: n_species complex values.  Replaces complexLangevin::compute_densities
 * (complexLangevin.cu:255-260) = polymerSpecies::solve_and_compute_densities
 * (polymer.cu:449-478) + ion::compute_densities (ion.cu:54-72). */
int ftsp_compute_densities(ftsp_handle* h, int which, double* Q_out);

/* Number of complex values in an observable record. */
int ftsp_record_length(const ftsp_handle* h);

/* Observable record at the fields selected by `which` (densities are
 * re-evaluated there).  Layout (complex, interleaved): chemical[S+J],
 * chemical_self[S+J], chemical_ideal[S+J], Hamiltonian density, stress
 * components (active ones, xx yy zz xy xz yz order), isotropic pressure.
 * Replaces observable::measure (observable.cu:53-67) with stress::measure
 * (stress.cu:161-196) and isotropic_pressure_operator (observable.cu:297-317). */
int ftsp_measure(ftsp_handle* h, int which, double* record);

/* Raw noise for the next ftsp_step only: [(n_modes+1)*V] float64, modes then
 * psi, before the psi mean removal (replaces generate_noises,
 * complexLangevin.cu:287-297, for parity runs). */
int ftsp_set_noise(ftsp_handle* h, const double* eta);
int ftsp_set_seed(ftsp_handle* h, unsigned long long seed);

/* One complex-Langevin step (complexLangevin::run_step,
 * complexLangevin.cu:669-698): densities, noise, drifts, predictor, densities
 * at the predictor, observables, corrector.  Optional outputs (may be NULL):
 * Q_bar [n_species complex], record [ftsp_record_length complex], drift_max
 * [n_modes+1] (complexLangevin.cu:474-498). */
int ftsp_step(ftsp_handle* h, double* Q_bar, double* record, double* drift_max);

/* Same step with no host copies and no host synchronisation: the record
 * and status stay on the device (ftsp_read_status fetches them).  Used for
 * resident timing and CUDA-graph capture. */
int ftsp_step_async(ftsp_handle* h);
int ftsp_read_status(ftsp_handle* h, double* record, double* drift_max);

/* Forward propagators of a chain of N identical segments in an external
 * field: q_1 = exp(-w), q_{s+1} = exp(-w) IFFT[Phi FFT[q_s] / V] with
 * Phi(k) = exp(-b^2 k^2 / 6); returns q_N in q_end and Q = mean(q_N) in
 * Q[0..1] (host).  w and q_end are device arrays of V complex128 values on the
 * handle's grid; complex128 handles only.  Replaces
 * polymerSpecies::propagate_chain and the Q of solve_chain_species_prepared
 * (polymer.cu:402-426) for one segment class.  Scratch: the handle's buffers. */
int ftsp_propagate_chain(ftsp_handle* h, const double* w, int N, double bond_length, double* q_end, double* Q);

/* ftsp_propagate_chain without any device allocation, for callers that
 * cannot call cudaMalloc: code that runs while a stream is being captured
 * into a CUDA graph, code inside a framework whose caching allocator owns the
 * device memory, real-time loops that must not block on the allocator.  No
 * counterpart in the reference.  No handle: the mesh (m1..m3) and box
 * lengths (L1..L3) are passed directly; w and q_end are device arrays of
 * m1*m2*m3 complex128 values, Q (host) receives mean(q_N).  All scratch lives
 * in one static device array of about 8.3 MiB inside the library, which every
 * GPU that loads libftsp.so keeps until the process exits.  Limits: at most
 * 262144 grid points (64^3) and 256 points per axis; larger meshes return
 * FTSP_ERROR with the reason in ftsp_last_error(NULL).  The first call on a
 * device looks the scratch address up with cudaGetSymbolAddress, so make that
 * first call before any stream capture begins.  Calls that overlap on the GPU
 * share the one scratch array and race: serialise them.  Runs on cuda_stream
 * (NULL: the legacy default stream) and returns after the stream has
 * finished the call's work. */
int ftsp_propagate_chain_noalloc(int m1, int m2, int m3, double L1, double L2, double L3, const double* w, int N,
                                 double bond_length, double* q_end, double* Q, void* cuda_stream);

/* Number of checkpoint rollbacks taken so far (restart_interval > 0);
 * -1 on error.  Synchronises the handle's stream. */
long long ftsp_restart_count(ftsp_handle* h);

/* Device pointers of the resident state (FP64 handles only), in the layout of
 * deviceState (deviceState.h:6-48). */
typedef struct ftsp_views {
    void* omega;
    void* psi;
    void* omega_bar;
    void* psi_bar;
    void* rho_type;
    void* rho_p;
    void* rho_c;
    void* rho_c_poly;
    void* rho_c_ion;
    void* ion_rho;
    void* drift;
    void* drift_bar;
    void* dpsi;
    void* dpsi_bar;
} ftsp_views;
int ftsp_state_views(ftsp_handle* h, ftsp_views* views);

/* Number of this library's kernels launched by the last ftsp_step /
 * ftsp_step_async. */
long long ftsp_last_launch_count(const ftsp_handle* h);

/* CUDA-event timing of the chain-propagator passes (no reference
 * counterpart: the reference prints only its total wall time, main.cu:89-91).
 * ftsp_profile_enable clears the accumulators; while enabled, every
 * real-space segment pass and k-space bond pass is bracketed by events on the
 * handle's stream.  ftsp_profile_read synchronises the stream and returns,
 * per pass kind, the summed device time, the launch count and the
 * algorithmic bytes (the minimum HBM traffic of the pass's work). */
typedef struct ftsp_kernel_stat {
    char name[48];
    double ms;
    long long launches;
    double bytes;
} ftsp_kernel_stat;
int ftsp_profile_enable(ftsp_handle* h, int on);
int ftsp_profile_read(ftsp_handle* h, ftsp_kernel_stat* out, int max_entries, int* count);

#ifdef __cplusplus
}
#endif
#endif
