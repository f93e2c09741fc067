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
    int autotune;                /* 1: time the launch-geometry alternatives of the
                                    runtime-plan passes at creation (cached per
                                    grid in the process); no reference counterpart */
    int max_restarts;            /* rollbacks allowed (restart_interval > 0) before a
                                    non-finite step becomes final: the reference's
                                    max_nan_restarts (param.h:74,
                                    complexLangevin.cu:626-636); <= 0: 20       */
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

/* ftsp_set_fields without waiting (no reference counterpart: the reference
 * copies its fields in once, complexLangevin.cu:166-191).  The fields are
 * copied from host memory into a device staging buffer on a separate copy
 * stream, so that an upload overlaps the step still running; the next call
 * that uses the fields (ftsp_step, ftsp_step_async, ftsp_compute_densities,
 * ftsp_measure, ftsp_get_field, ftsp_batch_create) installs them on the
 * handle's stream first, with the same effect as ftsp_set_fields.  With
 * pinned host memory the call returns at once; the host buffers must stay
 * unchanged until a later call has returned results to the host
 * (ftsp_step, ftsp_read_status, ftsp_get_field).  A synchronous
 * ftsp_set_fields supersedes an upload that is not yet installed. */
int ftsp_set_fields_async(ftsp_handle* h, const double* omega, const double* psi);

/* Copies a named field to host memory as interleaved complex float64.
 * Names follow deviceState (deviceState.h:6-48): omega psi omega_bar psi_bar
 * drift drift_bar dpsi dpsi_bar rho_type rho_p rho_c rho_c_poly rho_c_ion
 * ion_rho W_type_s psi_s qF, and eta: the last step's real Langevin noise
 * (modes, then psi after its mean removal; imaginary parts zero).  *count
 * receives the number of doubles. */
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
 * cannot call cudaMalloc: code inside a framework whose caching allocator
 * owns the device memory (a second allocator beside it fragments the pool or
 * fails once the framework has reserved it), and loops that must not block
 * on the driver's allocator.  No counterpart in the reference.  No handle:
 * the mesh (m1..m3) and box lengths (L1..L3) are passed directly; w and
 * q_end are device arrays of m1*m2*m3 complex128 values; Q points to 2 host
 * doubles that receive mean(q_N) (real, imaginary).  All scratch (the
 * exp(-w) table, the intermediate field, the reduction partials and the FFT
 * and bond tables) lives in one static device array of about 8.3 MiB inside
 * the library, which every GPU that loads libftsp.so keeps until the process
 * exits.  Limits: at most 262144 grid points (64^3) and 256 points per axis;
 * larger meshes return FTSP_ERROR with the reason in ftsp_last_error(NULL).
 * The first call on a device looks the scratch address up with
 * cudaGetSymbolAddress.  The call is synchronous: it copies its small tables
 * from host memory into the array, runs on cuda_stream (NULL: the legacy
 * default stream), copies Q back to the host and waits for the stream before
 * returning.  Every call on a device shares the one array, tables included,
 * so calls from different host threads whose work overlaps on the GPU race
 * (even on tiny meshes): serialise them. */
int ftsp_propagate_chain_noalloc(int m1, int m2, int m3, double L1, double L2, double L3, const double* w, int N,
                                 double bond_length, double* q_end, double* Q, void* cuda_stream);

/* Number of checkpoint rollbacks taken so far (restart_interval > 0);
 * -1 on error.  Synchronises the handle's stream. */
long long ftsp_restart_count(ftsp_handle* h);

/* Time averages of the observable record on the device, following
 * complexLangevin::accumulate_observable_record / write_observable_average
 * (complexLangevin.cu:424-467): after ftsp_average_start, the record of a
 * step is accumulated when more than `skip` steps (the reference's Nss) have
 * been taken since the start, fewer than `samples` (Ns) records have been
 * accumulated and the step is finite; the real part of every entry, as the
 * reference averages and writes it.  With the adaptive step each record is
 * weighted by its dt_eff / dt.  The records are also grouped into `blocks`
 * consecutive blocks (no reference counterpart): ftsp_average_read returns
 * the mean over all accumulated records (mean[ftsp_record_length]), the
 * standard error from the means of the complete blocks (std_error[...],
 * NaN with fewer than two complete blocks) and the number of records
 * accumulated (*count).  Nothing is copied to the host during the steps, so
 * averaging runs inside the step graph and replica batches; start it before
 * ftsp_batch_create.  ftsp_average_start restarts the accumulation. */
int ftsp_average_start(ftsp_handle* h, int skip, long long samples, int blocks);
int ftsp_average_read(ftsp_handle* h, double* mean, double* std_error, long long* count);

/* Rollback state: *restarts as ftsp_restart_count; *exhausted = 1 once a
 * non-finite step found max_restarts rollbacks already taken.  From then on
 * nothing is restored and every step returns FTSP_NONFINITE, as the
 * reference's run ends with "maximum non-finite restarts exceeded"
 * (complexLangevin.cu:626-636), until ftsp_set_fields starts a new run
 * (which clears both).  Synchronises the handle's stream. */
int ftsp_rollback_info(ftsp_handle* h, long long* restarts, int* exhausted);

/* Time step of the following steps (the noise amplitude, the predictor and
 * corrector coefficients and the semi-implicit P(k) follow it).  No
 * reference counterpart: the reference reads dt once from the param file
 * (param.cu:228). */
int ftsp_set_dt(ftsp_handle* h, double dt);

/* Adaptive step (no reference counterpart).  u_ref > 0: every step uses
 * dt_eff = dt * min(1, u_ref / max|u|), max|u| being the largest drift
 * magnitude of any field at the start of the step, in the noise amplitude,
 * the predictor, the corrector and the semi-implicit P(k) (the adaptive step
 * size of Aarts, James, Seiler and Stamatescu, Phys. Lett. B 687 (2010) 154,
 * which suppresses complex-Langevin runaways).  u_ref = 0: off (the
 * default).  ftsp_step_info returns the last step's dt_eff and max|u|
 * (synchronises); time averages over adaptive steps are weighted by dt_eff. */
int ftsp_set_adaptive(ftsp_handle* h, double u_ref);
int ftsp_step_info(ftsp_handle* h, double* dt_eff, double* umax);

/* Mirror-symmetric chains (no reference counterpart; the reference always
 * runs both sweeps, polymer.cu:402-416).  For a species whose segment
 * classes and bonds read the same from both ends, q-dagger(s) = q(N-1-s),
 * so its densities and connectivity stress are pair products over the
 * stored forward propagators and their spectra and the backward sweep is
 * skipped.  on = 1 (the default) uses that path for every such species;
 * on = 0 runs both sweeps for all species.  Takes effect at the next
 * evaluation (capture batches after setting it).  *n_species (optional)
 * returns how many species take the pair path. */
int ftsp_set_chain_symmetry(ftsp_handle* h, int on, int* n_species);

/* Step as a CUDA graph (no reference counterpart).  on = 1 (the default):
 * ftsp_step / ftsp_step_async capture the step's kernels once and replay
 * the graph on the handle's stream (the step index, noise key, adaptive
 * scale and checkpoint schedule are read on the device, so each replay is
 * the next step, bit-identical to launching the kernels one by one).
 * Steps with noise from ftsp_set_noise, with profiling on, or with the
 * learned preconditioner collecting or in use launch directly; setters that
 * change the step (dt, adaptive, chain symmetry, seed, stream, learned
 * preconditioner) drop the captured graph.  on = 0: always launch directly. */
int ftsp_set_step_graph(ftsp_handle* h, int on);

/* Learned semi-implicit preconditioner (no reference counterpart; the
 * reference has no semi-implicit scheme).  A per-k-mode MLP (features
 * log(1+k^2), log(1+P_w(k)), log(1+P_psi(k)), N/50, lB, 10*salt; two tanh
 * layers of width 64; FP32) predicts the linear-response coefficient G_f(k)
 * = G_f^Debye(k) exp(z_f) of every Langevin field f (interaction modes, then
 * psi), which replaces the analytic Debye-function G(k) in
 * P(k) = 1/(1 + lambda dt G(k)).  Handles with scheme FTSP_SCHEME_SI and at
 * most 3 interaction modes only.
 *
 *   ftsp_learn_configure  allocates the statistics and the network (weights
 *                         from the seed);
 *   ftsp_learn_collect    while on, every step accumulates, per field and k,
 *                         <Re(du conj(dw))> and <|dw|^2> of the drift change
 *                         du = u(omega_bar) - u(omega) and the predictor
 *                         increment dw (the "force, field-increment" pairs),
 *                         and the running spectral powers; it may stay on
 *                         while the learned G(k) is in use (online training);
 *   ftsp_learn_reset      clears those statistics and the residual sums
 *                         (network and optimiser kept);
 *   ftsp_learn_train      runs `iterations` Adam steps (hand-written forward,
 *                         backward and update kernels) regressing z_f on
 *                         log(<Re(du dw*)> / (<|dw|^2> G^Debye)); *loss
 *                         receives the last batch's mean squared error;
 *                         the number of usable (finite, positive) targets
 *                         is in ftsp_learn_stats.valid_targets, and with no
 *                         usable target the call fails (FTSP_ERROR);
 *   ftsp_learn_use        while on, the SI update uses the learned G(k),
 *                         re-evaluated every refresh_every steps, except after
 *                         a step whose force residual sum_k |du - G dw|^2 with
 *                         the learned G exceeds fallback_ratio times the one
 *                         with the analytic G: the next step then uses the
 *                         analytic G (counted in ftsp_learn_stats). */
typedef struct ftsp_learn_config {
    double N, lB, salt;          /* system features: chain length, Bjerrum length, salt density */
    double lr;                   /* Adam step size (<= 0: 1e-3) */
    int batch;                   /* wave vectors per Adam step, rounded up to 128 (<= 0: 4096) */
    int refresh_every;           /* steps between re-evaluations of G(k) in use (<= 0: 100) */
    double fallback_ratio;       /* residual ratio that triggers the analytic kernel (<= 0: 1.5) */
    unsigned long long seed;     /* weight initialisation and batch sampling */
} ftsp_learn_config;
typedef struct ftsp_learn_stats {
    long long collected;         /* steps whose statistics were accumulated */
    long long checks, fallbacks; /* steps judged by the residual test; of those, analytic fallbacks */
    double residual_learned;     /* last step's force residuals */
    double residual_analytic;
    double residual_learned_sum; /* their sums over the steps since the last reset */
    double residual_analytic_sum;
    double loss;                 /* last training batch loss */
    int iterations;              /* Adam steps taken */
    int using_learned;           /* the next step uses the learned G(k) */
    int n_params;                /* network size in floats */
    long long valid_targets;     /* (wave vector, field) targets the last ftsp_learn_train
                                    could use: finite, positive statistics; with none
                                    it fails with FTSP_ERROR */
} ftsp_learn_stats;
int ftsp_learn_configure(ftsp_handle* h, const ftsp_learn_config* cfg);
int ftsp_learn_collect(ftsp_handle* h, int on);
int ftsp_learn_reset(ftsp_handle* h);
int ftsp_learn_train(ftsp_handle* h, int iterations, double* loss);
int ftsp_learn_use(ftsp_handle* h, int on);
int ftsp_learn_get_stats(ftsp_handle* h, ftsp_learn_stats* stats);
/* Network weights (layout W1[64][6] b1[64] W2[64][64] b2[64] W3[nout][64]
 * b3[nout]): get copies them out, set replaces them; *n is the float count
 * (pass out = NULL to query it). */
int ftsp_learn_get_weights(ftsp_handle* h, float* out, int* n);
int ftsp_learn_set_weights(ftsp_handle* h, const float* w, int n);
/* Loss and its gradient with respect to the weights, through the training
 * kernels, on caller samples: x [n][6] features, t and m [n][nout] targets and
 * target weights (loss = sum m (z - t)^2 / sum m).  For gradient checks. */
int ftsp_learn_grad(ftsp_handle* h, const float* x, const float* t, const float* m, int n, double* loss, float* grad);

/* Launch geometry chosen for the handle's grid (autotune = 1): FFT radix
 * cap, strided tile width, how many alternatives were timed and the time of
 * one forward + inverse 3-D transform with the chosen and with the default
 * geometry.  compile_time = 1: every pass of this grid is a compile-time
 * kernel and nothing was tuned.  No reference counterpart. */
typedef struct ftsp_tune_info {
    int tuned, cached, compile_time;
    int max_radix, tile_width, candidates;
    double best_ms, default_ms;
} ftsp_tune_info;
int ftsp_tune_info_get(ftsp_handle* h, ftsp_tune_info* info);

/* Replica batches (no reference counterpart: the reference runs one system
 * per process).  ftsp_batch_create captures steps_per_graph steps of every
 * handle into one CUDA graph, each handle on its own branch stream, so the
 * kernels of independent replicas run concurrently and a batch step is one
 * graph launch.  The handles keep their state and can be read with
 * ftsp_read_status / ftsp_get_field after ftsp_batch_sync; they must not be
 * stepped on their own while the batch exists (they run on the batch's
 * branch streams until ftsp_batch_destroy gives them back their streams).
 * The noise index and the checkpoint schedule advance on the device, so
 * every replay takes fresh noise.  Settings that the step reads on the host
 * (dt, the learned-preconditioner mode) are fixed at capture time. */
typedef struct ftsp_batch ftsp_batch;
int ftsp_batch_create(ftsp_handle* const* handles, int n, int steps_per_graph, ftsp_batch** out);
int ftsp_batch_step(ftsp_batch* b, int graph_launches);       /* asynchronous */
int ftsp_batch_sync(ftsp_batch* b);
void* ftsp_batch_stream(ftsp_batch* b);                       /* the stream the graph runs on */
long long ftsp_batch_launch_count(const ftsp_batch* b);       /* kernels per graph launch */
const char* ftsp_batch_last_error(const ftsp_batch* b);       /* NULL: errors of ftsp_batch_create */
void ftsp_batch_destroy(ftsp_batch* b);

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
