/* Host front end of libftsp: the reference's input files and its step loop.
 *
 * These entry points replace the reference's host program (main.cu:9-93):
 * the param / sequence file readers (param.cu:165-334, polymer.cu:219-273),
 * the interaction-mode and ion setup (interactionMode.cu:9-263, ion.cu:3-46),
 * the field-file I/O (fieldIO.cu) and the step loop with its outputs and
 * non-finite restarts (complexLangevin.cu:191-230, 345-698).  The compute
 * underneath is the ftsp.h engine.
 *
 * Errors: functions return FTSP_OK / FTSP_ERROR; the message of a failed
 * call is returned by ftsp_last_error(NULL) on the calling thread. */
#ifndef FTSP_HOST_H
#define FTSP_HOST_H

#include "ftsp.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ftsp_model ftsp_model;

/* Reads the param file and its sequence file (sequence_file overrides the
 * param file's [polymer] sequence_file when not NULL), derives the
 * interaction modes, mobilities, ions and the short-range self pressure, and
 * validates the result: param::read + polymerSpecies::setup +
 * param::validate + ion::build (main.cu:16-27). */
int ftsp_model_load(const char* param_file, const char* sequence_file, ftsp_model** out);
void ftsp_model_free(ftsp_model* m);

/* Fills an engine configuration from the model; its arrays point into the
 * model, which must outlive the config.  precision, scheme, seed, device and
 * restart_interval are left at zero for the caller to set; max_restarts is
 * the param file's max_nan_restarts. */
int ftsp_model_config(ftsp_model* m, ftsp_config* cfg);

/* Scalar facts of a loaded model (no reference function; the reference
 * prints them with param::print, param.cu:503-567). */
typedef struct ftsp_model_info {
    int m1, m2, m3;
    int M;                  /* monomer types */
    int n_modes;            /* active interaction modes */
    int n_species, n_ions;
    int Nt, Nss, Ns, Ntmp, Nso, N_stat, max_nan_restarts;
    int noise;
    int legacy_ab;          /* omega files in the legacy A/B column order */
    double rho0, volume, self_pressure, eigen_tol_abs;
    long long total_segments;
} ftsp_model_info;
int ftsp_model_get_info(const ftsp_model* m, ftsp_model_info* info);

/* Eigenvalues (all M, descending) and eigenvectors O[l][alpha] (M x M,
 * row-major by mode) of K = xi + chi (interactionMode.cu:196-243). */
int ftsp_model_modes(const ftsp_model* m, double* eig, double* O);

/* Initial fields as the reference program reads them (main.cu:65-71,
 * fieldIO::read_omega_fields and read_psi_field, fieldIO.cu:432-520):
 * header-less files get their mesh inferred (a cube, or the model mesh
 * scaled by an integer factor), other meshes are resampled trilinearly, a
 * missing default "omega.rf" or a missing psi file gives zero fields, and in
 * the legacy A/B order the columns map to the composition-like and
 * density-like modes.  NULL names take the param file's omega_file /
 * psi_file.  omega: n_modes * V complex values; psi: V complex values (zero
 * when lB = 0).  The psi mean is not removed here (the engine does it). */
int ftsp_model_read_fields(const ftsp_model* m, const char* omega_file, const char* psi_file, double* omega, double* psi);

/* Field writers in the reference's .rf format (fieldIO.cu:409-430, 553-575):
 * "m1 m2 m3", "L1 L2 L3" (%.17g), then one row per point with "%.10f  %.10f"
 * per field.  ftsp_model_write_omega writes the omega fields in the model's
 * file order (legacy A/B or active modes); ftsp_model_write_fields writes
 * `count` fields of V complex values, field-major. */
int ftsp_model_write_omega(const ftsp_model* m, const char* file, const double* omega);
int ftsp_model_write_fields(const ftsp_model* m, const char* file, int count, const double* fields);

/* The reference program: `ftsp_main(argc, argv)` takes the reference's
 * command line (-p param, -i id, -s dir, --omega, --psi, --seq,
 * --screenprint) plus --fp32/--fp64, --si/--pc, --seed N and --device N, runs
 * the Nt steps with the reference's outputs (observables file with its
 * ensemble average, drift_max file, tmp checkpoints every Ntmp steps,
 * restarts from them on non-finite values, step outputs, final fields and
 * densities) and returns the process exit status (0 on success). */
int ftsp_main(int argc, char** argv);

#ifdef __cplusplus
}
#endif
#endif
