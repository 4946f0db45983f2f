/*
 * pwgpu_deck.h -- the reference's YAML input deck read inside the library.
 *
 * InputSettings::from_yaml_str (pwdft-core/src/settings.rs:27-511): the
 * blocks system / basis / kpoints / scf / electrons / xc / symmetry /
 * output / initial_density, unknown fields refused at every level
 * (deny_unknown_fields), `system` and `kpoints` required, every other field
 * defaulted as the reference defaults it. Plain scalars are typed by the
 * YAML 1.2 core rules of the reference's reader (serde_yaml_ng 0.10): an
 * exponent without a dot is a float, only true/false are booleans, ~ and
 * null are null, 0x / 0o / 0b prefix integers, digits with a leading zero
 * are strings. The reader takes the block and flow forms decks are written
 * in; anchors, aliases, tags, block scalars and multi-document streams are
 * refused. A deck that does not parse, or breaks the schema, returns
 * PWGPU_E_PARSE with the reason in pwgpu_last_error(); a custom k-grid
 * shift flag above 1 is PWGPU_E_INVALID (InvalidParam). Parameter checks
 * (ScfParams::validate, scf/mod.rs:166-225) are not part of parsing, as in
 * the reference.
 */
#ifndef PWGPU_DECK_H
#define PWGPU_DECK_H

#include "pwgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pwgpu_deck pwgpu_deck;

#define PWGPU_KPOINTS_MONKHORST_PACK 0
#define PWGPU_KPOINTS_BAND_PATH 1

/* The scalar settings of a deck, defaults filled in. Enumerations by their
 * position in the reference's variant lists:
 *   eigensolver  0 dense, 1 iterative
 *   mixing_mode  0 plain, 1 kerker, 2 broyden, 3 broyden_kerker,
 *                4 periodic_pulay, 5 periodic_pulay_kerker
 *                (= pwgpu_scf_params.mixing_mode)
 *   smearing     pwgpu_scf_params.smearing (0 fermi_dirac, 1 gaussian,
 *                2 methfessel_paxton, 3 cold, 4 fixed)
 *   occupations  0 smearing, 1 fixed
 *   functional   0 pz, 1 pbe, 2 pbe0, 3 hse06
 *   verbosity    0 low, 1 normal, 2 high */
typedef struct pwgpu_deck_settings {
  double lattice[9];          /* rows a, b, c, Å */
  int32_t n_atoms;
  double ecutwfc;             /* eV */
  int32_t ecutrho_ratio;
  int32_t fft_grid[3];        /* 0 0 0: chosen from the cutoff */
  int32_t kpoints_type;       /* PWGPU_KPOINTS_* */
  int32_t mp_grid[3];
  int32_t mp_shift[3];        /* half-shift flags: gamma_centered 0 0 0, mp1976 1 1 1, custom */
  int32_t n_path;             /* band_path points */
  int32_t band_npoints;
  int32_t max_iter;
  double conv_threshold;
  double energy_threshold;
  int32_t n_bands;            /* -1: not given (the driver's fallback applies) */
  int32_t eigensolver;
  int32_t wfrx_subspace;
  double mixing_beta;
  int32_t mixing_ndim;
  int32_t mixing_mode;
  int32_t pulay_period;
  int32_t adaptive_beta;
  int32_t smearing;
  double smearing_width;      /* eV */
  int32_t spin_polarized;
  int32_t n_starting_magnetization;
  int32_t has_tot_magnetization;
  double tot_magnetization;
  int32_t occupations;
  int32_t functional;
  int32_t symmetry_enabled;
  int32_t time_reversal;
  double symmetry_tolerance;
  int32_t verbosity;
  int32_t write_density;
  int32_t write_bands;
  double gaussian_sigma;      /* Å, initial_density.gaussian_sigma */
} pwgpu_deck_settings;

/* Parse len bytes of deck text; *out is freed with pwgpu_deck_free. */
pwgpu_status pwgpu_deck_parse(const char* text, int64_t len, pwgpu_deck** out);
pwgpu_status pwgpu_deck_get_settings(const pwgpu_deck* d, pwgpu_deck_settings* s);
/* Atoms in deck order: symbols n_atoms x 8 chars (NUL-terminated),
 * positions n_atoms x 3 fractional coordinates. */
pwgpu_status pwgpu_deck_get_atoms(const pwgpu_deck* d, char* symbols, double* positions);
/* electrons.starting_magnetization in deck order: symbols n x 8 chars,
 * values n doubles (n = n_starting_magnetization). */
pwgpu_status pwgpu_deck_get_starting_magnetization(const pwgpu_deck* d, char* symbols, double* values);
/* kpoints.path of a band_path deck: labels n_path x 16 chars, fractional
 * coordinates n_path x 3. */
pwgpu_status pwgpu_deck_get_band_path(const pwgpu_deck* d, char* labels, double* frac);
/* Free a parsed deck (NULL is a no-op). */
pwgpu_status pwgpu_deck_free(pwgpu_deck* d);

#ifdef __cplusplus
}
#endif

#endif /* PWGPU_DECK_H */
