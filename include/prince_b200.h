/*
 * prince_b200 -- C ABI of the B200-native ETD2 propagation core.
 *
 * Plain C types only (pointers, sizes, one POD struct); no torch types.  All
 * functions return PB_OK (0) on success or a PB_ERR_* code; the message of the
 * last failure is available from pb_last_error(ctx) (pb_global_error() for
 * failures of pb_create).  Host pointers are read during the call only.
 *
 * Each entry point names the reference interface it replaces (paths inside
 * the PriNCe project).  The reference's ETD2 path is Python, so there is no
 * reference C ABI; the Python binding in prince_b200/_lib.py is the layer a
 * reference backend would call.
 *
 * Threading: a context is used by one host thread at a time; all device work
 * of a context runs on the context's own stream.
 */
#ifndef PRINCE_B200_H
#define PRINCE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PB_OK 0
#define PB_ERR_ARG 1    /* invalid argument                       -> ValueError   */
#define PB_ERR_STATE 2  /* missing set-up / wrong call order       -> RuntimeError */
#define PB_ERR_CUDA 3   /* CUDA runtime failure                    -> RuntimeError */
#define PB_ERR_DEVICE 4 /* device-side status (timeout, non-finite) -> RuntimeError */

/* Solve flags: the solver enable switches of
 * UHECRPropagationSolver.__init__ (src/prince_cr/solvers/propagation.py:196-209). */
#define PB_ADIABATIC 1u     /* enable_adiabatic_losses      */
#define PB_PAIRPROD 2u      /* enable_pairprod_losses       */
#define PB_PHOTOHAD 4u      /* enable_photohad_losses       */
#define PB_INJECTION 8u     /* enable_injection_jacobian    */
#define PB_PARTIAL_DIFF 16u /* enable_partial_diff_jacobian */
#define PB_DECAY 32u        /* enable_decay (explicit Lambda operator) */
#define PB_EM_CASCADE 64u   /* co-evolved EM cascade (run.enable_em_cascade) */

/* pb_set_option / pb_get_info keys */
#define PB_OPT_BATCHED_KERNELS 1 /* 1 (default): bin-blocked kernels for K > 1 when the layout allows; 0: row kernels */
#define PB_INFO_BLOCKED_LAYOUT 2 /* 1 if pb_set_layout found a pattern the bin-blocked kernels handle */
#define PB_INFO_LAST_BLOCKED 3   /* 1 if the last pb_solve ran the bin-blocked kernels */
#define PB_INFO_BAND_SPECIES 4   /* species whose coupling rows leave their energy bin */
#define PB_INFO_BAND_ENTRIES 5   /* off-diagonal coupling entries of the band rows */
#define PB_INFO_SLAB_ENTRIES 6   /* off-diagonal coupling entries of the bin-local rows */
#define PB_INFO_SLAB_ROWS 7      /* bin-local rows */
#define PB_INFO_FD_DENSE 8       /* 1 if the forward FD term runs the register-blocked dense stencil */
#define PB_OPT_TMA_STAGING 9     /* 1 (default): the bin-local and band-tile kernels stage by TMA (tensor maps,
                                    bulk copies); 0: cp.async */
#define PB_INFO_LAST_TMA 10      /* 1 if the last pb_solve staged the bin-local kernel by TMA */
#define PB_OPT_BAND_WARPS 12       /* warps of a band-tile CTA: 8 (default, 64 columns, one CTA per SM) or 4
                                     (32 columns in half the registers and shared memory, so the band
                                     tiles run on the tensor pipe beside the bin-local gather on each SM) */
#define PB_OPT_SLAB_PREFETCH 13    /* row quartets whose FD term and F(x) a bin-local warp loads ahead: 1, 2 (default), 3 */
#define PB_OPT_STAGING_WAIT_TRIES 11 /* polls of k_slab's bounded staging wait before it gives up and the solve
                                     returns PB_ERR_DEVICE (default 2^24; < 0 restores it; 0 gives up at
                                     once, which tests the error path). The CTA still drains its copies. */

typedef struct pb_context pb_context;

/* Version of this ABI (bumped on any signature change). */
int pb_abi_version(void);

/* Create a context on CUDA device `device` (own stream, own device buffers).
 * Replaces: the per-solver backend state of ETD2SolverCUPY.__init__
 * (src/prince_cr/solvers/propagation.py:1595-1700). */
int pb_create(int device, pb_context** out);

/* Free every device buffer of the context.  Replaces ETD2Solver*.close()
 * (propagation.py:708-716, 970-978). */
void pb_destroy(pb_context* ctx);

const char* pb_last_error(const pb_context* ctx);
const char* pb_global_error(void);

/* Fixed CSR pattern of the coupling matrix M (n_states x n_states, n_entries
 * entries, rows sorted, columns sorted within rows).  Entry i of the pattern
 * is row i of the fold kernel.
 * Replaces: PhotoNuclearInteractionRate._init_coupling_mat
 * (src/prince_cr/interaction_rates.py:648-697). */
int pb_set_coupling(pb_context* ctx, int64_t n_states, int64_t n_entries,
                    const int64_t* indptr, const int32_t* indices);

/* Dense FP64 fold kernel, row-major (n_entries x n_photon), rows in CSR order.
 * Replaces: PhotoNuclearInteractionRate._batch_matrix
 * (interaction_rates.py:186-188, 629-631, 681) and the GPU mirror of
 * _ensure_coupling_mat_gpu (interaction_rates.py:852-928). */
int pb_set_fold_kernel(pb_context* ctx, int64_t n_entries, int32_t n_photon,
                       const double* kernel);

/* The fold kernel built on the device from per-channel response samples,
 * replacing pb_set_fold_kernel (no host kernel, no kernel upload).  With d
 * cosmic-ray bins per species block, dph photon bins, na = d + dph - 1 and
 * nb = 2 d - 1, entry e of the coupling pattern (daughter state r, mother
 * state c, mother bin i = c mod d, daughter bin k = r mod d) gets, for each
 * photon bin j and its channel q = entry_channel[e] = (kind, p1, p2, -):
 *   kind 0 (boost-conserving / non-elastic): 0 + f_i resp[p1][i+j] - f_i resp[p2][i+j]
 *          (a term is absent when its index is -1);
 *   kind 1 (redistributed, full table):      max(g_ik ddr[p1][i+j][k-i+d-1], 0)
 *   kind 2 (redistributed, outer product):   max(g_ik sep_a[p1][i+j] sep_b[p1][k-i+d-1], 0)
 *          minus f_i resp[p2][i+j] on the diagonal i = k when p2 >= 0;
 * f_i = f_mo[i] (m_p / E_i), g_ik = f_i (dE[i] / dE[k]).  Arrays are row-major
 * FP64 on the host; entry_channel has one value per coupling entry in CSR
 * order.  Needs pb_set_coupling.  Replaces: the Toeplitz assembly of
 * PhotoNuclearInteractionRate._init_matrices (src/prince_cr/interaction_rates.py:251-646),
 * given its sampled response increments (nonel_dR, incl_dR, diff_ddR). */
typedef struct pb_kernel_spec {
  int32_t d, dph;
  const double* f_mo;            /* d */
  const double* dE;              /* d */
  int32_t n_resp;
  const double* resp;            /* n_resp x na */
  int32_t n_ddr;
  const double* ddr;             /* n_ddr x na x nb */
  int32_t n_sep;
  const double* sep_a;           /* n_sep x na */
  const double* sep_b;           /* n_sep x nb */
  int32_t n_channels;
  const int32_t* channels;       /* n_channels x 4: kind, p1, p2, unused */
  const int32_t* entry_channel;  /* one per coupling entry, CSR order */
} pb_kernel_spec;
int pb_build_fold_kernel(pb_context* ctx, const pb_kernel_spec* spec);

/* Copies the device fold kernel (R x dph, coupling-CSR order) to the host.
 * No counterpart in the reference (its kernel lives on the host); exposed so
 * a device-built kernel can be checked or saved. */
int pb_get_fold_kernel(pb_context* ctx, int64_t n_entries, int32_t n_photon, double* kernel);

/* Photon-grid bin centres (n_photon) at which the fold samples n(E, z).
 * Replaces: the ph_grid.grid argument of photon_vector (interaction_rates.py:105-116). */
int pb_set_photon_grid(pb_context* ctx, int32_t n_photon, const double* energies);

/* Photon field: the sum of n_comp components, kinds[i] in {0: CMB black body,
 * 1: flat, 2: grey body, 3: the tabulated field of pb_set_photon_table},
 * params[3*i .. 3*i+2] = (p0, p1, p2) as documented in
 * prince_b200/photonfields.py (ignored for kind 3).  Replaces:
 * PhotonField.get_photon_density for the analytic fields and their sums
 * (src/prince_cr/photonfields.py:27-127). */
int pb_set_photon_field(pb_context* ctx, int32_t n_comp, const int32_t* kinds,
                        const double* params);

/* Tabulated photon field for kind 3: log10 dn/de [GeV^-1 cm^-3] on a regular
 * grid of nz increasing redshifts and ne increasing log10 energies [GeV]
 * (log10_density is nz x ne, row-major), interpolated bilinearly in
 * (z, log10 E) and zero outside the table.  Replaces: the corrected
 * tabulated EBL models CIBGilmore2012 / CIBFranceschini2008 and their
 * RegularGridInterpolator (src/prince_cr/photonfields.py:227-345), used by the
 * rate fold's photon vector and by the Bethe-Heitler loss
 * (interaction_rates.py:1296-1312). */
int pb_set_photon_table(pb_context* ctx, int32_t nz, int32_t ne, const double* z, const double* log10_e,
                        const double* log10_density);

/* Finite-difference loss operator split into its off-diagonal CSR part
 * (D_off, nnz entries) and its diagonal (n_states).
 * Replaces: DifferentialOperator.operator + _ensure_D_split
 * (src/prince_cr/solvers/partial_diff.py:28-110; propagation.py:1122-1146). */
int pb_set_fd_operator(pb_context* ctx, int64_t nnz, const int64_t* indptr,
                       const int32_t* indices, const double* values, const double* diag);

/* Continuous-loss inputs:
 *   adia_energy (n_states)  energy_vector of ContinuousAdiabaticLossRate
 *                           (interaction_rates.py:1194-1224);
 *   pair_scale (n_states)   scale_vec of ContinuousPairProductionLossRate;
 *   pair_bin (n_states)     cosmic-ray bin of each state on nucleus blocks, -1 elsewhere;
 *   xi (n_xi), phi_xi2 (n_xi), pair_photon_grid (n_cr_bins x n_xi): the
 *                           integration grid of loss_vector (interaction_rates.py:1238-1312). */
int pb_set_losses(pb_context* ctx, const double* adia_energy, const double* pair_scale,
                  const int32_t* pair_bin, int32_t n_cr_bins, int32_t n_xi,
                  const double* xi, const double* phi_xi2, const double* pair_photon_grid);

/* Constant explicit-decay operator: diagonal (n_states, may be NULL) and
 * off-diagonal CSR (nnz may be 0).  Replaces: _ensure_Lambda_split
 * (propagation.py:1148-1358). */
int pb_set_decay(pb_context* ctx, const double* diag, int64_t nnz, const int64_t* indptr,
                 const int32_t* indices, const double* values);

/* Injection basis: n_src source grids restricted to the n_rows state rows on
 * which any of them is non-zero.  rows (n_rows) lists those states; grids is
 * row-major (n_rows x n_src).  Source s feeds column src_col[s] (non-decreasing).
 * Replaces: the injection_grid arrays of CosmicRaySource
 * (src/prince_cr/cr_sources.py:32-48) consumed by injection()
 * (propagation.py:363-370, 2476-2488). */
int pb_set_injection(pb_context* ctx, int32_t n_src, int32_t n_rows, const int32_t* rows,
                     const double* grids, int32_t n_cols, const int32_t* src_col);

/* State layout: species blocks of d energy bins (n = n_species * d), the
 * SpeciesManager layout on a shared grid (src/prince_cr/data.py:1385-1450).
 * Classifies the coupling rows into
 * bin-local rows and band rows for the bin-blocked batched kernels.  No
 * reference counterpart (the reference multiplies the whole CSR operator). */
int pb_set_layout(pb_context* ctx, int32_t d);

/* The same with species blocks only in rows [0, n_blocks) (n_blocks a multiple
 * of d); rows [n_blocks, n) form a tail of species on another grid (gamma and
 * e+- on a decoupled EM grid, src/prince_cr/core.py:105-137, 206-214) that the
 * general row kernel steps beside the bin-blocked kernels.  The fold kernel's
 * coupling entries must lie inside the blocks; with coupling entries between
 * blocks and tail the general row kernels step everything. */
int pb_set_layout_rows(pb_context* ctx, int32_t d, int64_t n_blocks);

/* The caller's row order of the state: device row i holds the caller's row
 * caller_row[i] (a permutation of [0, n)).  pb_solve's state and pb_adjoint's
 * seed are read and written in the caller's order; every other per-row input
 * (coupling, losses, injection rows, EM offsets) is in the device order.  NULL
 * restores the identity; pb_set_coupling resets it.  No reference counterpart
 * (the reference keeps the species layout, where the EM species come first;
 * the device puts the species blocks of the shared grid first). */
int pb_set_row_map(pb_context* ctx, const int32_t* caller_row);

/* Execution options (PB_OPT_*) and read-only facts (PB_INFO_*) of a context.
 * No reference counterpart. */
int pb_set_option(pb_context* ctx, int32_t key, int64_t value);
int pb_get_info(pb_context* ctx, int32_t key, int64_t* value);

/* Measurement aid: re-runs the bin-blocked kernels of one stage (1 or 2) of
 * step `step` of the last solve, each kernel alone between CUDA events on the
 * context's stream, and returns the mean of `reps` launches in milliseconds:
 * ms[0] FD term, ms[1] bin-local rows, ms[2] band partial sums, ms[3] band
 * rows (0 for a kernel the stage does not run).  Overwrites the stage's
 * output buffers.  No reference counterpart. */
int pb_profile_stage(pb_context* ctx, int64_t step, int32_t stage, int32_t reps, double* ms);

/* Measured FP64 tensor-pipe (DMMA) throughput of the device in TFLOP/s, from a
 * register-only kernel on every SM.  No reference counterpart. */
int pb_fp64_peak(pb_context* ctx, double* tflops);

/* Co-evolved EM cascade layout: the gamma block (n_em states from gamma_off),
 * the e- and e+ blocks (offsets, -1 if absent), and the charged nuclei whose
 * Bethe-Heitler losses feed the pairs: n_bh blocks of n_cr states from
 * bh_off[s] with mass numbers bh_A[s]; inv_E (1/E) and dE (numpy.gradient of
 * E) on that nucleon grid.  Replaces: the EM attributes set in
 * UHECRPropagationSolver.__init__ (src/prince_cr/solvers/propagation.py:270-305). */
int pb_set_em(pb_context* ctx, int32_t n_em, int64_t gamma_off, int64_t em_off, int64_t ep_off,
              int32_t n_cr, int32_t n_bh, const int64_t* bh_off, const double* bh_A,
              const double* inv_E, const double* dE);

/* Per-window EM-cascade data of the next solve: T_gamma and T_electron
 * (n_windows x n_em x n_em), R_BH (n_windows x n_em x n_cr), row-major, and
 * dl_step = c |dz| / ((1+z) H(z)) at each window.  Applied after every step
 * (propagation.py:555-665: _inject_bh_pairs then _apply_em_cascade). */
int pb_set_em_windows(pb_context* ctx, int32_t n_windows, const double* Tg, const double* Te,
                      const double* R, const double* dl_step);

/* Kinetic EM-cascade transfer built on the device for the context's photon
 * field (times photon_scale): per redshift z[q] the photon transfer T_gamma
 * and the electron transfer T_electron (n x n each, row-major, written to
 * n_z x n x n host arrays) of the EM grid E (n increasing bin centres, GeV),
 * with per-step escape over dl_step[q] = c |dz| / ((1+z) H(z)) [cm].  eps is
 * the target grid of the inverse-Compton and pair kernels, eps_o / mu the
 * grids of the gamma-gamma opacity, n_E1 the points of the per-electron
 * IC-loss grid; m_electron [GeV], r_electron [cm] and c_cm [cm/s] are the
 * caller's unit constants.  Field-free kernels, their contractions with the
 * photon stacks (FP64 tensor-core GEMMs), the per-redshift matrices and the
 * scattering iteration (at most max_scatter passes, each redshift stopping
 * when the energy left in the box falls below tol of what entered) all run on
 * the device, in FP64.  *iterations (if given) receives the passes run.
 * Replaces: kinetic_cascade_transfer_batched (src/prince_cr/cascade/cascade.py:444-589),
 * with its kernels (cascade.py:78-171, 425-441; kernels.py:68-75; opacity.py:44-75)
 * and an FP64 iteration. */
typedef struct pb_em_transfer_args {
  int32_t n;
  const double* E;
  int32_t n_z;
  const double* z;
  const double* dl_step;
  int32_t n_eps;
  const double* eps;
  int32_t n_eps_o;
  const double* eps_o;
  int32_t n_mu;
  const double* mu;
  int32_t n_E1;
  double photon_scale;
  double cool_floor_frac;
  int32_t max_scatter;
  double tol;
  double m_electron, r_electron, c_cm;
  double* T_gamma;
  double* T_electron;
  int32_t* iterations;
} pb_em_transfer_args;
int pb_em_transfer(pb_context* ctx, const pb_em_transfer_args* args);

/* Bethe-Heitler e+- pair shape built on the device for the context's photon
 * field (times photon_scale): per redshift z[q] the matrix R (n_e x n_p,
 * row-major, written to n_z x n_e x n_p host memory): the one-sign lepton
 * spectrum dN/dE_e at E_e[i] (GeV) of a nucleon at E_p[j], from the
 * differential Born cross section integrated by nested fourth-order rules
 * into a field-free kernel on the target grid eps, contracted with the photon
 * density over ln eps (points with positive density), restricted to
 * 1e-6 E_p < E_e <= E_p and E_p >= e_p_min, and normalised so the pair
 * carries E_p[j].  m_electron, m_proton [GeV] are the caller's constants.
 * Replaces: bh_pair_shape_matrix with its kernel tensor
 * (src/prince_cr/cascade/bethe_heitler.py:27-297), as the solver's
 * _em_bh_at builds it (src/prince_cr/solvers/propagation.py:573-618). */
typedef struct pb_bh_shape_args {
  int32_t n_e;
  const double* E_e;
  int32_t n_p;
  const double* E_p;
  int32_t n_eps;
  const double* eps;
  int32_t n_z;
  const double* z;
  double photon_scale;
  double e_p_min;
  double m_electron, m_proton;
  double* R;
} pb_bh_shape_args;
int pb_bh_shape(pb_context* ctx, const pb_bh_shape_args* args);

/* One solve: the redshift stepping of UHECRPropagationSolverETD2.solve /
 * MultiRHSPropagationSolverETD2.solve (propagation.py:813-890; etd2.py:478-517;
 * _operator_at / apply_F propagation.py:1360-1508; multi-RHS 2495-2618).
 * All per-step scalars are evaluated by the caller in float64 exactly as the
 * reference does (z grid, window schedule, dl/dz, H(z) cm2sec, injection
 * prefactor dl/dz * cm2sec, source evolution); the device computes the
 * photon field, the pair-loss vectors, the fold, the operator split and every
 * ETD2 step. */
typedef struct pb_solve_args {
  int64_t n_steps;
  int32_t n_windows;
  int32_t n_cols;          /* K: state columns (1 for the single-RHS solver)        */
  uint32_t flags;          /* PB_* solve flags                                       */
  double photon_scale;     /* multiplies the photon field (1.0 nominal)             */
  const double* z_window;  /* n_windows: redshift of each rate-cache refresh       */
  const int32_t* window;   /* n_steps: window index of each step                    */
  const double* h;         /* n_steps: z[k+1] - z[k]                                 */
  const double* dldz;      /* n_steps: dl/dz at z[k]                                 */
  const double* hc;        /* n_steps: H(z[k]) * cm2sec (adiabatic loss scale)       */
  const double* finj;      /* n_steps: dl/dz(z[k]) * 1.0 * cm2sec (injection factor) */
  const double* coeff;     /* n_steps x n_src: norm * evolution(z[k]) per source     */
  const int32_t* n_active; /* n_steps: columns [0, n_active) may be non-zero; the
                              rest are exactly zero (sources not yet switched on)  */
  double* state;           /* n_states x n_cols row-major: in = initial state (if
                              init_state != 0), out = state at the final redshift  */
  int32_t init_state;      /* 0: start from zeros                                    */
  int32_t state_on_device; /* 1: `state` is a device pointer                         */
  int32_t ckpt_every;      /* > 0: keep the state every this many steps for pb_adjoint */
  const int32_t* out_cols; /* NULL, or n_cols: output column of each solve column (a
                              permutation); the final states are gathered on the
                              device into that order, and pb_adjoint reads its
                              seed in that order.  The initial state is read in
                              solve-column order. */
} pb_solve_args;

int pb_solve(pb_context* ctx, const pb_solve_args* args);

/* Autotuner of the batched bin-blocked stage: runs the solve described by
 * `args` (normally a short schedule with every column active, on the live
 * operator, injection and photon field) `reps` + 1 times for each candidate
 * (band-tile CTA warps 8 / 4, k_slab prefetch depth 2 / 3 / 4, k_slab staging
 * by TMA / cp.async), scores each by its fastest step loop, and leaves the
 * fastest set on the context (the PB_OPT_BAND_WARPS, PB_OPT_SLAB_PREFETCH and
 * PB_OPT_TMA_STAGING options).  Writes up to max_out candidates to out, the
 * chosen one first, and their count to n_out.  `args->state` receives the
 * short solve's states.  Replaces: the fixed K-dependent multi-RHS tile
 * choices of the reference's batched path (src/prince_cr/solvers/propagation.py:2375-2391),
 * which has no tuner of its own. */
typedef struct pb_tune_choice {
  int32_t band_warps, slab_prefetch, tma_staging;
  double steps_ms;   /* fastest step loop of the candidate's runs; 1e300 if it could not run */
} pb_tune_choice;
int pb_autotune(pb_context* ctx, const pb_solve_args* args, int32_t reps, int32_t max_out,
                pb_tune_choice* out, int32_t* n_out);

/* Discrete adjoint of the last solve: gradients of L = sum(seed * x_final) with
 * respect to the injection grids (n_rows x n_src, as passed to pb_set_injection),
 * the per-step source coefficients (n_steps x n_src) and the photon scale
 * (one value per column; the scale enters both the rate fold and kappa_pair).
 * `args` must be the arguments of that solve, which must have set ckpt_every:
 * the state is recomputed from the checkpoints segment by segment and the
 * ETD2 step is reversed with the transposed operator
 * (A^T = dl/dz (M_off^T + diag(kappa) D_off^T + Lambda_off^T)).  Any gradient
 * pointer may be NULL (no scale gradient: no scale recording).
 * Replaces: finite differences of the reference solver (no adjoint exists in
 * the reference; the forward it differentiates is etd2.py:412-439 with
 * propagation.py:1360-1508). */
int pb_adjoint(pb_context* ctx, const pb_solve_args* args, const double* seed, int32_t seed_on_device,
               double* grad_grids, double* grad_coeff, double* grad_scale);

/* Inspection after a solve: the off-diagonal operator pattern built from the
 * first window (split_operator + eliminate_zeros, src/prince_cr/solvers/etd2.py:234-268).
 * Call with indptr/indices NULL to query nnz. */
int pb_get_operator_pattern(pb_context* ctx, int64_t* nnz, int64_t* indptr, int32_t* indices);

/* Per-window operator values of the last solve: M_off.data (nnz), the
 * diagonal of M (n_states) and kappa_pair (n_states); any pointer may be NULL. */
int pb_get_window(pb_context* ctx, int32_t window, double* offdiag, double* diag,
                  double* kappa_pair);

/* ETD2 with a z-independent operator: d (n) diagonal, L_off CSR, no losses,
 * no injection, state (n) advanced in place along z_grid (n_steps + 1).
 * Replaces: etd2.integrate driven by a constant operator_at closure
 * (src/prince_cr/solvers/etd2.py:478-517; tests/test_explicit_decay_analytics.py:43-62). */
int pb_integrate_const(pb_context* ctx, int64_t n, const double* d, int64_t nnz,
                       const int64_t* indptr, const int32_t* indices, const double* values,
                       int64_t n_steps, const double* z_grid, double* state);

/* Limits of the static scratch used by pb_integrate_const_noalloc. */
#define PB_NOALLOC_MAX_STATES 65536
#define PB_NOALLOC_MAX_STEPS 16384

/* pb_integrate_const for callers that cannot allocate device memory: code
 * running inside another framework's custom-call or FFI handler, which may
 * only use the buffers it is handed, and hosts that reserved all device memory
 * up front, where a cudaMalloc would fail or take memory the host already
 * promised elsewhere.  No counterpart in the reference (its solvers allocate
 * freely).
 *
 * Every pointer is a DEVICE pointer owned by the caller: d (n), the CSR arrays
 * of L_off (indptr n + 1 int64, indices and values nnz each; indptr may be
 * NULL when nnz == 0), z_grid (n_steps + 1) and state (n, advanced in place).
 * Before any step, a check kernel verifies that indptr[0] = 0, that indptr
 * never decreases, that indptr[n] = nnz and that every column index lies in
 * [0, n); a malformed CSR is rejected with PB_ERR_ARG and nothing else runs.
 * The buffers themselves must hold the sizes above: the library cannot check
 * a device allocation's extent.
 *
 * The call allocates and frees nothing: its scratch (about 6 MB) is one static
 * device array sized for at most PB_NOALLOC_MAX_STATES states and
 * PB_NOALLOC_MAX_STEPS steps; larger sizes are rejected with PB_ERR_ARG.  Every
 * GPU that loads the library holds that array until the process exits.
 *
 * The first call on a device looks the array's device address up
 * (cudaGetSymbolAddress) and caches it for the life of the process, which
 * assumes the device's primary context is never reset (cudaDeviceReset)
 * while the library is loaded.  All calls share the one array and it keeps the
 * last call's contents; each call rewrites every part it reads before reading
 * it.  Calls whose work overlaps on the GPU (other contexts' streams, other host
 * threads) race on the shared scratch and must be serialised by the caller.
 * Work runs on the context's stream, and the call synchronises that stream
 * before it returns. */
int pb_integrate_const_noalloc(pb_context* ctx, int64_t n, const double* d, int64_t nnz,
                               const int64_t* indptr, const int32_t* indices, const double* values,
                               int64_t n_steps, const double* z_grid, double* state);

/* The exp used by the device phi functions, evaluated on n values: a
 * correctly rounded double-double exp (same operation sequence as the host
 * form in oracle/crexp.py).  Replaces: the numpy exp of _compute_diag_factors
 * (src/prince_cr/solvers/etd2.py:355); exposed to test it against exact values. */
int pb_eval_exp(pb_context* ctx, int64_t n, const double* x, double* y);

/* Timing of the last pb_solve from CUDA events on the context stream (ms):
 * solve_ms  -- whole call on the device, including the state copy-out;
 * device_ms -- photon field, pair losses, fold, split and all steps (inputs resident);
 * steps_ms  -- the ETD2 step kernels alone;
 * launches  -- number of kernels the solve launched. */
int pb_last_timing(pb_context* ctx, double* solve_ms, double* device_ms, double* steps_ms, int64_t* launches);

#ifdef __cplusplus
}
#endif

#endif /* PRINCE_B200_H */
