/*
 * cdd.h -- C ABI of the B200 continuum-dislocation-dynamics (CDD) time step.
 *
 * One library, libcdd.so (sm_100a), built from cuda-plasticity_b200/csrc. Every entry point takes
 * plain pointers and sizes; device buffers are raw device pointers, streams are cudaStream_t
 * passed as void*. Device memory is allocated only by cdd_plan_create (the plan's scratch: k-space
 * spectra, stage buffers, reduction partials) and, on the first adjoint call on a plan, by the
 * adjoint entry points (their scratch, kept until cdd_plan_destroy).
 *
 * Field layout ("packed field"): instances are concatenated; instance i starts at element
 * cdd_plan_field_offset(plan, i) and holds 9 components in the order xx, xy, xz, yx, yy, yz,
 * zx, zy, zz, each a C-order array over the grid (axis 0 = the reference's x, last axis
 * contiguous). That is the numpy C order of the reference's per-component GridArray
 * (Plasticity/Fields/Fields.py L247-249, Plasticity/GridArray/GridArray.py L7-13).
 * Stress outputs use 6 symmetric components xx, xy, xz, yy, yz, zz (same per-instance base,
 * cdd_plan_stress_offset).
 *
 * Element type: double for CDD_F64 plans, float for CDD_F32 plans. Time, dt, speed maxima,
 * energies and mean strains are always double.
 *
 * Errors: every int-returning call returns a CDD_* status; cdd_last_error() gives a message for
 * the calling thread's last failure. Nothing here exits the process.
 *
 * Concurrency: calls on one plan are stream-ordered on the stream they are given and share the
 * plan's scratch, so two calls on the same plan must not overlap on the GPU. Different plans are
 * independent.
 */
#ifndef CDD_H
#define CDD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum cdd_status {
    CDD_OK = 0,
    CDD_ERR_ARG = 1,          /* bad argument (null pointer, negative count, ...) */
    CDD_ERR_SHAPE = 2,        /* unsupported grid shape */
    CDD_ERR_CUDA = 3,         /* a CUDA runtime call failed */
    CDD_ERR_NONFINITE = 4,    /* a wave-speed maximum was NaN/Inf: the step was not applied */
    CDD_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up */
    CDD_ERR_UNSUPPORTED = 6,  /* option not supported by this build */
    CDD_ERR_ALLOC = 7,        /* device allocation failed */
    CDD_ERR_IO = 8            /* a file could not be opened, read or written, or is too short */
};

enum cdd_precision { CDD_F64 = 0, CDD_F32 = 1 };

/* One simulation instance: grid, material, dynamics, loading and integrator parameters.
 * Mirrors PlasticityState(gridShape, nu, mu) (Plasticity/PlasticityStates/PlasticityState.py
 * L23-39), BetaPDynamics(Lambda) (Plasticity/FieldDynamics/CentralUpwindHJBetaPDynamics3D.py
 * L10-23), TVDRungeKutta_FieldMover(CFLsafeFactor) (Plasticity/FieldMovers/FieldMover.py
 * L14-18) and the applied-strain loading of UpwindLoadingBetaPDynamics (Plasticity/RunPython.py
 * L21-26, L35-50): sigma_ii += lamb_L tr(eps) + 2 mu_L eps_i, eps = load_initial +
 * load_rate (t - load_t0), lamb_L = 2 mu_L nu_L / (1 - 2 nu_L). */
typedef struct cdd_instance {
    int ndim;              /* 2 or 3 */
    int shape[3];          /* grid; shape[2] ignored for ndim == 2. Each size even, >= 4,
                              of the form 2^a 3^b or 2^a 5^c, <= 1024 */
    double mu, nu;         /* shear modulus and Poisson ratio of the internal stress */
    double Lambda;         /* 0: glide and climb; != 0: glide-projected (H_3D L195-200) */
    double cfl;            /* CFLsafeFactor of the adaptive time step */
    int has_load;          /* nonzero: add the applied-strain stress */
    double load_rate[3], load_initial[3], load_t0;
    double load_mu, load_nu;   /* stiffness the load is converted with */
    int dynamics;          /* CDD_DYN_GLIDE_CLIMB (0) or CDD_DYN_GLIDE_ONLY (1) */
    /* Vacancy coupling (BetaP_VacancyDynamics, Plasticity/FieldDynamics/VacancyDynamics.py L16-45,
     * stepped by OperatorSplittingTVDRK_FieldMover, Plasticity/FieldMovers/FieldMover.py L318-380):
     * nonzero `vacancy` adds a vacancy concentration c (see cdd_set_vacancy) with
     * sigma_ii -= vac_alpha c in the flux, and after each TVD-RK3 step
     * c += vac_beta (tr beta^P_new - tr beta^P_old) followed by exact diffusion
     * c^ *= exp(-vac_gamma dt k^2) (DiffusionEvolution L41-61). */
    int vacancy;
    double vac_alpha, vac_beta, vac_gamma;
    double dt_max;         /* > 0: upper bound of the adaptive step before the end-time clamp (the
                              operator-splitting mover's dtBound, default 0.01 there); 0: none */
} cdd_instance;

/* Dynamics of an instance: BetaPDynamics of CentralUpwindHJBetaPDynamics3D.py (glide and climb,
 * Lambda optional), or the glide-only BetaPDynamics of CentralUpwindHJBetaPGlideOnlyDynamics.py
 * (the velocity projected so that it carries no climb, L152-201 / 2-D L96-129; Lambda must be 0).
 * The adjoint entry points support CDD_DYN_GLIDE_CLIMB only. */
enum cdd_dynamics { CDD_DYN_GLIDE_CLIMB = 0, CDD_DYN_GLIDE_ONLY = 1 };

typedef struct cdd_plan cdd_plan;

/* Per-instance launch-shape choices (no counterpart in the reference; the autotuner in
 * cdd/autotune.py picks them by timing). 0 in a field keeps the built-in rule. Values out of range
 * (column counts not powers of two, shared memory over the device limit) give CDD_ERR_ARG.
 * None changes the mathematics: results agree with the defaults to rounding. */
typedef struct cdd_tuning {
    int fft_radix;        /* largest radix of the FFT stage plans: 16 (built-in), 8 or 4 */
    int rows_lines;       /* R2C / C2R passes: line pairs per block (<= 1024) */
    int mid_cols;         /* axis-1 FFT pass (3-D): spectrum columns per block (power of two) */
    int green_cols;       /* fused axis-0 FFT + Green pass: spectrum columns per block (power of two) */
    int stencil_planes;   /* stencil (3-D): planes marched per block along axis 0 */
    int plane_fft;        /* stress transforms of 3-D FP32 instances: 1 fuses the contiguous-axis
                             and axis-1 passes of each z-plane into one cluster kernel each way
                             (CDD_ERR_ARG when the shape does not allow it); 0 (built-in) or -1
                             keep the separate passes, which measure faster on B200 */
} cdd_tuning;

/* Create a plan for n_inst instances at the given precision on the current CUDA device.
 * Allocates all scratch. Replaces the per-run header generation + make of the reference's CUDA
 * path (Plasticity/RunCUDA.py L26-29, L194-214) and setupSystem (plasticity_kernel.cu L931-949). */
int cdd_plan_create(const cdd_instance* inst, int n_inst, int precision, cdd_plan** out);

/* cdd_plan_create with per-instance launch-shape choices (tune: n_inst entries, or NULL for the
 * built-in rules). */
int cdd_plan_create_tuned(const cdd_instance* inst, int n_inst, int precision, const cdd_tuning* tune,
                          cdd_plan** out);

/* The launch shapes a plan uses for instance i (the built-in rule's values where not tuned). */
int cdd_plan_tuning(const cdd_plan* plan, int i, cdd_tuning* out);

int cdd_plan_destroy(cdd_plan* plan);

int cdd_plan_num_instances(const cdd_plan* plan);
int cdd_plan_precision(const cdd_plan* plan);
/* Total elements of a packed 9-component field, and the start of instance i in it. */
long long cdd_plan_field_elems(const cdd_plan* plan);
long long cdd_plan_field_offset(const cdd_plan* plan, int i);
/* Total elements of a packed 6-component stress field, and the start of instance i. */
long long cdd_plan_stress_elems(const cdd_plan* plan);
long long cdd_plan_stress_offset(const cdd_plan* plan, int i);
/* Total cells over all instances, and the cells of instance i. */
long long cdd_plan_cells(const cdd_plan* plan, int i);
/* Bytes of device scratch the plan holds. */
long long cdd_plan_scratch_bytes(const cdd_plan* plan);

/* Internal stress sigma(beta^P) through the Fourier-space Green's function, FP64 k=0 mode.
 * Replaces PlasticityState.CalculateSigma(type='k', source='betaE') +
 * CalculateBetaElastic (PlasticityState.py L85-127, L357-390); reference CUDA twin
 * calculateSigma/calculateKSigma (plasticity_kernel.cu L778-1041).
 * beta: packed 9-component field; sigma6: packed 6-component output. */
int cdd_stress(cdd_plan* plan, const void* beta, void* sigma6, void* stream);

/* Central-upwind Hamilton-Jacobi flux with the wave speed used by the CFL condition, at time t
 * (t sets the applied load). Replaces BetaPDynamics.CalculateFlux(time, state,
 * CFLCondition=True) (CentralUpwindHJBetaPDynamics3D.py L218-221 ->
 * CentralUpwindHJ3D.py L99-271); reference CUDA twin calculateFlux/centralHJ
 * (plasticity_kernel.cu L1068-1094, L118-697).
 * rhs: packed 9-component output; speed: one value per cell (packed, instance i at
 * sum of previous cells), may be NULL. */
int cdd_flux(cdd_plan* plan, const void* beta, double t, void* rhs, void* speed, void* stream);

/* cdd_flux with the internal stress given by the caller (packed 6-component sigma6, e.g. from
 * cdd_stress or from another stress model); the applied load of time t is still added. The
 * reference's dynamics take their stress from an overridable GetSigma (RunPython.py L35-50);
 * this is that seam. Launches only the stencil kernel. */
int cdd_flux_with_stress(cdd_plan* plan, const void* beta, const void* sigma6, double t, void* rhs, void* speed,
                         void* stream);

/* Per-instance clocks: t (current time) and t_end (end of the current Run interval).
 * Host arrays of length n_inst. */
int cdd_set_time(cdd_plan* plan, const double* t, const double* t_end);
/* Read t, the last dt and the active flags back (synchronises the plan's last stream).
 * Any pointer may be NULL. */
int cdd_get_time(cdd_plan* plan, double* t, double* dt_last, int* active);

/* One adaptive TVD-RK3 step of every active instance, in place on beta (device).
 * dt = cfl / (max(shape) * max_cells(speed)), clamped so t + dt <= t_end; the three stages use
 * the step-start time; t += dt on the device. An instance with t >= t_end is left untouched.
 * Replaces TVDRungeKutta_FieldMover.CalculateOneAdaptiveTimeStep (FieldMover.py L61-141);
 * reference CUDA twin TVD3rd (plasticity_kernel.cu L1139-1206). No host synchronisation. */
int cdd_step(cdd_plan* plan, void* beta, void* stream);

/* One TVD-RK3 step with a fixed dt (clamped to t_end).
 * Replaces CalculateOneFixedTimeStep (FieldMover.py L38-58). */
int cdd_step_fixed(cdd_plan* plan, void* beta, double dt, void* stream);

/* n_steps adaptive steps; with use_graph != 0 the step is captured once into a CUDA graph
 * (per plan, beta pointer and stream) and replayed. */
int cdd_run(cdd_plan* plan, void* beta, int n_steps, int use_graph, void* stream);

/* Elastic energy (sum over cells of 1/2 S:sigma sigma, PlasticityState.CalculateElasticEnergy
 * L317-330 as summed in Observers/Observer.py L99) and mean beta^P_zz of every instance,
 * accumulated in FP64. energy, mean_zz: host arrays of length n_inst (either may be NULL).
 * Synchronises the stream. */
int cdd_observables(cdd_plan* plan, const void* beta, double* energy, double* mean_zz,
                    void* stream);

/* ---- adjoint (reverse-mode) building blocks ----
 * Vector-Jacobian product of the flux at time t: with rhs = L(beta) = flux(beta, sigma(beta) + load),
 * given gbar = d(loss)/d(rhs) (packed 9-component field) it writes
 *   betabar = (dL/dbeta)^T gbar (packed 9-component field, overwritten),
 *   sigbar6 = d(loss)/d(total stress) at every cell (packed 6-component field, off-diagonal entries
 *             carry both (i,j) and (j,i)),
 * and adds sum over cells of the diagonal of sigbar (the applied-load cotangent, 3 per instance)
 * to the device array load_bar (may be NULL). The limiter selections and the corners attaining
 * the directional speed maxima are those of the forward evaluation at beta.
 * Reverse of BetaPDynamics.CalculateFlux (CentralUpwindHJBetaPDynamics3D.py L218-221 ->
 * CentralUpwindHJ3D.py L189-271); the reference has no adjoint. Allocates the plan's adjoint
 * scratch (54 derivative cotangents and 4 flag words per cell) on first use. */
int cdd_flux_vjp(cdd_plan* plan, const void* beta, double t, const void* gbar, void* betabar,
                 void* sigbar6, double* load_bar, void* stream);

/* Branch record of the flux at beta and time t: the branches that cdd_flux_vjp differentiates
 * through. flags (device): 4 words per cell, packed per instance like the field (instance i at
 * 4 * (its field offset / 9)), word q of cell x at q * cells + x. Limiter slot s = 3 * component +
 * axis holds 4 bits in word s / 8 at bit 4 * (s % 8): bits 0-1 the selection of the forward
 * one-sided derivative's minmod (0 zero, 1 first argument, 2 second), bits 2-3 the backward one's.
 * Bits 12-31 of word 3 hold, base 9, the corner (index + 1; 0 = the zero entry) attaining the max
 * and then the min of each axis' corner velocity (CentralUpwindHJ3D.py L197-234). Two states
 * with equal records lie on the same smooth piece of the flux. The reference has no counterpart. */
int cdd_flux_branches(cdd_plan* plan, const void* beta, double t, uint32_t* flags, void* stream);

/* Transposed stress operator: betabar9 = S^T sigbar6 (packed 6 -> packed 9 components,
 * overwritten), S = the map of cdd_stress. Adjoint of PlasticityState.CalculateSigma
 * (PlasticityState.py L85-127). */
int cdd_stress_adjoint(cdd_plan* plan, const void* sigbar6, void* betabar9, void* stream);

/* Derivative of the internal stress with respect to nu at fixed mu and beta:
 * out6 = (dS/dnu) beta (packed 6 components). (dS/dmu) beta = S beta / mu needs no call. */
int cdd_stress_dnu(cdd_plan* plan, const void* beta, void* out6, void* stream);

/* ---- checkpointed reverse sweep of fixed-dt runs (no counterpart in the reference) ----
 * A "step record" holds what the reverse of one fixed-dt step needs: the step's input u, its
 * stage states F0 and F1 (FieldMover.py L38-58), their internal stresses and, per k point, the
 * scalar spectrum s1 / kSq - r / kSqSq of each of the three states (s1 = trace, r = k.beta.k of
 * the transformed beta), from which the nu gradient follows by Parseval without extra FFTs.
 * cdd_plan_record_elems gives its size in plan elements (double or float); the caller owns the
 * records (device memory, 256-byte aligned). */
long long cdd_plan_record_elems(const cdd_plan* plan);

/* One TVD-RK3 step of every instance with the fixed dt, starting at time t (the plan clock is set
 * to t with no end time and advanced by dt). Bitwise the same update as cdd_set_time + cdd_step_fixed.
 * rec (device, may be NULL): when given, the step's record is written there. No host
 * synchronisation. */
int cdd_step_record(cdd_plan* plan, void* beta, double t, double dt, void* rec, void* stream);

/* Number of doubles per instance of the parameter cotangent array of cdd_step_adjoint. */
#define CDD_PBAR 9

/* Reverse of the step recorded in rec (taken at time t with the fixed dt): ubar holds the
 * cotangent of the step's output on entry and that of its input u on return (packed field):
 *   F1b = 2/3 ubar + 2/3 dt L_{F1}^T ubar,  F0b = 1/4 F1b + 1/4 dt L_{F0}^T F1b,
 *   ubar <- 1/3 ubar + 3/4 F1b + F0b + dt L_u^T F0b,
 * L_v^T the flux VJP of cdd_flux_vjp at v (recorded limiter selections and speed-max corners).
 * pbar (device, CDD_PBAR doubles per instance, may be NULL): parameter cotangents of the three
 * stages are added: [0] sum <sigbar, sigma_int> (d/d mu = [0] / mu), [1] sum tr(sigbar) tr(sigma_int)
 * (d/d nu through lambda = [1] * dlambda/dnu / (2 mu + 3 lambda)), [2] the k-space part of d/d nu
 * per unit d(lambda / (lambda + 2 mu))/dnu, [3..5] the diagonal of sigbar summed over cells (the
 * applied-load cotangent), [6..8] the same times (t - load_t0). Each stage's terms carry its
 * weight (2/3 dt, 1/4 dt, dt). No host synchronisation. */
int cdd_step_adjoint(cdd_plan* plan, const void* rec, double t, double dt, void* ubar, double* pbar,
                     void* stream);

/* Device status flags accumulated by kernels (CDD_ERR_NONFINITE, ...); clears them. */
int cdd_check_status(cdd_plan* plan);

/* Size of the fixed device scratch of cdd_stress_noalloc. Every GPU that loads the library holds
 * this much device memory until the process exits. */
#define CDD_STRESS_NOALLOC_MAX_BYTES (32u << 20)

/* Internal stress of ONE instance, like cdd_stress, without allocating any device memory.
 * No counterpart in the reference: it exists for callers that cannot call cudaMalloc (and so
 * cannot create a plan) -- hosts that own all device memory through their own allocator and
 * forbid libraries from allocating, services that must not allocate after start-up. The scratch (k-space spectra, FFT and k tables, FP64 row sums) is a fixed
 * CDD_STRESS_NOALLOC_MAX_BYTES array inside the library; a grid that needs more is rejected with
 * CDD_ERR_SHAPE and a message giving both sizes (e.g. FP64 64^3 and FP32 80^3 fit, 128^3 does
 * not). The first call on a device looks the array's device address up (once per device, with
 * that device current); make that first call before any stream capture. A cudaDeviceReset makes
 * the looked-up address stale, like every other device pointer. All calls share the
 * array: calls that overlap on the GPU race and must be serialised by the caller. Each call
 * writes every scratch byte it reads, so nothing needs clearing between calls.
 * inst: one instance (shape, mu, nu); precision: CDD_F64 or CDD_F32; beta: 9 * cells elements
 * (device); sigma6: 6 * cells elements (device), components xx, xy, xz, yy, yz, zz. */
int cdd_stress_noalloc(const cdd_instance* inst, int precision, const void* beta, void* sigma6,
                       void* stream);

/* Message for the calling thread's last failing call ("" if none). */
/* Register the device buffer of vacancy concentrations used by every later step and flux call of
 * the plan (NULL clears it): field_elems / 9 elements of the plan's precision, instance i at
 * cdd_plan_field_offset(i) / 9 (one value per cell); entries of instances without vacancy coupling
 * are ignored. Steps update it in place. Required (CDD_ERR_ARG otherwise) before stepping or
 * evaluating the flux of a plan that has a vacancy instance. A CUDA graph of cdd_run is re-captured
 * when the buffer changes. The adjoint entry points do not support vacancy instances. */
int cdd_set_vacancy(cdd_plan* plan, void* c);

/* ---- Field observables in k space (PlasticityState.py) ----
 * out: a packed field buffer of the plan's precision. 9-component observables are written in the
 * field layout (instance i at cdd_plan_field_offset(i)); 3-component ones in a packed 3-component
 * layout (instance i at cdd_plan_field_offset(i) / 3, components back to back, cells apart).
 *  CDD_OBS_BETA_ELASTIC: beta^E = IFFT(kmask T beta^P^) - beta^P, 9 components
 *                        (CalculateBetaElastic L357-390);
 *  CDD_OBS_ROTATION:     (beta^E_ij - beta^E_ji) / 2 for (xy, xz, yz), 3 components
 *                        (CalculateRotationField L435-446: the other entries follow by antisymmetry);
 *  CDD_OBS_RODRIGUES:    the Rodrigues rotation vector (x, y, z) from beta^P, 3 components
 *                        (CalculateRotationRodrigues L447-475, source 'betaP');
 *  CDD_OBS_RHO:          the Nye dislocation density rho_ij = -eps_ikl d_k beta^P_lj by Fourier
 *                        derivatives, 9 components (CalculateRhoFourier L264-304).
 * Uses the plan's spectrum scratch (stream-ordered with the other entry points). CDD_ERR_SHAPE when
 * the k-space pass of 12 component slots does not fit the device's shared memory. */
/*  CDD_OBS_RODRIGUES_RHO: the Rodrigues vector from the Nye density (CalculateRotationRodrigues L472-494,
 *                        source 'rho'): `beta` holds the density field as CDD_OBS_RHO returns it (field
 *                        layout, 9 components), transformed again and contracted with
 *                        D_imn = i (2 k_n d_im - k_m d_in - k_i d_mn) / (2 kSq) + i k_i k_n k_m / (2 kSqSq);
 *                        3 components, no real-space term (the means are lost, as in the reference).
 * kind | CDD_OBS_SINK uses the k tables of FourierSpaceTools(gridShape, func=sin) (the reference's type
 * 'sinK', n sin(2 pi i / n) per axis) instead of the wrapped identity ones; kmask is the same. */
enum cdd_observable { CDD_OBS_BETA_ELASTIC = 0, CDD_OBS_ROTATION = 1, CDD_OBS_RODRIGUES = 2, CDD_OBS_RHO = 3,
                      CDD_OBS_RODRIGUES_RHO = 4 };
#define CDD_OBS_SINK 0x100
int cdd_observe_field(cdd_plan* plan, int kind, const void* beta, void* out, void* stream);

/* ---- The reference CUDA solver's on-disk formats ----
 * File layout of one field: the 9 components in the order xx xy xz yx yy yz zx zy zz, each with
 * grid axis 0 fastest (element (i0, i1, i2) at i0 + n0 (i1 + n1 i2); 2-D: i0 + n0 i1): the
 * reference writes every component transposed (Plasticity/RunCUDA.py L9-22, convertStateToCUDA)
 * and reads it back transposed (Plasticity/FieldInitializers/FieldInitializer.py L61-103,
 * LoadStateRaw). A plan stores each component with the last axis contiguous.
 *  .ics : one field in float64, no time (read by plasticity.cu L126-140 with ReadDoubleMatrixFile,
 *         assist.h L65-97; written by convertStateToCUDA).
 *  .plas: frames [t][field], t and the field in the file's precision (the solver's data_type:
 *         float64 or float32), appended by ContinueWriteMatrix (assist.h L164-192,
 *         plasticity.cu L153-159); a restart continues from the last frame (plasticity.cu L107-123).
 * `beta` is always the plan's packed field; i selects the instance whose part is converted.
 * The file functions synchronise `stream` and stage through a temporary device buffer. */

/* Device conversion between instance i's part of beta and a device buffer in the file layout
 * (9 * cells elements of src_precision / dst_precision; FP64 -> FP32 rounds to nearest). */
int cdd_field_import(cdd_plan* plan, int i, const void* src, int src_precision, void* beta, void* stream);
int cdd_field_export(cdd_plan* plan, int i, const void* beta, void* dst, int dst_precision, void* stream);

/* .ics: read the first 9 * cells float64 values of `path` into instance i; write instance i. */
int cdd_ics_read(cdd_plan* plan, int i, const char* path, void* beta, void* stream);
int cdd_ics_write(cdd_plan* plan, int i, const char* path, const void* beta, void* stream);

/* .plas: append the frame (t, instance i) in file_precision (creating the file); count the whole
 * frames of a file (a trailing partial frame is ignored, as LoadStateRaw does); read frame
 * `frame` (0-based; negative counts from the end, -1 = the last frame, the restart state) into
 * instance i and its time into *t. */
int cdd_plas_append(cdd_plan* plan, int i, const char* path, double t, const void* beta, int file_precision,
                    void* stream);
int cdd_plas_frames(cdd_plan* plan, int i, const char* path, int file_precision, long long* frames);
int cdd_plas_read(cdd_plan* plan, int i, const char* path, int file_precision, long long frame, double* t,
                  void* beta, void* stream);

const char* cdd_last_error(void);

/* Library version string. */
const char* cdd_version(void);

#ifdef __cplusplus
}
#endif
#endif /* CDD_H */
