/*
 * hops_b200.h -- C ABI of the B200-native HOPS trajectory hot path.
 *
 * Every entry point is plain C (extern "C"), takes plain pointers and sizes and
 * returns an int status: 0 = success, > 0 = one of the HOPS_E* codes below; the
 * text of the last error of the calling thread is available from
 * hops_last_error().  All array pointers named *_dev are CUDA device pointers
 * owned by the caller; the library allocates no device memory on these paths
 * except the cuFFT plan work area inside hops_noise_filter.  `stream` is a
 * cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Reference interfaces replaced (paths inside the MesoHOPS source tree
 * src/mesohops):
 *   hops_dsystem_dt          <- eom/hops_eom.py:196-441 (nonlinear dsystem_dt closure)
 *                               and hops_eom.py:445-542 (LINEAR closure)
 *   hops_rk4_propagate       <- trajectory/hops_trajectory.py:456-533 loop body:
 *                               integrator/integrator_rk.py:78-134 (noise at
 *                               t, t+tau/2, t+tau), integrator_rk.py:10-75 (RK4)
 *                               and hops_trajectory.py:616-634 (normalize)
 *   hops_resident_propagate  <- same loop, one CTA per trajectory with its own
 *                               (possibly uneven) basis, all steps in one launch
 *   hops_noise_filter        <- noise/hops_noise.py:630-716 (_construct_correlated_noise)
 *                               with hops_noise.py:167-192,232-247 (alpha, complex64)
 *   hops_noise_window_mean   <- integrator/integrator_rk.py:115-128 (effective noise)
 *   hops_noise_draw          <- noise/hops_noise.py:558-628 (_generate_noise_samples with
 *                               PCG64(SEED).jumped(lop) streams, _construct_indexing)
 *                               and hops_noise.py:522-553 (complex64 raw noise)
 */
#ifndef HOPS_B200_H
#define HOPS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HOPS_OK 0
#define HOPS_EINVAL 1       /* bad argument (sizes, null pointers, unsupported mode) */
#define HOPS_ECUDA 2        /* a CUDA runtime / driver call failed */
#define HOPS_ENOTSUP 3      /* request outside what the library implements */
#define HOPS_ENONFINITE 5   /* a trajectory produced NaN/Inf (status word set) */
#define HOPS_ETIMEOUT 6     /* a wait inside a kernel ran out of time (status word set) */

#define HOPS_PREC_C128 0    /* complex128 state and arithmetic */
#define HOPS_PREC_C64 1     /* complex64 state/SpMM, FP64 <L>, norm, z_mem */
#define HOPS_PREC_MIXED 2   /* complex128 state; complex64 storage of the stage vectors;
                               FP64 arithmetic and scalars */

#define HOPS_EOM_NORMALIZED_NONLINEAR 0
#define HOPS_EOM_NONLINEAR 1
#define HOPS_EOM_LINEAR 2

/*
 * One hierarchy basis in device memory (all pointers are device pointers).
 * Complex numbers are stored as interleaved (re, im) doubles; *_f arrays hold
 * the same coefficients rounded to float for HOPS_PREC_C64.
 * Aux index a, state index s; phi element (a, s, b) of a batch of B
 * trajectories lives at ((a * n_state) + s) * B + b (trajectory fastest; for
 * B = 1 this is the reference's flat index a * n_state + s).
 */
typedef struct hops_structure {
  int32_t n_hier, n_state, n_mode, n_lop;
  int32_t n_first;        /* first-level aux entries used by the norm correction */
  int32_t n_up, n_dn;     /* connection counts */
  int32_t site_projector; /* 1: every L_j = v_j |s_j><s_j| (fast path) */
  int32_t max_up, max_dn; /* longest connection list of any aux */
  /* per aux */
  const double* k_decay;  /* [n_hier] complex: -sum_m k_m w_m (K2_k diagonal) */
  const float* k_decay_f;
  const int32_t* up_ptr;  /* [n_hier+1] CSR over aux of the k+1 connections */
  const int32_t* up_aux;  /* [n_up] aux index a + e_m */
  const int32_t* up_mode; /* [n_up] relative mode m */
  const int32_t* dn_ptr;  /* [n_hier+1] CSR over aux of the k-1 connections */
  const int32_t* dn_aux;  /* [n_dn] aux index a - e_m */
  const int32_t* dn_mode; /* [n_dn] relative mode m */
  const double* dn_coef;  /* [n_dn] complex: k_m(a) * w_m */
  const float* dn_coef_f;
  /* per relative mode */
  const int32_t* mode_lop; /* [n_mode] relative L index of the mode */
  const double* mode_g;    /* [n_mode] complex g_m */
  const double* mode_w;    /* [n_mode] complex w_m */
  const double* mode_gw;   /* [n_mode] complex g_m / w_m */
  const float* mode_gw_f;
  /* first-level aux (hops_eom.py:186-194) */
  const int32_t* first_aux;  /* [n_first] */
  const int32_t* first_mode; /* [n_first] */
  /* L operators in the state basis: CSR of L_j and CSR of L_j^H */
  const int32_t* l_ptr; /* [n_lop * (n_state+1)] */
  const int32_t* l_col;
  const double* l_val;  /* complex */
  const float* l_val_f;
  const int32_t* lh_ptr;
  const int32_t* lh_col;
  const double* lh_val;
  const float* lh_val_f;
  const int32_t* lop_active; /* [n_lop] 1 if L_j has a nonzero in the basis */
  const int32_t* lop_site;   /* [n_lop] s_j (site-projector form) */
  const double* lop_sval;    /* [n_lop] complex v_j (site-projector form) */
  /* -i H as CSR over states */
  const int32_t* h_ptr; /* [n_state+1] */
  const int32_t* h_col;
  const double* h_val;  /* complex, already multiplied by -i */
  const float* h_val_f;
  /* site-projector form, per relative mode m and per down connection p */
  const int32_t* mode_site;    /* [n_mode] s_{l(m)} */
  const double* mode_gwv;      /* [n_mode] complex (g_m/w_m) v_{l(m)} */
  const float* mode_gwv_f;
  const double* dn_coef_site;  /* [n_dn] complex k_m(a) w_m conj(v_{l(m)}) */
  const float* dn_coef_site_f;
  const int32_t* up_site;      /* [n_up] s_{l(m)} of the connection's mode, or -1 */
  const int32_t* dn_site;      /* [n_dn] s_{l(m)} of the connection's mode, or -1 */
  /* site-projector form: diagonal of -i H, kept out of the H CSR above and
     added to the per-state diagonal coefficient; NULL otherwise */
  const double* h_diag;        /* [n_state] complex */
  /* low-temperature correction (eom/eom_functions.py:215-309 as applied by
     eom/hops_eom.py:357-403,527-529); NULL when every coefficient is zero */
  const double* lt_coef;  /* [n_lop] complex c_j (summed PARAM_LT_CORR of L_j) */
  const int32_t* l2_ptr;  /* [n_lop * (n_state+1)] CSR of L_j^2 */
  const int32_t* l2_col;
  const double* l2_val;   /* complex */
  /* every aux a >= n_up_prefix has no up connection (0: not known); task
     order 3 of the batched stage kernel runs the aux below it state by state */
  int32_t n_up_prefix;
  int32_t reserved;
} hops_structure;

/*
 * A batch of B trajectories sharing one hops_structure.  Vectors phi, acc,
 * y0, y1 have n_hier * n_state * B complex elements, laid out
 * [aux][state][trajectory]; phi is complex128 for HOPS_PREC_C128 and
 * HOPS_PREC_MIXED, complex64 for HOPS_PREC_C64; acc, y0, y1 (and phi_lo) are
 * complex64 unless the precision is HOPS_PREC_C128.
 */
typedef struct hops_batch {
  int32_t n_traj;
  int32_t precision; /* HOPS_PREC_* */
  int32_t eom;       /* HOPS_EOM_* */
  int32_t n_t1, n_t2;   /* noise time-axis lengths */
  void* phi;   /* state; normalised lazily by `scale` (see hops_rk4_propagate) */
  void* acc;   /* RK4 accumulator */
  void* y0;    /* stage inputs (ping-pong) */
  void* y1;
  double* zmem;  /* [B][n_mode] complex noise memory */
  double* work;  /* scalar workspace of hops_scalar_workspace_doubles() doubles */
  const float* noise1; /* [B][n_lop][n_t1] complex64 (complex128 if noise_c128) */
  const float* noise2; /* [B][n_lop][n_t2] likewise, or NULL for zero noise 2 */
  int32_t* status;     /* [B] 0 ok, HOPS_ENONFINITE if a norm went NaN/Inf */
  void* phi_lo;        /* HOPS_PREC_MIXED: complex64 copy of phi read by stage 1 */
  int32_t defer_scale; /* 1: hops_rk4_propagate leaves the renormalisation of its
                          last step pending (see there) */
  int32_t noise_c128;  /* 1: noise1 / noise2 hold complex128 samples (noise with
                          INTERPOLATE, hops_noise.py:242-279: the cubic spline
                          through the samples, evaluated at them); 0: complex64 */
} hops_batch;

/* One trajectory of hops_resident_propagate (array in device memory). */
typedef struct hops_task {
  const hops_structure* st; /* device pointer to the structure */
  void* phi;                /* [n_hier][n_state]: complex64 for HOPS_PREC_C64, else complex128 */
  double* zmem;             /* [n_mode] complex */
  const float* noise1;      /* [n_lop][n_t1] complex64 (complex128 if noise_c128) */
  const float* noise2;      /* [n_lop][n_t2] complex64 or NULL */
  double* psi_out;          /* [n_steps][n_state] complex128, or NULL */
  void* scratch;            /* 3 * n_hier * n_state stage elements (complex128 for
                               HOPS_PREC_C128, else complex64) used when the vectors
                               do not fit shared memory */
  int32_t n_t1, n_t2;
  int32_t it0;      /* noise index of the start time */
  int32_t di;       /* noise index step per half time step */
  int32_t n_steps;
  int32_t precision;
  int32_t eom;
  int32_t status;   /* written by the kernel: 0 ok, HOPS_ENONFINITE */
  double tau_over_hbar;
  double scale;     /* pending normalisation factor of phi (1 = none) */
  int32_t noise_c128; /* 1: noise1 / noise2 hold complex128 samples (see hops_batch) */
  int32_t pad;
} hops_task;

/* One trajectory of hops_flux_errors (array in device memory). */
typedef struct hops_flux_task {
  const hops_structure* st; /* device pointer to the structure of the current basis */
  const double* phi;        /* [n_hier][n_state] complex128, normalised */
  const double* zmem;       /* [n_mode] complex128 noise memory */
  const float* z1;          /* [n_lop] complex64 noise 1 at the current time */
  const float* z2;          /* [n_lop] complex64 noise 2 or NULL */
  const int32_t* aux_mask;  /* [n_hier] 1 = keep, 0 = zero before the derivative; or NULL */
  double* e_deriv;          /* out [n_hier][n_state] */
  double* e_up;             /* out [n_mode][n_hier], or NULL to skip e_up/e_down */
  double* e_down;           /* out [n_mode][n_hier] */
  const uint8_t* k_aux;     /* [n_mode][n_hier] depth of each aux in each mode */
  double dt;                /* time step of the error estimate [fs] */
  int32_t eom;
  int32_t pad;
} hops_flux_task;

const char* hops_last_error(void);
int hops_version(void);
int hops_device_query(int device, int* sm_count, int* smem_optin_bytes);

/* Doubles of scalar workspace hops_batch.work must hold. */
size_t hops_scalar_workspace_doubles(int32_t n_state, int32_t n_mode, int32_t n_lop,
                                     int32_t n_traj);

/* Reset the scalar workspace (pending scale = 1, status = 0). */
int hops_batch_reset(const hops_structure* st, hops_batch* bt, void* stream);

/*
 * dsystem_dt for the B trajectories of bt at the state bt->phi (scale applied),
 * memory bt->zmem and one noise sample per L: z1_dev / z2_dev are [B][n_lop]
 * complex64 (z2_dev may be NULL).  Writes dphi (layout of phi, in cm^-1, not
 * divided by hbar) and dzmem ([B][n_mode] complex128).
 */
int hops_dsystem_dt(const hops_structure* st, hops_batch* bt, const float* z1_dev,
                    const float* z2_dev, void* dphi_dev, double* dzmem_dev, void* stream);

/*
 * n_steps RK4 steps of size tau (tau_over_hbar = tau / hbar) from the noise
 * index it0; stage noise is read at it0 + 2*n*di + {0, di, di, 2*di}.  For the
 * normalized EOM the state is renormalised after every step; psi_out_dev
 * (nullable) receives [n_steps][B][n_state] complex128 normalised psi_0 after
 * each step.  On return phi holds the normalised state -- unless
 * bt->defer_scale is set: then the last step's 1/||psi_0|| stays pending in
 * the workspace (phi and phi_lo unscaled, psi_out_dev already normalised),
 * the next hops_rk4_propagate or hops_dsystem_dt applies it on the fly as the
 * steps within one call do, and hops_batch_settle applies it to phi.  That
 * saves a read and write of the whole state per call when the caller steps
 * one call at a time (hops_trajectory.py:456-533 calls the integrator once
 * per step).
 */
int hops_rk4_propagate(const hops_structure* st, hops_batch* bt, int32_t it0,
                       int32_t di, int32_t n_steps, double tau_over_hbar,
                       double* psi_out_dev, void* stream);

/* Apply a pending renormalisation (bt->defer_scale) to phi and phi_lo and
 * reset it to 1; status is kept.  No counterpart in the reference. */
int hops_batch_settle(const hops_structure* st, hops_batch* bt, void* stream);

/*
 * Resident propagation: one CTA per task, all n_steps steps of every task in
 * one launch, stage vectors in shared memory when they fit (otherwise in the
 * task's scratch).  tasks_dev is a device array of n_tasks hops_task; the
 * kernel writes each task's status and leaves its phi normalised.
 * max_elems: largest n_hier*n_state of any task; max_scalar_doubles: largest
 * hops_resident_scalar_doubles() of any task; all_site_projector: 1 if every
 * task's structure has site_projector = 1 (selects the fast path).
 */
int hops_resident_propagate(hops_task* tasks_dev, int32_t n_tasks, int32_t max_elems,
                            int32_t max_scalar_doubles, int32_t precision,
                            int32_t all_site_projector, void* stream);

/*
 * Adaptive-basis error estimates, one CTA per task, FP64 (replaces the array
 * parts of basis/basis_functions_adaptive.py: error_deriv :10-74,
 * error_flux_up_hier_stable :165-266, error_flux_down_hier_stable :517-624).
 * max_smem_doubles: largest hops_flux_errors_smem_doubles() of any task.
 */
int hops_flux_errors(hops_flux_task* tasks_dev, int32_t n_tasks, int32_t max_smem_doubles,
                     double hbar, void* stream);
int32_t hops_flux_errors_smem_doubles(int32_t n_state, int32_t n_mode, int32_t n_lop);

/*
 * Structure builder for a full triangular hierarchy (every aux of depth
 * <= depth over n_mode modes, no static filters), replacing the host-side
 * construction of the aux list, its connections (hops_hierarchy.py:340-368,
 * 470-523) and K2_k (eom_hops_ksuper.py:36-90).  Aux g is the g-th multiset in
 * (size, lexicographic) order.  binom_dev: int64 C(n, j) for n <= n_mode +
 * depth + 1, j <= depth + 1, row stride depth + 2.
 * pass1: k_decay_dev[g] = -sum_m k_m(g) w_m (complex128, w_dev [n_mode]) and
 *        dn_count_dev[g] = number of distinct modes of g.
 * pass2: dn_ptr_dev = exclusive prefix sum of dn_count (n_hier + 1 entries,
 *        from the caller); writes the n_below * n_mode up connections of the
 *        aux of depth < depth (aux g, mode m at g * n_mode + m) and, per aux,
 *        its down connections in increasing mode order with k_m(g).
 */
int32_t hops_tri_max_depth(void);
int hops_tri_pass1(int32_t n_mode, int32_t depth, const int64_t* binom_dev, int64_t n_hier,
                   const double* w_dev, double* k_decay_dev, int32_t* dn_count_dev,
                   void* stream);
int hops_tri_pass2(int32_t n_mode, int32_t depth, const int64_t* binom_dev, int64_t n_hier,
                   int64_t n_below, const int32_t* dn_ptr_dev, int32_t* up_aux_dev,
                   int32_t* up_mode_dev, int32_t* dn_aux_dev, int32_t* dn_mode_dev,
                   int32_t* dn_k_dev, void* stream);

/* Shared-memory doubles of per-stage scalars one resident task needs. */
int32_t hops_resident_scalar_doubles(int32_t n_state, int32_t n_mode, int32_t n_lop);

/*
 * FFT-filtered correlated noise in FP64.  For each of n_lop rows:
 * alpha (complex128 [n_lop][n_t], already summed over the noise modes of the
 * row) is rounded to complex64 (hops_noise.py:236), rotated so its last sample
 * is real, embedded in a circulant of length 2(n_t-1), transformed, clipped at
 * zero and used to filter the complex64 draws z_dev ([n_lop][2(n_t-1)]); the
 * first n_t samples, un-rotated, are written to out_dev as complex128
 * ([n_lop][n_t]; nullable) and, if out64_dev is not NULL, as complex64.
 * The transforms use cuFFT (plan created and destroyed inside the call).
 * n_negative_host (nullable) receives the number of clipped spectral values.
 */
int hops_noise_filter(const double* alpha_dev, const float* z_dev, int32_t n_lop,
                      int32_t n_t, double* work_dev, double* out_dev, float* out64_dev,
                      int64_t* n_negative_host, void* stream);

/* Doubles of device work area hops_noise_filter needs (work_dev). */
size_t hops_noise_filter_work_doubles(int32_t n_lop, int32_t n_t);

/* hops_noise_filter for rows that share correlation functions (the
 * trajectories of an ensemble: the same system, their own noise): z_dev and
 * the outputs have n_rows rows, alpha_dev n_alpha rows, and row r is filtered
 * with alpha row r % n_alpha (n_rows a multiple of n_alpha).  The result
 * equals hops_noise_filter on alpha tiled to n_rows rows, without the tiled
 * copy.  The work area of hops_noise_filter_work_doubles(n_rows, n_t)
 * suffices.  Both filter entry points take their cuFFT plan from a pool of
 * at most 8 idle plans (per device, length and batch; each holds cuFFT's work
 * area) and return it when the call has synchronised (n_negative_host set),
 * so repeated set-ups of one shape skip the plan construction.  Same replaced
 * interface as hops_noise_filter. */
int hops_noise_filter_shared(const double* alpha_dev, int32_t n_alpha, const float* z_dev,
                             int32_t n_rows, int32_t n_t, double* work_dev, double* out_dev,
                             float* out64_dev, int64_t* n_negative_host, void* stream);

/* Effective noise of EFFECTIVE_NOISE_INTEGRATION: replaces the window means of
 * integrator/integrator_rk.py:115-128 (np.mean over complex64 samples).
 * noise_dev: complex64 [rows][n_t]; out_dev: complex64 [rows][n_out] with
 * out[r][w] = mean(noise[r][start + w*k .. start + (w+1)*k - 1]), summed in
 * numpy's pairwise order and divided by k in single precision, so the means
 * are bit-identical to the reference's.  real_only: FLAG_REAL noise (the real
 * parts averaged as float32, imaginary parts 0).  The RK slots of step n are
 * then windows 2n, 2n+1, 2n+2 of the series that starts at the step's time,
 * i.e. hops_rk4_propagate with it0 = 0, di = 1 on out_dev.
 * Requires start + n_out*k <= n_t. */
int hops_noise_window_mean(const float* noise_dev, int64_t rows, int32_t n_t, int32_t start,
                           int32_t k, int32_t n_out, int32_t real_only, float* out_dev,
                           void* stream);

/* Raw (uncorrelated) white noise of the FFT_FILTER model drawn on the device:
 * replaces noise/hops_noise.py:558-628 (one PCG64(SEED).jumped(lop) stream per
 * L-operator, numpy's Generator.normal for RAND_MODEL "SUM_GAUSSIAN" = model 0
 * or Generator.random with the Box-Muller transform for "BOX_MULLER" = model 1,
 * draws placed by _construct_indexing) and the complex64 assembly of
 * hops_noise.py:522-553.  seed_states_dev: device uint64 [n_traj][4], each
 * trajectory's un-jumped PCG64 state (state high and low 64 bits, increment
 * high and low 64 bits: numpy's PCG64(SEED).state); lops_dev: device int32
 * [n_lop], the absolute L-operator index (>= 0) of each row; z_dev: complex64
 * [n_traj * n_lop][2(n_t-1)] out, row b*n_lop + j for trajectory b and
 * L-operator lops[j].  SUM_GAUSSIAN draws equal numpy's bit for bit (a tail
 * draw, about 3e-4 of them, goes through log1p, whose last bit may differ
 * between math libraries: after the rounding to complex64 that changes a
 * sample with probability ~1e-8); BOX_MULLER uses the device's log and sincos,
 * so a sample can differ from numpy's in its last complex64 bit.  The output
 * is the z_dev input of hops_noise_filter.  Requires n_t >= 2. */
int hops_noise_draw(const uint64_t* seed_states_dev, int32_t n_traj, const int32_t* lops_dev,
                    int32_t n_lop, int32_t n_t, int32_t model, float* z_dev, void* stream);

/* The seed_states_dev input of hops_noise_draw from integer SEEDs, on the
 * device: numpy's SeedSequence(SEED) hashing and PCG64 seeding (the
 * reference's np.random.PCG64(seed=SEED), hops_noise.py:584).  SEED b is given
 * as its 32-bit words, least significant first, in seed_words_dev[
 * seed_ptr_dev[b] .. seed_ptr_dev[b+1]) (SEED 0: one word 0; SEEDs >= 0);
 * seed_states_dev: uint64 [n_traj][4] out, as hops_noise_draw reads it. */
int hops_noise_seed_states(const uint32_t* seed_words_dev, const int32_t* seed_ptr_dev,
                           int32_t n_traj, uint64_t* seed_states_dev, void* stream);

/*
 * Shape of the batched stage kernel (batches of >= 32 trajectories): 32*nb
 * trajectories per warp task and the
 * task order: 0 = (aux, state) with the trajectory chunks innermost, 1 = chunk
 * outermost, 2 = chunk outermost then state, aux innermost, 3 = chunk
 * outermost, then the aux below n_up_prefix state by state, then the rest in
 * (aux, state) order; nb = 0 / chunk_major = -1 restore the automatic choice.
 * Process-wide setting used by the autotuner; has no counterpart in the
 * reference.
 */
int hops_stage_tuning(int32_t nb, int32_t chunk_major);

/*
 * Step fusion of hops_rk4_propagate for batches of >= 32 trajectories:
 * 1 = a scalar launch and a stage launch per RK4 stage (8 per step);
 * 2 = one cooperative persistent launch per call that runs every stage of
 * every step with grid barriers in between (used with the 128-trajectory
 * task shape, nb = 0 or 4); 0 = automatic.  A grid barrier that waits longer
 * than its time limit sets HOPS_ETIMEOUT in the status word of the
 * trajectories and the kernel returns.  Process-wide setting used by the
 * autotuner; the reference integrates one trajectory in Python
 * (integrator/integrator_rk.py:33-77).
 */
int hops_step_fusion(int32_t mode);

/*
 * Self-test of the step kernel's grid barrier (failure detection without a
 * GPU fault): a cooperative launch of n_ctas (<= SM count) CTAs, each but
 * `absent` (-1: none) passing n_sync barriers on bar (4 uint32 of device
 * memory, zeroed here); out[c] = 1 passed, 0 failed, 2 absent.  With an
 * absent CTA every other CTA gives up after limit_ns and bar[2] = 1.
 */
int hops_grid_barrier_test(uint32_t* bar, int32_t* out, int32_t n_ctas, int32_t n_sync,
                           int32_t absent, int64_t limit_ns, void* stream);


/*
 * Profiling aid: when enabled, every streaming stage-kernel launch is bracketed
 * by CUDA events on its stream; hops_kernel_timing_read synchronises, returns
 * the summed kernel time and the launch count, and clears the record.  Not
 * thread-safe; has no counterpart in the reference (timing support only).
 */
int hops_kernel_timing(int enable);
int hops_kernel_timing_read(double* total_ms, int64_t* n_launches);

/* ===================================================== host-array entry points
 * For callers that hold only host arrays (any language with a C FFI): the
 * library derives every table of hops_structure from a minimal description,
 * owns the device memory of structures and batches, and moves states, noise
 * and psi(t) between host buffers and the device.  These replace, for such a
 * caller, the reference's construction of the super-operators
 * (eom/hops_eom.py:118-218 through eom/eom_hops_ksuper.py:36-230) and the
 * state I/O of trajectory/hops_trajectory.py:253-336 (initialize) and
 * :1072-1125 (phi, psi, z_mem read-outs).
 */

/* Minimal description of one basis; all pointers are HOST pointers, complex
 * numbers interleaved (re, im) doubles.  Aux 0 must be the zero vector (the
 * physical wavefunction); the first-level aux, K2_k = -sum_m k_m(a) w_m and the
 * site-projector form are derived from the connection lists and L. */
typedef struct hops_structure_desc {
  int32_t n_hier, n_state, n_mode, n_lop;
  const int32_t* up_ptr;  /* [n_hier+1] CSR over aux of the k+1 connections */
  const int32_t* up_aux;  /* [up_ptr[n_hier]] aux a + e_m */
  const int32_t* up_mode; /* mode m (index into the mode arrays) */
  const int32_t* dn_ptr;  /* [n_hier+1] CSR over aux of the k-1 connections */
  const int32_t* dn_aux;  /* [dn_ptr[n_hier]] aux a - e_m */
  const int32_t* dn_mode; /* mode m */
  const int32_t* dn_k;    /* k_m(a) >= 1, the depth of aux a in mode m */
  const int32_t* mode_lop;  /* [n_mode] index of the mode's L operator */
  const double* mode_g;     /* [n_mode] complex g_m */
  const double* mode_w;     /* [n_mode] complex w_m (nonzero) */
  const double* lops;       /* [n_lop][n_state][n_state] complex, dense, row-major */
  const double* hamiltonian; /* [n_state][n_state] complex, dense, row-major */
  const double* lt_coef;    /* [n_lop] complex low-temperature coefficients, or NULL */
} hops_structure_desc;

typedef struct hops_structure_owned hops_structure_owned;  /* opaque */

/* Derive and upload every table (one device allocation owned by the library;
 * returns after the copy has completed).  Inputs are validated (sizes, index
 * ranges, w != 0, aux 0 without down connections) before anything is
 * allocated. */
int hops_structure_upload(const hops_structure_desc* desc, void* stream,
                          hops_structure_owned** out);
/* The structure as the entry points above take it: a host struct of device
 * pointers (hops_rk4_propagate, hops_dsystem_dt, ...) or its device copy
 * (hops_task.st, hops_flux_task.st).  Valid until hops_structure_destroy. */
const hops_structure* hops_structure_host_view(const hops_structure_owned* s);
const hops_structure* hops_structure_device_view(const hops_structure_owned* s);
int hops_structure_destroy(hops_structure_owned* s);

/* A batch of n_traj trajectories whose buffers the library allocates (and
 * frees in hops_batch_destroy); status words start at 0. */
int hops_batch_create(const hops_structure* st, int32_t n_traj, int32_t precision, int32_t eom,
                      hops_batch** out);
int hops_batch_destroy(hops_batch* bt);
/* phi_host: [n_traj][n_hier*n_state] complex128 in the reference's flat order
 * (aux-major, hops_trajectory.py:316-320); zmem_host: [n_traj][n_mode] complex128
 * or NULL for zero memory.  Resets the pending scale and the status words;
 * returns once the host buffers may be reused. */
int hops_batch_set_state_host(const hops_structure* st, hops_batch* bt, const double* phi_host,
                              const double* zmem_host, void* stream);
/* noise: [n_traj][n_lop][n_t] complex64 per noise (noise2_host may be NULL);
 * copied into batch-owned device memory. */
int hops_batch_set_noise_host(hops_batch* bt, const float* noise1_host, int32_t n_t1,
                              const float* noise2_host, int32_t n_t2, void* stream);
/* hops_rk4_propagate with psi(t) delivered to psi_out_host ([n_steps][n_traj]
 * [n_state] complex128, or NULL) and the status words to status_host ([n_traj],
 * or NULL); returns after both copies completed. */
int hops_batch_propagate_host(const hops_structure* st, hops_batch* bt, int32_t it0, int32_t di,
                              int32_t n_steps, double tau_over_hbar, double* psi_out_host,
                              int32_t* status_host, void* stream);
/* The normalised state and memory back in host buffers (layouts of
 * hops_batch_set_state_host; either may be NULL). */
int hops_batch_get_state_host(const hops_structure* st, hops_batch* bt, double* phi_host,
                              double* zmem_host, void* stream);

/*
 * No counterpart in the reference.  hops_rk4_propagate without any device
 * allocation, for callers that cannot call cudaMalloc when they step: hosts
 * whose own pool owns all device memory, and per-step callbacks that must not
 * synchronise the device.  The caller passes the state (phi in the batch
 * layout and precision, z_mem), the noise, psi_out and one int32 status word
 * per trajectory; the stage vectors, accumulator and scalar workspace live in a
 * static device array of HOPS_NOALLOC_SCRATCH_BYTES that every GPU loading the
 * library keeps until exit (it sits in a CUDA module of its own, so under lazy
 * module loading -- the CUDA 12 default -- a process holds it on a GPU only
 * after its first call there).  Problems needing more scratch than that
 * (hops_noalloc_scratch_bytes) are rejected with HOPS_EINVAL.  Every argument
 * is checked before anything is launched, so a rejected call changes nothing on
 * the device.  The status words are never cleared by the call: it only sets the
 * word of a trajectory whose norm became NaN/Inf to HOPS_ENONFINITE, so a flag
 * survives later calls until the caller zeroes the words (zero them before the
 * first call).  The first call on each device (and the first after
 * cudaDeviceReset or a change of the current context) looks the array up with
 * cudaGetSymbolAddress; make it before any stream capture.  All calls share the
 * array: calls that overlap on the GPU (different streams or threads without
 * ordering) race and corrupt each other.
 */
#define HOPS_NOALLOC_SCRATCH_BYTES (64u << 20)
size_t hops_noalloc_scratch_bytes(const hops_structure* st, int32_t n_traj, int32_t precision);
int hops_rk4_propagate_noalloc(const hops_structure* st, int32_t n_traj, int32_t precision,
                               int32_t eom, void* phi_dev, double* zmem_dev,
                               const float* noise1_dev, int32_t n_t1, const float* noise2_dev,
                               int32_t n_t2, int32_t it0, int32_t di, int32_t n_steps,
                               double tau_over_hbar, double* psi_out_dev, int32_t* status_dev,
                               void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HOPS_B200_H */
