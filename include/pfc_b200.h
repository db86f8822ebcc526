/*
 * pfc_b200.h — C ABI of the B200 (sm_100a) pseudo-spectral ETD1 stepper for
 * standard and log phase-field-crystal models in 2D.
 *
 * Plain C types only: ints, doubles, raw device pointers, and a CUDA stream
 * passed as `void*` (a cudaStream_t; NULL is the legacy default stream).
 * Every function returns PFC_OK (0) or a PFC_E_* code; pfc_last_error()
 * returns the message of the last failure on the calling thread. No C++
 * exception crosses this boundary. A plan is not thread-safe: use one plan per
 * host thread / stream at a time.
 *
 * Reference interfaces (paths relative to the reference's src/pfc_models/):
 * each entry point below names the Python call of the reference it replaces.
 */
#ifndef PFC_B200_H
#define PFC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PFC_ABI_VERSION 1

/* return codes */
#define PFC_OK 0
#define PFC_E_ARG 1         /* invalid argument or unsupported size */
#define PFC_E_CUDA 2        /* a CUDA runtime call failed */
#define PFC_E_NAN 3         /* a non-finite value was detected in the state */
#define PFC_E_TIMEOUT 4     /* a bounded device-side wait gave up */
#define PFC_E_STATE 5       /* call out of order (e.g. step before set_state) */
#define PFC_E_NOMEM 6       /* device allocation failed */

/* models */
#define PFC_MODEL_STD 0     /* nonlinearity g n^2 + n^3        (models/stdpfc) */
#define PFC_MODEL_LOG 1     /* nonlinearity ln(phi) + g phi^2 + phi^3 (models/logpfc) */

/* precision forms */
#define PFC_FP64_PLAIN 0    /* FP64 end to end */
#define PFC_FP32_MIXED 1    /* FP32 FFTs and pointwise math on the deviation psi - mean;
                               FP64 mean, ETD coefficients, near-singular log, reductions */

/* fields for pfc_get_field */
#define PFC_FIELD_N 0           /* current density field n (or phi) */
#define PFC_FIELD_MU 1          /* mu of the state at the start of the last step */
#define PFC_FIELD_LOCAL_MU 2    /* Gaussian-filtered mu, same state */
#define PFC_FIELD_LOCAL_N 3     /* Gaussian-filtered n of the state at the start of the last step */
#define PFC_FIELD_NONLIN_MU 4   /* nonlinear part of mu, same state */
#define PFC_FIELD_OF_CURRENT 0x100  /* OR-ed in: use the current state instead */

/* spectra for pfc_get_spectrum (complex128, shape (ny, nx/2+1), row-major, unnormalised rfft2) */
#define PFC_SPEC_N_HAT 0        /* rfft2 of n at the start of the last step (State.n_hat) */
#define PFC_SPEC_N_HAT_NOW 1    /* rfft2 of the current n */

/* status bits (pfc_status) */
#define PFC_STATUS_NONFINITE 1  /* a reduction met a NaN/Inf */
#define PFC_STATUS_TIMEOUT 2    /* a bounded device-side wait gave up (the step is void) */

/*
 * Problem description. Field meanings follow
 * BuildStdPFCModelParameters / BuildLogPFCModelParameters
 * (models/stdpfc/simulation.py:60-80, models/logpfc/simulation.py:51-75) and
 * Build2DGeometry (discretization/spectral/geometry_2d.py:70-88).
 * nx must be even; nx and ny may contain only the prime factors 2, 3, 5, 7, 11, 13.
 */
typedef struct pfc_problem {
  int32_t nx, ny;          /* grid points along x (fast axis) and y */
  int32_t model;           /* PFC_MODEL_* */
  int32_t precision;       /* PFC_FP64_PLAIN or PFC_FP32_MIXED */
  double lx, ly;           /* box lengths */
  double gamma, beta, q0, epsilon, g, dt;
  double small_z_tol;      /* ETD1 series threshold, kernels.py:55 (default 2e-5) */
  double min_phi;          /* log model: clamp floor when clamp_log != 0 */
  int32_t clamp_log;       /* 0: unclamped log, as the reference (logpfc/simulation.py:296) */
  int32_t flags;           /* PFC_FLAG_* bits, normally 0 */
} pfc_problem;

typedef struct pfc_plan pfc_plan;

/* Replaces BuildCupyGPU_Simulation (models/stdpfc/simulation.py:270-286,
 * models/logpfc/simulation.py:265-281) with _SimulationState.__init__
 * (models/stdpfc/simulation.py:99-164): builds the k-space operator, the ETD1
 * coefficients (kernel_etd, discretization/spectral/kernels.py:55-71) in FP64,
 * twiddle tables and the device buffers, on the current CUDA device. */
int pfc_plan_create(const pfc_problem* problem, pfc_plan** out);

/* Frees every device buffer the plan owns. */
int pfc_plan_destroy(pfc_plan* plan);

/* Replaces `sim.State.n[...] = cp.asarray(n0)` (tests/test_smoke_models.py:226-239,
 * phase_diagram adapter set_state, models/stdpfc_cpu/phase_diagram.py:262-263):
 * loads a real FP64 field of shape (ny, nx), row-major, from device memory. */
int pfc_set_state(pfc_plan* plan, const double* dev_field, void* stream);

/* Replaces reads of `sim.State.n` / `sim.n.get()` (models/stdpfc/simulation.py:283):
 * writes the current field as FP64 (ny, nx) to device memory. */
int pfc_get_state(pfc_plan* plan, double* dev_field, void* stream);

/* Replaces `for _ in range(nsteps): sim.TimeStep()` (models/stdpfc/simulation.py:225-235,
 * models/logpfc/simulation.py:220-230). Stream-ordered, no host synchronisation.
 * Whole blocks of 16 steps, and the remaining single steps, are replayed from CUDA
 * graphs that the plan records the first time it needs each (once per starting
 * ping-pong parity; with PFC_FLAG_NO_GRAPHS every kernel is launched directly). */
int pfc_step(pfc_plan* plan, int64_t nsteps, void* stream);

/* pfc_step with instrumentation: also returns the summed device time (ms) of
 * the row-pass and column-pass kernels, measured with CUDA events recorded on
 * `stream` around each launch. Synchronises the stream before returning. */
int pfc_step_timed(pfc_plan* plan, int64_t nsteps, double* ms_row, double* ms_col, void* stream);

/* Replaces CalculateFreeEnergy (models/stdpfc/simulation.py:249-268,
 * models/logpfc/simulation.py:244-263) without the full-field device-to-host copy:
 * writes three doubles to dev_out3 = {F per site, mean mu per site, mean density},
 * accumulated in compensated FP64 on the device. */
int pfc_reduce(pfc_plan* plan, double* dev_out3, void* stream);

/* Replaces State.mu / State.local_mu (models/stdpfc/simulation.py:143-155, 217-219),
 * Get_local_n (:237-247) and State.nonlin_mu, computed on demand. `w` is the
 * Gaussian width of kernel_local (kernels.py:49-52; the models use 2*pi). */
int pfc_get_field(pfc_plan* plan, int which, double w, double* dev_field, void* stream);

/* Replaces State.n_hat (models/stdpfc/simulation.py:133-137): complex128 (ny, nx/2+1). */
int pfc_get_spectrum(pfc_plan* plan, int which, double* dev_c128, void* stream);

/* Host copies of the FP64 ETD1 coefficients the plan built: A = exp(L dt) and
 * Bg = B * Gamma * lap (kernels.py:55-71 times the factor of calc_n_next_impl,
 * models/stdpfc/simulation.py:326-331), each (ny, nx/2+1) row-major. */
int pfc_get_coefficients(pfc_plan* plan, double* host_a, double* host_bg);

/* Device status bits (PFC_STATUS_*), read synchronously on the plan's last stream. */
int pfc_status(pfc_plan* plan, int32_t* out_status);

/* Launch configuration chosen for this plan, for reporting: out[0..15] =
 * {generic row: rows/CTA, threads/FFT, CTAs; generic column: columns/CTA,
 *  threads/FFT, CTAs; generic row smem, column smem bytes;
 *  1 if the power-of-two step kernels are used; their row rows/CTA, threads/CTA,
 *  CTAs, smem bytes; column threads/CTA, CTAs, smem bytes}. */
int pfc_plan_info(pfc_plan* plan, int64_t* out16);

/* problem.flags bits */
#define PFC_FLAG_GENERIC_ONLY 1   /* do not use the power-of-two step kernels */
#define PFC_FLAG_NO_GRAPHS 2      /* pfc_step launches every kernel directly */
#define PFC_FLAG_PDL 4            /* launch the power-of-two step kernels with programmatic
                                     dependent launch: each may start (and send its column's
                                     state towards L2) while the kernel before it drains */
#define PFC_FLAG_PDL_COL 128      /* as PFC_FLAG_PDL for the column step kernel only (the row
                                     kernel waits for the column kernel before it launches) */
#define PFC_FLAG_NO_ONE_CTA 8     /* step small FP64 mixed-radix grids with the two-kernel
                                     step instead of the one-CTA whole-grid kernel */
#define PFC_FLAG_EXTV 32          /* log PFC with an external potential and the re-optimised
                                     linear shift M (models/logpfc_extv/simulation.py): needs
                                     FP64 plain, the log model and clamp_log = 1 with
                                     min_phi > 0; steps with the mixed-radix two-kernel step
                                     plus two small kernels, alone (not in a batch) */
#define PFC_FLAG_TMA 64           /* with PFC_FLAG_PACKED: the row kernel stages its tile of W
                                     with the tensor memory accelerator (cp.async.bulk.tensor
                                     boxes, mbarrier completion) instead of 16-byte copies;
                                     single plans only (a batch's launch uses the copies) */
#define PFC_FLAG_PACKED 16        /* FP32-mixed power-of-two grids: the two-lane packed step
                                     kernels (two rows / two columns per thread in packed
                                     f32x2 arithmetic); PFC_FLAG_ROW_EE / COL_EE then give the
                                     values per lane (8 or 16), PFC_FLAG_ROW_TILE the rows per
                                     CTA (even) and PFC_FLAG_COL_CTA the column pairs per CTA */
/* Variant of the power-of-two step kernels (0 in a field = the precision's default):
 * complex values per thread of the row and of the column kernel (FP32: 8, 16 or 32,
 * default 32; FP64: 8 or 16, default 16) and rows per CTA of the row kernel
 * (1 .. 16; a height other than a power of two, which spreads the rows evenly over the
 * SMs, is taken where the CTA is whole multiples of it, else the plan uses the run-time
 * kernels; packed: a power of two >= 2). Other values make pfc_plan_create return
 * PFC_E_ARG. The
 * autotuner (pfc_models_b200/tune.py) measures these per grid and caches the best. */
/* OR-ed into a PFC_FLAG_ROW_EE / PFC_FLAG_COL_EE value: that pass's two-lane packed FP32
 * kernel (8 or 16 values per lane) */
#define PFC_EE_PACKED 0x80
#define PFC_FLAG_ROW_EE(e) ((int32_t)(e) << 8)
#define PFC_FLAG_COL_EE(e) ((int32_t)(e) << 16)
#define PFC_FLAG_ROW_TILE(r) ((int32_t)(r) << 24)
/* columns per CTA of the column kernel: 1, 2 or 4, at most as many as fill 256 threads
 * (0 = that many) */
#define PFC_FLAG_COL_CTA(c) ((int32_t)((c) == 4 ? 3 : (c) == 2 ? 2 : (c) == 1 ? 1 : 0) << 29)
#define PFC_FLAG_ROW_EE_OF(f) (((f) >> 8) & 0xff)
#define PFC_FLAG_COL_EE_OF(f) (((f) >> 16) & 0xff)
#define PFC_FLAG_ROW_TILE_OF(f) (((f) >> 24) & 0x1f)
#define PFC_FLAG_COL_CTA_OF(f) ((((f) >> 29) & 3) ? 1 << ((((f) >> 29) & 3) - 1) : 0)

/* The variant a plan uses: out4 = {row values per thread, column values per thread,
 * row tile rows, 1 if the power-of-two step kernels are used} (zeros when not). */
int pfc_plan_variant(pfc_plan* plan, int32_t* out4);

/* The step path of a plan: PFC_PATH_MIXED_RADIX (row and column kernels of any radix
 * set), PFC_PATH_POW2 (the power-of-two step kernels) or PFC_PATH_ONE_CTA (FP64 grids
 * whose spectra and transforms fit one CTA: every step of a pfc_step / pfc_batch_step
 * call runs in one launch per 2048 steps, one CTA per plan, the grid in shared memory;
 * the results equal the two-kernel step's). */
#define PFC_PATH_MIXED_RADIX 0
#define PFC_PATH_POW2 1
#define PFC_PATH_ONE_CTA 2
#define PFC_PATH_FAST_MIXED 3   /* the register-resident step kernels on a grid whose sides
                                   are N = ODD * 2^k (ODD = 3, 5, 7; 2^k = 16 .. 512) or
                                   powers of two, not both powers of two */
int pfc_plan_path(pfc_plan* plan, int32_t* path);

/* Kernel launches issued by this plan since creation (for accounting). */
int64_t pfc_launch_count(pfc_plan* plan);

/*
 * Batches: many independent plans stepped in lockstep, as a phase-diagram scan
 * steps hundreds of small simulations (the `ad.step(sim)` loop of
 * phase_diagram/q0star.py:271-272, run once per point of a scan; adapter step,
 * models/stdpfc_cpu/phase_diagram.py:278-279). Plans with the same sizes, step
 * kernels and nonlinearity parameters (g, clamp, min_phi) form a class; each pass
 * of a step is one launch per class with one grid row per plan, reading that
 * plan's buffers from a device table. Whole blocks of 16 steps replay a recorded
 * CUDA graph. Power-of-two and mixed-radix plans may be mixed (each kind forms its own
 * classes); all plans must use one precision and one device (current when the batch is
 * created); at most 65535 plans. The batch
 * borrows the plans: destroy it before them. Each plan keeps its own state, so
 * pfc_reduce / pfc_get_state work on any of them between batch steps.
 */
typedef struct pfc_batch pfc_batch;

int pfc_batch_create(pfc_plan* const* plans, int32_t count, pfc_batch** out);

/* Advances every plan of the batch by nsteps. Every plan must hold a state and
 * all must be at the same step parity (the same number of steps since their
 * states were set, mod 2), else PFC_E_STATE. Stream-ordered. */
int pfc_batch_step(pfc_batch* batch, int64_t nsteps, void* stream);

int pfc_batch_destroy(pfc_batch* batch);

/* Kernel launches issued by pfc_batch_step so far; number of classes. */
int64_t pfc_batch_launch_count(pfc_batch* batch);
int pfc_batch_classes(pfc_batch* batch);

/*
 * Work-queue batches: the same lockstep stepping of many plans (the ad.step loop of
 * phase_diagram/q0star.py:271-272, as for pfc_batch) in ONE persistent launch per block
 * of steps. The launch is cooperative (every CTA resident) and walks a device list of
 * work items, one row or column tile of one plan at one step, each waiting only for the
 * tiles of its own plan that it depends on (per-plan completion counters, bounded waits).
 * No counterpart in the reference. Plans must be FP32-mixed or FP64 stdPFC on the
 * one-lane power-of-two kernels, nx in 64 .. 1024 and ny in 64 .. 1024, holding the
 * values per thread the queue kernel is built with (FP32: 8 for row transforms of up
 * to 128 points and columns of up to 512, else 16; FP64: 8), with CTAs of whole warps
 * and at most 48 KiB of shared memory per pass; else PFC_E_ARG says which. Results are
 * bit-identical to pfc_step of each plan. Blocks of 16 steps replay a recorded graph.
 */
typedef struct pfc_queue pfc_queue;

int pfc_queue_create(pfc_plan* const* plans, int32_t count, pfc_queue** out);

/* As pfc_batch_step. A wait that runs out sets PFC_STATUS_TIMEOUT (pfc_queue_status)
 * and ends the launch early, leaving the plans' states undefined. */
int pfc_queue_step(pfc_queue* queue, int64_t nsteps, void* stream);

/* Synchronises the device and writes the status bits of the queue's launches so far
 * (0, or PFC_STATUS_TIMEOUT). */
int pfc_queue_status(pfc_queue* queue, int32_t* status);

/* out4: CTAs of the launch, CTAs per SM, work items per step, classes. */
int pfc_queue_info(pfc_queue* queue, int32_t* out4);

int64_t pfc_queue_launch_count(pfc_queue* queue);

int pfc_queue_destroy(pfc_queue* queue);

/* Test hook, no counterpart in the reference: makes the first column item of the next
 * launches wait for `extra` more completions than exist (0 restores the normal waits)
 * and sets the poll limit of every wait (0: the default, about a second), so that a test
 * can run a wait out and read PFC_STATUS_TIMEOUT. */
int pfc_test_queue_wait(pfc_queue* queue, int32_t extra, int64_t wait_limit);

/* The mean of `count` FP64 values at dev_field, summed with compensation
 * (Neumaier) on the device, written as one double to dev_mean. This entry point
 * has no counterpart in the reference. It exists for callers that must not
 * allocate device memory: code running while another allocator (a caching pool
 * such as PyTorch's) has reserved the GPU's memory, where an allocation here
 * could fail part-way through a run, and loops that cannot afford cudaFree,
 * which waits for all work on the device. It allocates nothing: its partial sums
 * live in a fixed array of 128 KiB that every GPU loading this library holds
 * until the process exits, so count may be at most 2^26 (an 8192 x 8192
 * field); larger counts return PFC_E_ARG. The first call on each device looks
 * up that array's device address; make that first call before any stream
 * capture. All calls share the array: calls whose kernels overlap on the GPU
 * (other streams, other host threads) race and give wrong results. Needs no
 * plan. Stream-ordered. */
int pfc_field_mean_noalloc(const double* dev_field, int64_t count, double* dev_mean, void* stream);

/* 3-mode fitness diagnostics of a crystal, on the device: what the phase-diagram
 * adapters' `diagnose` computes (src/pfc_models/models/stdpfc_cpu/phase_diagram.py:178-215;
 * logpfc_cpu/phase_diagram.py has the same code). dev_field: the plan's n (ny x nx FP64,
 * as pfc_get_state writes it); dev_spectrum: its rfft2 (as pfc_get_spectrum writes
 * PFC_SPEC_N_HAT_NOW). mode_rc: host, n_modes (row, col) index pairs into the half
 * spectrum, already scaled to the box (NumPy indexing: negative values count from the
 * end), mode_set: host, n_modes set numbers 0, 1, 2 (the 1-, 2- and 3-mode sets);
 * amplitude_sign: the structure's amplitudeSign. Writes 6 doubles to dev_out6:
 * fitness = 1 - |mean((n - n3)^2)| with n3 the field rebuilt from the mean and the set
 * amplitudes, |A|, |B|, |C| (NaN-skipping mean of |n_hat| over each set, per site),
 * the mean, and the number of strict local maxima over the 8 periodic neighbours.
 * n_modes <= 64; a pair outside the half spectrum returns PFC_E_ARG (the reference
 * raises IndexError). Uses the plan's reduction scratch: one call at a time per plan.
 * Allocates nothing, stream-ordered. */
int pfc_diagnose_modes(pfc_plan* plan, const double* dev_field, const double* dev_spectrum, const int32_t* mode_rc,
                       const int32_t* mode_set, int32_t n_modes, double amplitude_sign, double* dev_out6,
                       void* stream);

/* Frozen-field moments of a logPFC field, on the device: what FrozenField
 * (src/pfc_models/models/logpfc_cpu/phase_diagram.py:465-505) computes for frozen_q.
 * dev_field / dev_spectrum as for pfc_diagnose_modes; lx_ref, ly_ref: the q00 = 1 box of the
 * cell (Mx 4 pi / sqrt 3, My 4 pi). Writes 4 doubles to dev_out4: A_n = sum over the full
 * fft2 grid of |phi_hat_k / N|^2 |k_ref|^(2n), n = 0, 1, 2, and the local term
 * mean(phi ln phi + temp/2 phi^2 + g/3 phi^3 + v0/4 phi^4). Uses the plan's reduction
 * scratch: one call at a time per plan. Allocates nothing, stream-ordered. */
int pfc_frozen_moments(pfc_plan* plan, const double* dev_field, const double* dev_spectrum, double lx_ref,
                       double ly_ref, double temp, double g, double v0, double* dev_out4, void* stream);

/* Defect screen of a logPFC field, on the device: what defect_diagnostics
 * (src/pfc_models/models/logpfc_cpu/phase_diagram.py:512-528) computes for frozen_q.
 * dev_field / dev_spectrum as for pfc_diagnose_modes; lx_ref, ly_ref as for
 * pfc_frozen_moments. Writes 4 doubles to dev_out4: the peak spread (max - min) / mean
 * of the heights above the mean of the sites >= their 8 periodic neighbours and above
 * the mean, the sub-q ratio (largest |phi_hat|^2 at 0 < |k_ref| < 0.95 over the largest
 * at k != 0), the peak count, and 0; NaN where there is no peak or no power. Uses the
 * plan's reduction scratch: one call at a time per plan. Allocates nothing,
 * stream-ordered. */
int pfc_defect_screen(pfc_plan* plan, const double* dev_field, const double* dev_spectrum, double lx_ref,
                      double ly_ref, double* dev_out4, void* stream);

/* Vacancy tracking on the device: for each of `count` vacancies, the position that
 * _VacancyTracker.LocateVacancy (src/pfc_models/analysis/vacancy_tracker.py:22-60)
 * computes from a local (coarse-grained) density field, so that a tracker needs no
 * copy of the field to the host. dev_field: ny x nx FP64, row-major, the layout
 * pfc_get_field writes (e.g. PFC_FIELD_LOCAL_N). dev_xy: 2*count doubles (x, y) in
 * length units (pixel * dx, pixel * dy), read as the previous positions and
 * overwritten with the new ones. dev_status: count int32, 0 = located; where the
 * reference raises, the position is left as it was and the status is 1 for its
 * ValueError (a non-finite position, a 3 x 3 neighbourhood that NumPy slicing leaves
 * empty) or 2 for its IndexError (a cross neighbour past the last row or column). Bit-identical to the reference's FP64 arithmetic. Needs no plan,
 * allocates nothing, stream-ordered. */
int pfc_locate_vacancies(const double* dev_field, int32_t nx, int32_t ny, double dx, double dy, double* dev_xy,
                         int32_t count, int32_t* dev_status, void* stream);

/* Copies the last error message of this thread into buf (NUL-terminated). */
int pfc_last_error(char* buf, size_t len);

int pfc_abi_version(void);

/* ---- log PFC with an external potential (plans created with PFC_FLAG_EXTV) ----
 * The reference's logpfc_extv model (models/logpfc_extv/simulation.py) on the log stepper:
 * every pfc_step step does what its TimeStep (:301-330) does. ValidatePhiRange (:375-405)
 * reads the field's range and, on the first step or when the range leaves the last
 * optimised one by more than the floor / ceiling tolerances (relative, 0.1 by default),
 * OptimizeM (:332-373) sets M = (N(max) - N(min)) / (max - min), N(x) = g x^2 + x^3 + ln x,
 * and rebuilds the ETD1 coefficients of beta (q0^2 + lap)^2 + eps + M; the update is
 * phi_hat' = A_M phi_hat + B_M (Gamma lap (N_hat - M phi_hat) + lap V_hat) with the clamped
 * log (:524-577). The decision, M and the rebuild run on the device, stream-ordered. */

/* Replaces _ExternalPotential.SetPotential / SetGaussianDipolePotential /
 * SetPotential_alongX / SetDoubleVacancyAlongX_TanhPotential (models/logpfc_extv/
 * external_potentials.py:109-131): V as a real FP64 (ny, nx) device field; its rfft2 is
 * taken on the device and the next step rebuilds the forcing B lap V_hat. */
int pfc_set_potential(pfc_plan* plan, const double* dev_v, void* stream);

/* Reads the M-shift state (State.M, State.phi_min, State.phi_max of
 * models/logpfc_extv/simulation.py:130-144) after synchronising: out6 = {M, phi_min,
 * phi_max of the last optimisation (NaN before the first step), the field's min and max
 * seen by the last step, number of optimisations}. */
int pfc_extv_state(pfc_plan* plan, double* host_out6);

/* Sets State.phi_floor_tol / State.phi_ceiling_tol (models/logpfc_extv/simulation.py:143-144). */
int pfc_extv_set_tolerances(pfc_plan* plan, double floor_tol, double ceiling_tol);

/* Testing the bounded device wait (no counterpart in the reference, whose CuPy path has
 * no device waits): on a plan whose row pass stages its tile by TMA (PFC_FLAG_TMA), the
 * following steps make that pass's mbarrier expect `extra_bytes` more than the tile
 * (a multiple of 16, 0 restores the normal count), so its wait runs out after
 * `wait_limit` polls (0: the default limit); the pass then leaves without computing and
 * sets PFC_STATUS_TIMEOUT, which pfc_status reads, and the context stays usable. The
 * plan's recorded graphs are dropped so the next steps use the new arguments. */
int pfc_test_tma_wait(pfc_plan* plan, int32_t extra_bytes, int32_t wait_limit);

#ifdef __cplusplus
}
#endif

#endif /* PFC_B200_H */
