/* conan_pm.h -- C ABI of the B200 particle-mesh library (libconan_pm.so).
 *
 * Drop-in for the hot path of conan's `ic` and `run` tools: the initial
 * conditions (Gaussian random field, potential, Zel'dovich displacement) and
 * the particle-mesh leapfrog solver. Reference interfaces replaced by each
 * entry point are cited as path:line within the reference project.
 *
 * Conventions
 *  - Meshes are N^dim values with axis 0 fastest, exactly as the reference's
 *    Box<R> stores them (src/base/box.hh:51-53). Particle vectors are dim
 *    doubles per particle (mVector<double,R>, AoS), particle i sitting at
 *    lattice point i of the mass mesh (src/base/box.hh:11-24).
 *  - Host pointers are borrowed for the duration of the call. Device
 *    buffers belong to the handle and are released by the matching destroy.
 *  - Every call returns CONAN_OK (0) or an error code; conan_last_error()
 *    gives the message for the calling thread. This replaces the
 *    reference's `throw char const*` / `throw std::string`, caught in main
 *    (src/base/main.cc:101-116).
 *  - A handle is bound to one device and one CUDA stream and is not
 *    thread-safe; use one handle per host thread. Calls are stream-ordered;
 *    calls that return host data synchronise the stream.
 */
#ifndef CONAN_PM_H
#define CONAN_PM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CONAN_OK 0
#define CONAN_ERR_ARG 1
#define CONAN_ERR_ALLOC 2
#define CONAN_ERR_CUDA 3
#define CONAN_ERR_TIMEOUT 4
#define CONAN_ERR_IO 5
#define CONAN_ERR_STATE 6
#define CONAN_ERR_UNSUPPORTED 7

#define CONAN_FP32 0
#define CONAN_FP64 1

#define CONAN_GRAD_FD4 0      /* 4-point finite difference, src/run/numeric.hh:72-103 */
#define CONAN_GRAD_SPECTRAL 1 /* i k phi_hat, three extra inverse transforms */

#define CONAN_NOISE_HOST 0    /* caller supplies the white noise (e.g. mt19937) */
#define CONAN_NOISE_PHILOX 1  /* counter-based Philox4x32-10 + Box-Muller on the GPU */

/* Message for the last failed call on this thread ("" if none). */
const char *conan_last_error(void);
/* Library version string. */
const char *conan_version(void);
/* Number of visible CUDA devices (0 without a GPU). */
int conan_device_count(int *n);
/* Health check of the failure path of the kernels' bounded waits (no
 * reference counterpart: the reference has no GPU waits). One CTA on the
 * current device waits, `polls` polls at most, on a shared-memory barrier
 * that nothing completes, with the wait the TMA-staged kernels use; the wait
 * runs out, and the call returns CONAN_ERR_TIMEOUT as those kernels' host
 * check does. Any other result is a fault in that path. The context stays
 * usable. stream: cudaStream_t (NULL: default stream); returns after the
 * kernel. */
int conan_selftest_bounded_wait(unsigned polls, void *stream);

/* ------------------------------------------------------------------ ic -- */

/* Options of the `ic` tool, src/ic/main.cc:15-65 (same names and meaning).
 * `scale` is the smoothing scale in Mpc/h, `sigma` the normalisation. */
typedef struct {
    int dim;             /* --dim, 1..3 */
    int mbits;           /* --mbits, N = 1 << mbits */
    double size;         /* --size, box size L in Mpc/h */
    unsigned long seed;  /* --seed */
    double ns;           /* --ns, power-spectrum slope */
    int smooth;          /* --smooth */
    int scale_free;      /* --scale-free */
    double scale;        /* --scale */
    double sigma;        /* --sigma */
    double Omega0;       /* --Omega0 (CDM branch) */
    double H0;           /* --H0 (CDM branch) */
    int precision;       /* CONAN_FP32 or CONAN_FP64 mesh arithmetic */
    int device;          /* CUDA device ordinal */
} conan_ic_params;

/* Seeded unit white noise generated on the GPU (Philox4x32-10, Box-Muller),
 * N^dim doubles in memory order. New: the reference draws its noise with
 * std::mt19937 on the host, src/base/misc.hh:179-188. */
int conan_ic_noise(const conan_ic_params *p, double *noise_out);

/* Conan::generate_random_field, src/ic/ic.hh:14 / src/ic/ic.cc:148-161.
 * noise_or_null: N^dim unit normals in memory order (the reference's
 * mt19937 sequence reproduces its field bit-for-bit up to FFT rounding), or
 * NULL for GPU Philox noise from p->seed. density_out: N^dim doubles. */
int conan_ic_generate(const conan_ic_params *p, const double *noise_or_null,
                      double *density_out);

/* Conan::compute_potential, src/ic/ic.hh:15 / src/ic/ic.cc:163-176:
 * in place, phi = IFFT(-FFT(density)/k^2) with physical k and DC = 0. */
int conan_ic_potential(const conan_ic_params *p, double *inout);

/* Conan::compute_displacement, src/ic/ic.hh:16-17 / src/ic/ic.cc:119-146
 * without the file write: psi_out receives N^dim x dim doubles (AoS). */
int conan_ic_displacement(const conan_ic_params *p, const double *potential, double *psi_out);

/* ----------------------------------------------------------------- cic -- */

/* Options of the `cic` tool, src/cic/main.cc:17-32, with the snapshot's box. */
typedef struct {
    int dim;         /* 1..3 */
    int n_mass;      /* particles per side N of the snapshot (power of two) */
    int f;           /* --f, Eulerian mesh = f * N per side (power of two) */
    double size;     /* box size L */
    int sub_sample;  /* --sub-sample s >= 1 (power of two) */
    int device;      /* CUDA device ordinal */
} conan_cic_params;

/* cic_run<R>, src/cic/cic.hh:49-81: the density of a snapshot on the (f N)^dim
 * mesh. X: N^dim absolute positions (AoS doubles, the snapshot's `pos`
 * record). s = 1: CIC deposit of unit masses (md_cic_T, src/cic/cic.hh:8-47).
 * s > 1: the displacement X - q is interpolated linearly on the mass grid at
 * the points of an (s N)^dim grid, which are deposited with mass
 * (s N / (f N))^-dim. rho_out: (f N)^dim doubles, the sum of the deposited
 * masses per cell (no normalisation). FP64 positions and weights; integer
 * accumulation (2^-40 units), so the result does not depend on the order. */
int conan_cic(const conan_cic_params *p, const double *X, double *rho_out);

/* ----------------------------------------------------------------- fof -- */

/* Options of the `fof` tool, src/fof/fof.cc:282-333, with the snapshot's box. */
typedef struct {
    int dim;                        /* 2 or 3 (fof_run<2>, fof_run<3>) */
    unsigned long long n_particles; /* particles in the snapshot (< 2^32 - 1) */
    double size;                    /* box size L */
    double linking_length;          /* --linking-length, same units as L */
    int device;                     /* CUDA device ordinal */
} conan_fof_params;

/* fof_run<R>, src/fof/fof.cc:164-231: friends-of-friends groups of the
 * positions X (n_particles x dim doubles, AoS, the snapshot's `pos` record,
 * not wrapped). Two particles are friends when the squared length of their
 * coordinate difference, wrapped once per axis into [-L/2, L/2], is at most
 * linking_length^2 (Proximity, src/fof/fof.cc:85-99); groups are the
 * connected sets of friends. tags[i] receives particle i's group number:
 * groups are numbered from 1 in the order of their lowest particle index, as
 * the reference's `tags` array. *n_groups receives the number of groups. */
int conan_fof(const conan_fof_params *p, const double *X, unsigned long long *tags,
              unsigned long long *n_groups);

/* The same with the device buffers kept between calls (one problem size). */
typedef struct conan_fof_engine conan_fof_engine;
conan_fof_engine *conan_fof_create(const conan_fof_params *p);
void conan_fof_destroy(conan_fof_engine *h);
/* Host positions in, host tags out. */
int conan_fof_run(conan_fof_engine *h, const double *X, unsigned long long *tags, unsigned long long *n_groups);
/* Device positions in, device tags out, enqueued on `stream` (a
 * cudaStream_t, NULL = legacy default stream); returns after the group count
 * is known. */
int conan_fof_run_device(conan_fof_engine *h, const double *X, unsigned long long *tags,
                         unsigned long long *n_groups, void *stream);

/* ------------------------------------------------------------------ pm -- */

/* Parameters of the `run` tool, src/run/main.cc:20-61,82-103, as the
 * Gravity<R> solver receives them (src/run/nbody.hh:75-86). */
typedef struct {
    int dim;             /* 1..3 */
    int n_mass;          /* particles per side N (power of two) */
    int f;               /* --f, force mesh = f * N per side (power of two) */
    double size;         /* box size L in Mpc/h */
    double H0;           /* --H0 */
    double Omega_m;      /* --Omega_m */
    double Omega_L;      /* --Omega_L */
    int precision;       /* CONAN_FP32 (default product path) or CONAN_FP64 */
    int gradient;        /* CONAN_GRAD_FD4 (reference) or CONAN_GRAD_SPECTRAL */
    int periodic_gather; /* 0: reproduce the reference gather's unwrapped,
                            truncating origin (src/run/numeric.hh:19-29);
                            1: periodic floor for every particle */
    int device;          /* CUDA device ordinal */
} conan_pm_params;

typedef struct conan_pm conan_pm;

/* Builds the solver: Gravity<R>::Gravity, src/run/nbody.hh:75-86. Returns
 * NULL on failure (see conan_last_error). All device memory is allocated
 * here. */
conan_pm *conan_pm_create(const conan_pm_params *p);
void conan_pm_destroy(conan_pm *h);

/* Gravity<R>::init, src/run/nbody.hh:88-95: Zel'dovich positions at a_pos
 * and momenta at a_mom from the potential phi on the mass mesh
 * (N^dim doubles, the "potential" record of the ic file). */
int conan_pm_init(conan_pm *h, const double *phi, double a_pos, double a_mom);

/* Gravity<R>::drift, src/run/nbody.hh:122-133: X += P da / (a^2 adot(a)). */
int conan_pm_drift(conan_pm *h, double a, double da);

/* Gravity<R>::kick, src/run/nbody.hh:97-120: CIC deposit, Poisson solve,
 * CIC gather of the gradient, P -= grad(phi) da / adot(a). */
int conan_pm_kick(conan_pm *h, double a, double da);

/* Called after step i of conan_pm_run (0-based) with the scale factor a at
 * the end of the step; a nonzero return stops the run with CONAN_ERR_STATE.
 * The reference saves a snapshot after every step with (i+1) % 10 == 0
 * (src/run/nbody.hh:185-218). */
typedef int (*conan_step_cb)(conan_pm *h, unsigned step, double a, void *user);

/* The callback of conan_pm_run fires after steps with (i+1) % k == 0 and
 * after the last step (default k = 1). Steps between callbacks run as one
 * CUDA graph with the kick of one step fused to the drift of the next. */
int conan_pm_set_callback_interval(conan_pm *h, unsigned k);

/* Deposit algorithm of the handle (both give the same density, bit for bit,
 * in FP32; md_cic, src/run/numeric.hh:106-139, in both cases):
 * CONAN_DEPOSIT_SORTED      counting sort by cell, tiled integer reduction
 *                           (FP32 and FP64);
 * CONAN_DEPOSIT_LAGRANGIAN  lattice tiles summed into shared-memory windows
 *                           of integer slots, then into an integer mesh
 *                           (FP32, the FP32 default when the lattice holds
 *                           one tile per axis; CONAN_ERR_UNSUPPORTED else). */
#define CONAN_DEPOSIT_SORTED 0
#define CONAN_DEPOSIT_LAGRANGIAN 1
int conan_pm_set_deposit(conan_pm *h, int mode);
int conan_pm_get_deposit(conan_pm *h, int *mode);

/* LeapFrog::run, src/run/leapfrog.hh:33-46: init from phi (if phi is not
 * NULL) at (a0, a0 + da/2), then n x (drift(a, da); kick(a + da/2, da);
 * a += da; cb(i, a)). */
int conan_pm_run(conan_pm *h, const double *phi, double a0, double da, unsigned n,
                 conan_step_cb cb, void *user);

/* Absolute positions X and momenta P as the reference holds them
 * (N^dim x dim doubles each, AoS; either may be NULL). */
int conan_pm_get_state(conan_pm *h, double *X, double *P);
/* Replaces the particle state from absolute X and P (AoS doubles). */
int conan_pm_set_state(conan_pm *h, const double *X, const double *P, double a_pos,
                       double a_mom);
/* Scale factors of the last drift and kick (the snapshot's a-pos, a-mom,
 * src/run/nbody.hh:168-183). */
int conan_pm_scale_factors(conan_pm *h, double *a_pos, double *a_mom);

/* CIC density contrast of the current positions on the force mesh,
 * md_cic(...) - 1 (src/run/numeric.hh:106-139, src/run/nbody.hh:99-104);
 * N_f^dim doubles. */
int conan_pm_density(conan_pm *h, double *delta_out);

/* Potential of the last kick on the force mesh (N_f^dim doubles). */
int conan_pm_potential(conan_pm *h, double *phi_out);

/* Shell-averaged power spectrum of the current CIC density: bin j holds
 * modes with floor(|n| + 1/2) == j; P = <|delta_hat|^2> L^dim / N_f^(2 dim),
 * k = mean |k| of the bin, count = number of modes. */
int conan_pm_power_spectrum(conan_pm *h, int nbins, double *k, double *P, double *count);

/* Per-kernel CUDA-event timing of every launch on the handle's stream
 * (0 = off). */
int conan_pm_set_profiling(conan_pm *h, int enable);
/* Kernel i of the profile: name (<= 63 chars), launches, total milliseconds.
 * Returns CONAN_ERR_ARG when i is past the last kernel. Synchronises. */
int conan_pm_profile_entry(conan_pm *h, int i, char *name, int *launches, double *total_ms);
int conan_pm_profile_reset(conan_pm *h);
/* Device bytes held by the handle. */
int conan_pm_device_bytes(conan_pm *h, size_t *bytes);
/* Synchronises the handle's stream. */
int conan_pm_sync(conan_pm *h);
/* The handle's CUDA stream (a cudaStream_t), e.g. to record timing events
 * around library calls. */
int conan_pm_get_stream(conan_pm *h, void **stream);
/* Autotuner (no reference counterpart: the reference has one code path).
 * On the handle's current particle state -- best a clustered one, e.g.
 * half way through a run, since tile costs grow with clustering -- it times
 * every fitting candidate of each knob over leapfrog steps from a copy of
 * the state and keeps the fastest: the deposit (sorted tile variants;
 * Lagrangian window tiles; the direct two-cell window) and the
 * gradient-mesh kernel (thread per cell at 128/256/512 threads; z-marching
 * tiles). a: scale factor of the next drift; da: the step. The state and
 * scale factors are left as they were. `report` (may be NULL) receives a
 * JSON list of {knob, value, ms_per_step, chosen}. Allocates a temporary
 * copy of the particle state. */
int conan_pm_autotune(conan_pm *h, double a, double da, char *report, size_t len);

/* --------------------------------------------------------- adjoint -- */

/* Differentiable forward model: white noise -> ic -> Zel'dovich -> n
 * leapfrog steps -> final CIC density. No reference counterpart (the
 * reference has no adjoint). */
typedef struct {
    conan_ic_params ic;  /* dim, mbits, size, ns, smooth, scale, sigma used */
    conan_pm_params pm;  /* n_mass must equal 1 << ic.mbits */
    double a0, da;
    unsigned n;
    unsigned checkpoint_every; /* k: exact state stored every k steps */
} conan_diff_params;

typedef struct conan_diff conan_diff;
conan_diff *conan_diff_create(const conan_diff_params *p);
void conan_diff_destroy(conan_diff *h);
/* Device pointers of the handle's precision (float or double):
 * noise N^dim, density_out N_f^dim. `stream` is a cudaStream_t (NULL: the
 * handle's stream); the call is ordered after prior work on it. */
int conan_diff_forward(conan_diff *h, const void *noise_dev, void *density_out_dev, void *stream);
/* Gradient of a scalar loss w.r.t. the noise given its gradient w.r.t. the
 * final density of the last forward call. */
int conan_diff_backward(conan_diff *h, const void *grad_density_dev, void *grad_noise_dev,
                        void *stream);

/* -------------------------------------------------------- ensemble -- */

/* A batch of independent realisations with possibly different mesh sizes,
 * run together: every phase of a step is one launch over all members of a
 * size class, and the whole run is one CUDA graph. */
typedef struct {
    int mbits;           /* N = 1 << mbits particles and mesh cells per side */
    double size;         /* L */
    double ns;           /* spectral index */
    unsigned long seed;  /* Philox seed */
} conan_ens_member;

typedef struct {
    int dim;             /* 3 (or 2) */
    double H0, Omega_m, Omega_L;
    double sigma, scale; /* ic normalisation; smoothing off */
    double a0, da;
    unsigned n;
    int precision;
    int device;
    int autotune;        /* 1: time tile shapes on first run and keep the best */
} conan_ens_params;

typedef struct conan_ens conan_ens;
conan_ens *conan_ens_create(const conan_ens_params *p, int n_members, const conan_ens_member *m);
void conan_ens_destroy(conan_ens *h);
/* Generates every member's initial conditions (Philox noise, GRF,
 * potential, Zel'dovich) on the GPU. */
int conan_ens_init(conan_ens *h);
/* Runs all members n steps (one graph launch). */
int conan_ens_run(conan_ens *h);
/* Forward run plus the adjoint of loss = sum over members of
 * mean((delta_final - delta_target)^2), targets from seeds + 1000000;
 * writes the loss per member (host, n_members doubles). */
int conan_ens_forward_adjoint(conan_ens *h, double *loss_out);
int conan_ens_power_spectrum(conan_ens *h, int member, int nbins, double *k, double *P,
                             double *count);
int conan_ens_state(conan_ens *h, int member, double *X, double *P);
/* A member's white noise, its target density (the model run from seed +
 * 1000000) and, after conan_ens_forward_adjoint, the gradient of its loss
 * with respect to the noise: host doubles, N^dim values each; a null
 * pointer skips that field. No reference counterpart (for checking the
 * batched adjoint against a single-box one). */
int conan_ens_member_fields(conan_ens *h, int member, double *noise, double *target, double *gnoise);
/* Milliseconds of the last conan_ens_run / forward_adjoint (CUDA events). */
int conan_ens_last_ms(conan_ens *h, double *run_ms, double *adjoint_ms);
int conan_ens_total_particles(conan_ens *h, size_t *n);
/* JSON description of the size classes and the autotuner's choices. */
int conan_ens_describe(conan_ens *h, char *buf, size_t len);

/* ------------------------------------------------- no-allocation deposit -- */

/* No counterpart in the reference (its md_cic, src/run/numeric.hh:106-139,
 * is the arithmetic, not the interface). The FP32 CIC density contrast of
 * conan_pm_density, for callers that may not allocate device memory: a
 * framework that has already reserved the GPU for its own allocator, a
 * process with a fixed memory budget, a latency-bound loop that must not
 * wait on cudaMalloc/cudaFree. Allocates nothing: the integer accumulator is
 * one static device array of CONAN_DEPOSIT_STATIC_MAX_CELLS 64-bit cells
 * (16 MiB held by every GPU that loads the library), so meshes of at most
 * that many cells (128^3, 2048^2) are accepted; larger ones return
 * CONAN_ERR_ARG.
 *   d0, d1, d2: device arrays of n_mass^dim FP32 displacements in force-mesh
 *               cells, particle i at lattice point i (axis 0 fastest), as
 *               conan_pm stores them (d1, d2 unused below dim 2, 3);
 *   delta_out:  device array of (f n_mass)^dim floats;
 *   stream:     cudaStream_t of the work (NULL: the default stream).
 * The first call on a device looks up the array's address and sets kernel
 * limits for that device (the device must be current); make it before any
 * stream capture. All calls on a device share the array: calls whose GPU
 * work overlaps race; order them on one stream. Each call clears the cells
 * it uses before depositing. Needs n_mass >= 8 (3D), 16 (2D), 128 (1D). */
#define CONAN_DEPOSIT_STATIC_MAX_CELLS (1u << 21)
int conan_deposit_static(int dim, int n_mass, int f, const float *d0, const float *d1, const float *d2,
                         float *delta_out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CONAN_PM_H */
