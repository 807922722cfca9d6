/* spdk.h - C ABI of the spd_K B200 solver (libspdk_cuda.so).
 *
 * Plain C types only: a caller binds these with ctypes, cgo, JNI or a C++
 * host exactly as it would the reference's C++ entry points. All device
 * buffers are owned by the library; host buffers are owned by the caller.
 * Every function returns 0 on success, a negative SPDK_E* code on a usage
 * or CUDA error, and a positive code for a device-detected numerical fault.
 * spdk_last_error() gives the message of the last failure on this thread.
 *
 * Correspondence with the reference (paths inside davidvelasco07/spd_K):
 *   spdk_hydro_config      RunConfig + ProblemParams + <mesh> (src/global.hpp:20-60,
 *                          src/main.cpp:126-189)
 *   spdk_hydro_create      Hydro_ader::Hydro_ader (src/hydro_ader.hpp:76-213)
 *   spdk_hydro_step        one pass of the loop body of Hydro_ader::time_evolution
 *                          (src/hydro_ader.hpp:234-243): ADER_step (:291-305) or
 *                          RK_step (:313-325), compute_primitives, transform_sp_to_cv,
 *                          compute_dt
 *   spdk_hydro_evolve      Hydro_ader::time_evolution (src/hydro_ader.hpp:215-273)
 *   spdk_hydro_get_dt      compute_dt result (src/hydro.cpp:208-262)
 */
#ifndef SPDK_H
#define SPDK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPDK_ABI_VERSION 1

enum {
    SPDK_OK = 0,
    SPDK_E_ARG = -1,       /* invalid argument / unsupported configuration */
    SPDK_E_CUDA = -2,      /* CUDA runtime error (message in spdk_last_error) */
    SPDK_E_NOMEM = -3,     /* device allocation failed */
    SPDK_E_STATE = -4,     /* call out of order */
    SPDK_E_IO = -5         /* a file could not be read or written */
};

enum { SPDK_BC_PERIODIC = 0, SPDK_BC_GRADFREE = 1, SPDK_BC_REFLECTIVE = 2 };
enum { SPDK_INTEGRATOR_ADER = 0, SPDK_INTEGRATOR_RK = 1 };

/* initial conditions: 0-9 are the reference's (src/define.hpp:58-60),
 * 10-12 are project problems without a reference counterpart */
enum {
    SPDK_IC_SINE_WAVE = 0, SPDK_IC_SEDOV = 1, SPDK_IC_SPHERICAL_BLAST = 2,
    SPDK_IC_SQUARE = 3, SPDK_IC_SOD = 4, SPDK_IC_SHU_OSHER = 5,
    SPDK_IC_KELVIN_HELMHOLTZ = 6, SPDK_IC_IMPLOSION = 7, SPDK_IC_RTI = 8,
    SPDK_IC_USER = 9, SPDK_IC_KH_NOISE = 10, SPDK_IC_QUADRANT = 11,
    SPDK_IC_RTI_TOP = 12
};

/* arithmetic of the solver */
enum {
    SPDK_PRECISION_FP64 = 0,  /* plain form: FP64, reference operation order */
    SPDK_PRECISION_FP32 = 1   /* precision form: FP32 state, transforms and fluxes
                                 (FMA contraction allowed); FP64 for pressure
                                 recovery, the detector's bound comparisons and
                                 the dt reduction. No reference counterpart. */
};

typedef struct spdk_hydro_config {
    int p;                 /* polynomial degree, 1..7 */
    int N[3];              /* elements per direction; N=1 marks an inactive direction */
    double L[3];           /* box lengths */
    int bc[3];             /* SPDK_BC_* per direction */
    int integrator;        /* SPDK_INTEGRATOR_* */
    int rk_order;          /* 1, 2 or 3 (SSP-RK) */
    int fallback;          /* a-posteriori NAD + MUSCL-Hancock fallback */
    double gamma, cfl;
    double g[3];           /* constant gravitational acceleration */
    double nad_tolerance;
    int nad_delta, nad_moore, sed, blending;
    int problem;           /* SPDK_IC_* */
    double amp, v1, v2, v3, d0, d1, p0, p1, radius, sigma;
    int dir;
    double cx, cy, cz;
    double q[16];          /* extra parameters of project problems */
    unsigned long long seed;
    int precision;         /* SPDK_PRECISION_* */
    int device;            /* CUDA device ordinal */
    double nu;             /* kinematic viscosity; > 0 switches the viscous terms on
                              (hydro/nu, src/main.cpp:236; src/hydro.cpp:420-572) */
    double beta;           /* bulk coefficient (hydro/beta, default -2/3 nu, src/main.cpp:237) */
    /* slab of a domain-decomposed run (0, 0: the whole domain). The solver
     * holds element rows [slab_lo, slab_lo + N[a]) of a domain of slab_n rows
     * along its slowest active axis a (y in 2D, z in 3D), which must have a
     * non-periodic boundary; geometry and initial condition are those rows of
     * the whole domain's. Halo rows are refreshed by the caller
     * (spdk_hydro_rows) and the step's dt restricted to the owned rows
     * (spdk_hydro_slab_dt). No counterpart in the reference (its MPI path is
     * disabled, src/boundary.cpp:3-24). */
    int slab_lo, slab_n;
} spdk_hydro_config;

typedef struct spdk_hydro spdk_hydro;

typedef struct spdk_hydro_info {
    int ndim, p, n_points, nvar;  /* points per element, conserved slots (ndim+2) */
    int N[3];
    long long n_elements;
    long long n_dof;              /* active solution points */
    int n_time_slices;            /* p+1 (ADER) or 1 (RK) */
    int launches_per_step;        /* kernels launched by one spdk_hydro_step */
    size_t device_bytes;          /* device memory held by the solver */
} spdk_hydro_info;

/* fields for spdk_hydro_read / spdk_hydro_write; layout [element][var][point]
 * with element = (k*N[1] + j)*N[0] + i over active elements and
 * point = (kk*n + jj)*n + ii, n = p+1 */
enum {
    SPDK_FIELD_U_SP = 0,      /* conserved state at solution points */
    SPDK_FIELD_W_CV = 1,      /* primitive sub-cell averages (written every step) */
    SPDK_FIELD_TROUBLES = 2,  /* last fallback slice's trouble flags, 0/1 per sub-cell */
    SPDK_FIELD_THETA = 3,     /* last fallback slice's blending factor per sub-cell */
    SPDK_FIELD_ELEMENT_TROUBLES = 4,  /* per element: 1 if NAD/SED/PAD flagged a sub-cell in any slice of the last step */
    SPDK_FIELD_ELEMENT_PREDICTED = 5  /* per element: the learned indicator's a-priori flag of the last step */
};

const char* spdk_last_error(void);
int spdk_abi_version(void);

int spdk_hydro_create(const spdk_hydro_config* cfg, spdk_hydro** out);
int spdk_hydro_destroy(spdk_hydro* h);
int spdk_hydro_get_info(const spdk_hydro* h, spdk_hydro_info* info);

/* time step for the next spdk_hydro_step (blocks on the solver stream) */
int spdk_hydro_get_dt(spdk_hydro* h, double* dt);
/* impose the next dt (the reference's output clamping) */
int spdk_hydro_set_dt(spdk_hydro* h, double dt);
/* one step with the current dt; the next dt is reduced on the device.
 * Asynchronous with respect to the host. */
int spdk_hydro_step(spdk_hydro* h);
/* n steps, each with the dt its predecessor computed, replayed from a CUDA
 * graph; asynchronous */
int spdk_hydro_steps(spdk_hydro* h, int n);
/* time_evolution: steps until t >= t_end; dt_output > 0 clamps dt to hit
 * output times exactly. Returns the number of steps and the final t. The
 * loop runs on the device: each step's last kernel advances t, clamps the
 * next dt and closes a stop gate at t_end (the host loop's FP64 operations,
 * so the steps and states equal a host loop's bit for bit); the host
 * launches captured steps in batches and reads the loop state once per
 * batch. Steps launched past the gate do nothing. The loop starts at t = 0
 * with the first output time dt_output, as a fresh run does. */
int spdk_hydro_evolve(spdk_hydro* h, double t_end, double dt_output, long long* steps, double* t);
/* the same loop resumed at t0 with the next output time t_output0 (ignored
 * when dt_output <= 0): after spdk_hydro_restore, pass the checkpoint's t and
 * t_output from spdk_checkpoint_info to continue the interrupted run. *t
 * receives the final time (t0 when t0 >= t_end: no step is taken). */
int spdk_hydro_evolve_from(spdk_hydro* h, double t0, double t_output0, double t_end, double dt_output,
                           long long* steps, double* t);
int spdk_hydro_sync(spdk_hydro* h);
/* the CUDA stream (cudaStream_t) every solver launch is ordered on */
int spdk_hydro_get_stream(spdk_hydro* h, void** stream);
/* kernel kinds timed by spdk_hydro_profile */
enum {
    SPDK_KERNEL_PREDICT = 0,  /* Picard predictor pass */
    SPDK_KERNEL_CORRECT = 1,  /* corrector / RK stage + W_cv + dt */
    SPDK_KERNEL_FLUX = 2,     /* last Picard pass writing FV face fluxes */
    SPDK_KERNEL_DETECT = 3,   /* NAD/SED/PAD */
    SPDK_KERNEL_THETA = 4,    /* theta blending (computed inside the update kernel: no launches) */
    SPDK_KERNEL_UPDATE = 5,   /* fallback fluxes + FV update (+ W_cv, dt) */
    SPDK_KERNEL_OTHER = 6,    /* dt hand-over */
    SPDK_KERNEL_KINDS = 7
};
/* run n steps without graph replay, bracketing every launch with CUDA events
 * on the solver stream; adds the device time (ms) and launch count of each
 * kernel kind to ms[kind] and launches[kind] (arrays of SPDK_KERNEL_KINDS) */
int spdk_hydro_profile(spdk_hydro* h, int n, double* ms, long long* launches);
/* copy a field to / from host memory (count = number of doubles); writing
 * SPDK_FIELD_U_SP recomputes W_cv and dt */
int spdk_hydro_read(spdk_hydro* h, int field, double* host, size_t count);
int spdk_hydro_write(spdk_hydro* h, int field, const double* host, size_t count);
/* domain integrals of the conserved variables (rho, m_1..m_D, E; count =
 * D + 2): the sub-cell averages U_cv (sp_to_cv of U_sp along each
 * direction) times the sub-cell volumes, summed over the active cells in
 * FP64 with compensated (Neumaier) summation in a fixed order, in both forms
 * (the reference's mass diagnostic, src/hydro_ader.hpp:481-497, for every
 * variable). Ordered after the solver's pending work; blocking. Slab
 * solvers (slab_n != 0), whose rows include halo rows, are rejected. */
int spdk_hydro_conserved(spdk_hydro* h, double* sums, int count);

/* Domain decomposition (slabs; no counterpart in the reference).
 * spdk_hydro_rows copies element rows [lo, hi) of U_sp along the slab axis
 * between the solver and a caller DEVICE buffer of (hi-lo) rows in the
 * solver's arithmetic (to_solver = 0: solver -> buffer, 1: buffer -> solver),
 * ordered on the solver stream, asynchronous. spdk_hydro_slab_dt sets the
 * next dt to the minimum over the element rows [lo, hi) (the owned rows) of
 * the CFL / diffusion candidates of the current W_cv, on the device; read it
 * with spdk_hydro_get_dt, reduce across slabs, impose it with
 * spdk_hydro_set_dt. */
int spdk_hydro_rows(spdk_hydro* h, int to_solver, int lo, int hi, void* device_buffer);
int spdk_hydro_slab_dt(spdk_hydro* h, int lo, int hi);

/* Checkpoint / restart (no counterpart in the reference, whose runs start
 * from the initial condition). A checkpoint file holds U_sp in the solver's
 * own arithmetic (raw doubles or floats), the next step's dt as the device
 * holds it (after any output clamping) and the caller's time_evolution
 * bookkeeping; restoring it into a solver created from the same
 * configuration and stepping on gives the same states, bit for bit, as the
 * run that was never interrupted. Little-endian binary: a 256-byte header
 * (magic "SPDKCKP1") and the state. */
typedef struct spdk_checkpoint_info {
    double t;             /* simulated time of the state */
    double t_output;      /* the caller's next output time */
    long long steps;      /* steps taken so far */
    long long outputs;    /* output files written so far */
} spdk_checkpoint_info;
/* blocking: waits for the solver's stream, then writes the file */
int spdk_hydro_checkpoint(spdk_hydro* h, const char* path, const spdk_checkpoint_info* info);
/* asynchronous: snapshots the state on the solver's stream (device copy)
 * and returns; a copy stream and a writer thread move it to the file while
 * the caller keeps stepping. One checkpoint is in flight at a time (a second
 * call first waits for the first); spdk_hydro_checkpoint_wait returns the
 * status of the write, and destroy waits too. */
int spdk_hydro_checkpoint_async(spdk_hydro* h, const char* path, const spdk_checkpoint_info* info);
int spdk_hydro_checkpoint_wait(spdk_hydro* h);
/* load a checkpoint (configuration checked against the solver's); fills
 * info when not NULL */
int spdk_hydro_restore(spdk_hydro* h, const char* path, spdk_checkpoint_info* info);
/* read a checkpoint's header without a solver or a GPU: its bookkeeping,
 * precision (SPDK_PRECISION_*), order, element counts and time-stepping
 * (integrator, RK order); any output pointer may be NULL */
int spdk_checkpoint_peek(const char* path, spdk_checkpoint_info* info, int* precision, int* p, int N[3],
                         int* integrator, int* rk_order);

/* Host-only set-up (no GPU needed).
 * spdk_build_matrices: the transform matrices of degree p, as the reference
 * builds them in Hydro_ader::Hydro_ader (src/hydro_ader.hpp:129-141, from
 * src/polynomials.cpp): sp_to_fp [(p+2)(p+1)], dfp_to_sp [(p+1)(p+2)],
 * sp_to_cv and cv_to_sp [(p+1)^2], invader [(p+1)^2, ADER only] and the time
 * weights wt [p+1]. Any output pointer may be NULL. */
int spdk_build_matrices(int p, int ader, double* sp_to_fp, double* dfp_to_sp, double* sp_to_cv,
                        double* cv_to_sp, double* invader, double* wt);
/* spdk_initial_wcv: the initial primitive sub-cell averages of a
 * configuration (src/initial_conditions.cpp:179-228) in the solver layout
 * [element][var][point]; count = elements * (ndim+2) * points. */
int spdk_initial_wcv(const spdk_hydro_config* cfg, double* out, size_t count);
/* spdk_fv_faces: the FV sub-cell face coordinates of one direction, ghost
 * frame included (the reference's dimension::fv_faces, src/structs.hpp:40-75):
 * count = N (p+1) + 5 for an active direction, 1 for an inactive one. */
int spdk_fv_faces(int N, int p, double L, int active, double* out, size_t count);

/* Allocation-free step. No counterpart in the reference: it serves callers
 * that cannot allocate device memory when they advance the solution -- a
 * host that owns all device memory through its own pool, a plugin running
 * inside a stream capture it does not own, a real-time loop that cannot
 * absorb the synchronisation an allocation may cause. It runs one ADER or
 * SSP-RK step without the fallback for configuration cfg on caller-owned
 * device buffers: u_in / u_out [element][var][point] (may be the same
 * buffer), wcv_out (nullable) receives W_cv, *dt_inout holds this step's dt
 * on entry and the next dt on exit; all work is ordered on `stream` (a
 * cudaStream_t). Working storage is one fixed array inside the library of
 * SPDK_NOALLOC_SCRATCH_BYTES bytes, held on every GPU that loads the library
 * until exit; problems that need more (ADER: 2(p+1) states, RK: 2 states)
 * are rejected with SPDK_E_ARG. The first call on a device, with that device
 * current, resolves the array's device address and sets kernel attributes:
 * make it before any stream capture. Calls share the array, so calls that
 * overlap on the GPU race; order them on one stream. No call allocates.
 * Slab configurations (slab_lo, slab_n != 0) are rejected with SPDK_E_ARG.
 * Device-detected faults: every call clears the array's status word when it
 * starts; if a bounded shared-memory staging wait runs out during the call,
 * *dt_inout receives NaN instead of the next dt (the state it leaves is not
 * to be trusted) and the status word keeps the fault bit. */
#define SPDK_NOALLOC_SCRATCH_BYTES (16u << 20)
int spdk_hydro_step_noalloc(const spdk_hydro_config* cfg, const double* u_in, double* u_out, double* wcv_out,
                            double* dt_inout, void* stream);
/* Status word of the last spdk_hydro_step_noalloc call on the current
 * device: 0 = clean, bit 0 (value 1) = a staging wait timed out. Blocking:
 * it reads the word on `stream` (a cudaStream_t; order it after the step)
 * and waits for that stream. 0 when no step ran on the device yet. No
 * counterpart in the reference; allocates nothing. */
int spdk_hydro_noalloc_status(int* status_out, void* stream);

/* Measurement of the FP32 Picard pass's divergence contraction on CUDA cores
 * against tensor cores (no counterpart in the reference): for count
 * element-variables of a 2D p = 3 run, dudt[ev][jj][ii] = sum_ll
 * fx[ev][jj][ll] D[ii][ll] + fy[ev][ii][ll] D[jj][ll], D = dfp_to_sp; fx, fy
 * are [count][4][5] and dudt [count][4][4] FP32 device arrays. mode 0: FP32
 * FMAs (the Picard pass's form); mode 1: mma.sync m16n8k8 TF32 with the
 * 3xTF32 split and FP32 accumulation. Asynchronous on `stream`. */
int spdk_study_divergence(int mode, int p, long long count, const float* fx, const float* fy, float* dudt,
                          void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SPDK_H */
