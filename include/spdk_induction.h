/* spd_K induction solver on B200 (libspdk_cuda.so): the reference's
 * Induction_ader (src/induction_ader.hpp:1-644, src/induction.cpp:52-720).
 *
 * The magnetic field is kept on the element faces (B_x at x flux points,
 * B_y at y flux points, B_z at z flux points) and advanced with the edge
 * electric field E = v x B: per ADER Picard pass, E at the edge points from
 * the interpolated face fields (compute_E), ghost-element fill, upwind edge
 * Riemann solve (E_riemann_solver), and dB/dt = curl E through dfp_to_sp
 * (update_B_prediction / update_B_solution); with the fallback switched on
 * the corrector runs on the sub-cell faces instead (edge_integral,
 * fv_update_B_solution) and the NAD/SED detector flags B (the reference
 * applies no fallback flux for B). SSP-RK1/2/3 stages as in RK_step. The
 * velocity field is the reference's fixed v = (1, 1, 0) and the initial
 * vector potential its magnetic loop (A_z = 1e-3 (0.3 - r), r < 0.3, about
 * the box centre). 3D only, FP64, reference operation order: the outputs
 * are bit-identical to the reference's CPU build.
 *
 * Replaces the Induction_ader object that src/main.cpp:227-249 builds for
 * job/system = induction. Status codes and spdk_last_error() as in spdk.h.
 */
#ifndef SPDK_INDUCTION_H
#define SPDK_INDUCTION_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spdk_induction_config {
    int p;               /* polynomial degree, 1..7 */
    int N[3];            /* elements per direction; all three active */
    double L[3];         /* box lengths */
    int bc[3];           /* SPDK_BC_* of spdk.h */
    int integrator;      /* SPDK_INTEGRATOR_ADER / _RK */
    int rk_order;        /* 1..3 for RK */
    int fallback;        /* FV corrector + trouble detection */
    double cfl;
    double nu;           /* resistivity: caps dt only (Ohmic terms are compiled out in the reference) */
    double nad_tolerance;
    int nad_delta, nad_moore, sed;
    int device;
    /* apply a fallback where the corrector detects troubles (no reference
     * counterpart: the reference detects and stops there). Each slice's
     * candidate face update is judged by the detector as in the reference;
     * then the edges touching a troubled sub-cell take the first-order
     * upwind EMF of the slice-start face averages instead of the high-order
     * one, and the slice-start faces are updated again from the edges
     * (constrained transport: the discrete divergence is unchanged).
     * Bit-identical to the reference built with that step added to its
     * corrector. 0 = the reference's behaviour. Needs fallback = 1. */
    int fallback_apply;
} spdk_induction_config;

typedef struct spdk_induction spdk_induction;

/* fields for spdk_induction_read, in the reference's layout with ghost
 * elements (the bytes its Write() dumps) */
enum {
    SPDK_IND_FIELD_B2_CV = 0,     /* (4, Nz+2, Ny+2, Nx+2, n, n, n): Bx, By, Bz, |B|^2 sub-cell averages */
    SPDK_IND_FIELD_TROUBLES = 1,  /* (4, F, F, F), F = N n + 4 (fallback only) */
    SPDK_IND_FIELD_BX_FP = 2,     /* (Nz+2, Ny+2, Nx+2, n, n, n+1) */
    SPDK_IND_FIELD_BY_FP = 3,     /* (Nz+2, Ny+2, Nx+2, n, n+1, n) */
    SPDK_IND_FIELD_BZ_FP = 4      /* (Nz+2, Ny+2, Nx+2, n+1, n, n) */
};

int spdk_induction_create(const spdk_induction_config* cfg, spdk_induction** out);
int spdk_induction_destroy(spdk_induction* s);
/* the step size the next step uses (the reference's Dt, or a clamped value) */
int spdk_induction_get_dt(spdk_induction* s, double* dt);
int spdk_induction_set_dt(spdk_induction* s, double dt);
/* one ADER step / one SSP-RK step (asynchronous on the solver's stream) */
int spdk_induction_step(spdk_induction* s);
/* Induction_ader::time_evolution: steps until t >= t_end, dt reset to Dt
 * after every step and clamped to output times when dt_output > 0 */
int spdk_induction_evolve(spdk_induction* s, double t_end, double dt_output, long long* steps, double* t);
int spdk_induction_field_size(spdk_induction* s, int field, size_t* count);
/* blocking copy of a field to host doubles (B2_cv is computed on demand) */
int spdk_induction_read(spdk_induction* s, int field, double* host, size_t count);

/* ---------------------------------------------------------------------------
 * 2D induction solver: the field-loop advection of the induction solver on a
 * plane field B = (B_x, B_y, 0) with a uniform in-plane velocity, where only
 * the edge EMF E_z is nonzero. No counterpart in the reference as a 2D code
 * (Induction_ader requires three active directions,
 * src/induction_ader.hpp:106-110, and fixes v = (1, 1, 0) and the loop centre,
 * src/induction.cpp:28-31, src/initial_conditions.cpp:235-249): it computes
 * what a quasi-2D reference run computes (nx3 = 2, periodic z, induction/nu =
 * 0, the reference's velocity() and magnetic_loop() returning the values
 * given here), and its FP64 face fields are that run's. Box
 * [0, L_x] x [0, L_y], periodic; ADER or SSP-RK1/2/3; no fallback (the
 * reference detects troubles but applies no fallback for B). Same status
 * codes as spdk.h.
 * ------------------------------------------------------------------------- */
typedef struct spdk_induction2d_config {
    int p;                    /* polynomial degree, 1..7 */
    int N[2];                 /* elements along x and y (>= 2) */
    double L[2];              /* box lengths */
    int integrator;           /* SPDK_INTEGRATOR_ADER / _RK (spdk.h) */
    int rk_order;             /* 1..3 for RK */
    double cfl;
    double velocity[2];       /* uniform advection velocity (v_x, v_y) */
    double loop_center[2];    /* magnetic loop: A_z = A0 (R - r) for r <= R about the centre */
    double loop_A0, loop_R;
    int precision;            /* SPDK_PRECISION_FP64 (reference arithmetic) or _FP32 (FP32 state) */
    int device;
} spdk_induction2d_config;

typedef struct spdk_induction2d spdk_induction2d;

typedef struct spdk_induction2d_info {
    int p, N[2];
    long long n_elements;
    long long n_face_values;      /* B_x and B_y values: 2 E (p+1)(p+2) */
    int n_time_slices;
    int launches_per_step;
} spdk_induction2d_info;

enum {
    SPDK_IND2_FIELD_BX = 0,     /* [element][jj][ix]: (p+1) x (p+2) per element, element = j Nx + i */
    SPDK_IND2_FIELD_BY = 1,     /* [element][jy][ii]: (p+2) x (p+1) */
    SPDK_IND2_FIELD_B2_CV = 2   /* [element][4][jj][ii]: the quasi-2D reference run's B2_cv
                                   (Bx, By, Bz, |B|^2 sub-cell averages) at its z sub-cell row 0 */
};

int spdk_induction2d_create(const spdk_induction2d_config* cfg, spdk_induction2d** out);
int spdk_induction2d_destroy(spdk_induction2d* s);
int spdk_induction2d_get_info(const spdk_induction2d* s, spdk_induction2d_info* info);
/* the step size of the next step (the reference's Dt unless clamped) */
int spdk_induction2d_get_dt(spdk_induction2d* s, double* dt);
int spdk_induction2d_set_dt(spdk_induction2d* s, double dt);
/* one ADER / SSP-RK step, asynchronous on the solver's stream */
int spdk_induction2d_step(spdk_induction2d* s);
int spdk_induction2d_sync(spdk_induction2d* s);
/* the CUDA stream (cudaStream_t) every launch of the solver is ordered on */
int spdk_induction2d_get_stream(spdk_induction2d* s, void** stream);
/* Induction_ader::time_evolution (src/induction_ader.hpp:273-330): steps of
 * Dt from t = 0 until t >= t_end, clamped to output times when dt_output > 0 */
int spdk_induction2d_evolve(spdk_induction2d* s, double t_end, double dt_output, long long* steps, double* t);
/* blocking copy of a field to host doubles */
int spdk_induction2d_read(spdk_induction2d* s, int field, double* host, size_t count);

#ifdef __cplusplus
}
#endif
#endif /* SPDK_INDUCTION_H */
