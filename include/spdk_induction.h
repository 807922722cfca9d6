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
     * edges touching a troubled sub-cell take the first-order upwind EMF of
     * the slice-start face averages instead of the high-order one, and the
     * faces are updated again from the edges (constrained transport: the
     * discrete divergence is unchanged). 0 = the reference's behaviour.
     * Needs fallback = 1. */
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

#ifdef __cplusplus
}
#endif
#endif /* SPDK_INDUCTION_H */
