/* CPU restatement of spd_K's spectral-difference hydro step (TEST
 * INFRASTRUCTURE ONLY: the checker for the CUDA path, never the product).
 *
 * Arrays use the reference's own layout so dumps compare byte for byte:
 *   SD arrays  (t, var, k, j, i, kk, jj, ii), one ghost element per active
 *              side (src/define.hpp:99-130, src/structs.hpp:78-121);
 *   FV arrays  (var, K, J, I) with a 2-cell ghost frame
 *              (src/fv_structs.hpp:41-100).
 * The reference carries NVAR=6 slots; slot 5 only ever holds the trouble
 * aggregate or uninitialised values that never feed back into slots 0-4, so
 * the oracle stores NV=5 conserved slots (rho, mx, my, mz, E) and keeps the
 * aggregate in slot 5 of its trouble array. Parity pins: the reference
 * build under oracle/_ref (both committed goldens reproduce bitwise) and the
 * fixtures under tests/golden. */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_PERIODIC = 0, ORC_GRADFREE = 1, ORC_REFLECTIVE = 2 };
enum { ORC_ADER = 0, ORC_RK = 1 };
/* Initial conditions: ids 0-9 follow src/define.hpp:58-60; 10-12 are the
 * project's extra problems (no reference counterpart). */
enum {
    ORC_IC_SINE = 0, ORC_IC_SEDOV, ORC_IC_BLAST, ORC_IC_SQUARE, ORC_IC_SOD,
    ORC_IC_SHU_OSHER, ORC_IC_KH, ORC_IC_IMPLOSION, ORC_IC_RTI, ORC_IC_USER,
    ORC_IC_KH_NOISE, ORC_IC_QUADRANT, ORC_IC_RTI_TOP
};

typedef struct {
    int p;
    int N[3];          /* elements per direction (1 = inactive) */
    double L[3];       /* box lengths */
    int bc[3];
    int integrator;    /* ORC_ADER / ORC_RK */
    int rk_order;
    int fallback;
    double gamma, cfl;
    double g[3];
    double nad_tolerance;
    int nad_delta, nad_moore, sed, blending;
    int problem;
    /* ProblemParams (src/global.hpp:20-35) */
    double amp, v1, v2, v3, d0, d1, p0, p1, radius, sigma;
    int dir;
    double cx, cy, cz;
    /* extra problem parameters (project ICs) */
    double q[16];
    unsigned long long seed;
    /* viscosity (src/main.cpp:236-243): hydro/nu, hydro/beta (default -2/3 nu) */
    double nu, beta;
} orc_cfg;

typedef struct orc orc;

orc* orc_create(const orc_cfg* cfg);
void orc_destroy(orc* s);
/* dt of the current state (src/hydro.cpp:208-262) */
double orc_compute_dt(orc* s);
/* one full step with the given dt: ADER or SSP-RK, with or without the
 * fallback, followed by W_sp = prim(U_sp), W_cv = sp_to_cv(W_sp)
 * (src/hydro_ader.hpp:234-241) */
void orc_step(orc* s, double dt);
/* sub-steps for kernel-level parity checks */
void orc_copy_ader(orc* s);
void orc_solve_fluxes(orc* s);
void orc_update_prediction(orc* s, double dt);
void orc_update_solution(orc* s, double dt);
void orc_fv_update(orc* s, double dt);
void orc_primitives_to_cv(orc* s);
/* array access by name: U_sp W_sp W_cv U_cv U_ader_sp U_ader_fp_{x,y,z}
 * F_ader_fp_{x,y,z} troubles theta U_new U_old W_new W_old F_{x,y,z}
 * alpha_{x,y,z}; also matrices sp_to_fp dfp_to_sp sp_to_cv cv_to_sp
 * invader ader x_sp x_fp wt xt fv_faces_{x,y,z} fv_centers_{x,y,z}.
 * dims[8] receives the extents (unused trailing extents = 1). */
double* orc_array(orc* s, const char* name, int* dims);

#ifdef __cplusplus
}
#endif
