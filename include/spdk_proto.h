/* spd_K prototype-level C ABI (libspdk_cuda.so).
 *
 * One export per function group of the reference's src/prototypes.hpp,
 * with the reference's name prefixed by spdk_, the same argument order and
 * argument meaning, so that a host that drives the reference's free
 * functions (the way Hydro_ader does, src/hydro_ader.hpp:215-586) can call
 * these instead. Differences a binding must know:
 *
 *  - Arrays are views of DEVICE memory in the reference's own layout,
 *    LayoutRight: SD arrays (t, var, k, j, i, kk, jj, ii) with one ghost
 *    element per active side (src/define.hpp:99-130), FV arrays
 *    (var, K, J, I) with a two-cell ghost frame (src/fv_structs.hpp:41-100),
 *    matrices (rows, cols), vectors (n). The caller owns every buffer.
 *  - The reference's global cfg (src/global.hpp:41-60) is passed explicitly
 *    as spdk_proto_cfg.
 *  - Every call is enqueued on `stream` (a cudaStream_t, NULL = legacy
 *    default stream) and returns at once; status 0 = ok, < 0 = argument or
 *    launch error (message in spdk_last_error()).
 *  - compute_dt writes its minimum to a device double instead of returning
 *    it, so a step can stay on the device.
 *  - Physics slots are rho, m_x, m_y, m_z, E (0..4) of the var extent;
 *    further slots (the reference's bookkeeping slot 5) are left untouched
 *    by the pointwise physics and carried by the transforms.
 *
 * Every function is FP64 and follows the reference's operation order (the
 * library is built without FMA contraction), so results are bit-identical
 * to the reference's CPU build.
 */
#ifndef SPDK_PROTO_H
#define SPDK_PROTO_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spdk_sd {
    double* data;  /* device */
    int ext[8];    /* t, var, k, j, i, kk, jj, ii */
} spdk_sd;

typedef struct spdk_fv {
    double* data;  /* device */
    int ext[4];    /* var, K, J, I */
} spdk_fv;

typedef struct spdk_mat {
    const double* data;  /* device */
    int rows, cols;
} spdk_mat;

typedef struct spdk_vec {
    const double* data;  /* device */
    int n;
} spdk_vec;

/* the fields of the reference's cfg these functions read */
typedef struct spdk_proto_cfg {
    int p;                /* polynomial degree (SED only for p > 1) */
    int active[3];        /* active directions */
    double gamma;
    double cfl;
    double g[3];          /* gravity; all zero = no source */
    double nad_tolerance;
    int nad_delta;        /* 1: tolerance relative to max-min */
    int nad_moore;        /* 1: 3^d box; 0: face neighbours */
    int sed;              /* smooth-extrema relaxation */
} spdk_proto_cfg;

enum { SPDK_PROTO_PERIODIC = 0, SPDK_PROTO_GRADFREE = 1, SPDK_PROTO_REFLECTIVE = 2 };

/* --- transforms (src/transforms.cpp) ------------------------------------ */
/* src/prototypes.hpp:15 transform_a_to_b(U_a, U_b, T, a_to_b): d sweeps */
int spdk_transform_a_to_b(const spdk_sd* a, const spdk_sd* b, const spdk_sd* tmp, const spdk_mat* m,
                          const spdk_proto_cfg* cfg, void* stream);
/* src/prototypes.hpp:16 transform_a_to_b_1d(A, B, M, dim) */
int spdk_transform_a_to_b_1d(const spdk_sd* a, const spdk_sd* b, const spdk_mat* m, int dim, void* stream);
/* src/prototypes.hpp:17 transform_a_to_b_1d_slice(A, B, M, dim, t): slice t of A -> slice 0 of B */
int spdk_transform_a_to_b_1d_slice(const spdk_sd* a, const spdk_sd* b, const spdk_mat* m, int dim, int t,
                                   void* stream);
/* src/prototypes.hpp:20 combine_solution(U, U0, a): U <- a U0 + (1-a) U */
int spdk_combine_solution(const spdk_sd* u, const spdk_sd* u0, double a, void* stream);
/* src/prototypes.hpp:22 update_prediction(U, U_ader, F_x, F_y, F_z, dfp_to_sp, invader, w, dt, dx, dy, dz) */
int spdk_update_prediction(const spdk_sd* u, const spdk_sd* u_ader, const spdk_sd* fx, const spdk_sd* fy,
                           const spdk_sd* fz, const spdk_mat* dfp_to_sp, const spdk_mat* invader,
                           const spdk_vec* w, double dt, double dx, double dy, double dz,
                           const spdk_proto_cfg* cfg, void* stream);
/* src/prototypes.hpp:23 update_solution(U, U_ader, F_x, F_y, F_z, dfp_to_sp, w, dt, dx, dy, dz) */
int spdk_update_solution(const spdk_sd* u, const spdk_sd* u_ader, const spdk_sd* fx, const spdk_sd* fy,
                         const spdk_sd* fz, const spdk_mat* dfp_to_sp, const spdk_vec* w, double dt, double dx,
                         double dy, double dz, const spdk_proto_cfg* cfg, void* stream);

/* --- hydro (src/hydro.cpp) ---------------------------------------------- */
/* src/prototypes.hpp:33-34 compute_conservatives(W, U) / compute_primitives(U, W), every slice */
int spdk_compute_conservatives(const spdk_sd* w, const spdk_sd* u, const spdk_proto_cfg* cfg, void* stream);
int spdk_compute_primitives(const spdk_sd* u, const spdk_sd* w, const spdk_proto_cfg* cfg, void* stream);
/* src/prototypes.hpp:41-42 (FV overloads) */
int spdk_fv_compute_conservatives(const spdk_fv* w, const spdk_fv* u, const spdk_proto_cfg* cfg, void* stream);
int spdk_fv_compute_primitives(const spdk_fv* u, const spdk_fv* w, const spdk_proto_cfg* cfg, void* stream);
/* src/prototypes.hpp:35 compute_fluxes(U, F, v1, v2, v3): v1 = normal velocity slot */
int spdk_compute_fluxes(const spdk_sd* u, const spdk_sd* f, int v1, int v2, int v3, const spdk_proto_cfg* cfg,
                        void* stream);
/* src/prototypes.hpp:36 compute_dt(W, dx, dy, dz, nu): min over active points -> *dt_out (device);
 * nu > 0 adds the diffusion limit 0.25 cfl (dx_min/(p+1))^2 / nu (src/hydro.cpp:245-254) */
int spdk_compute_dt(const spdk_sd* w, double dx, double dy, double dz, double nu, double* dt_out,
                    const spdk_proto_cfg* cfg, void* stream);
/* src/prototypes.hpp:54 sd_riemann_solver(U, F, v1, v2, v3, dim, viscous): LLF written to both
 * interface flux points of F; viscous != 0 also writes the central interface state
 * 0.5(uR+uL) + 0.5(uR-uL) over both interface points of U (src/hydro.cpp:370-413) */
int spdk_sd_riemann_solver(const spdk_sd* u, const spdk_sd* f, int v1, int v2, int v3, int dim, int viscous,
                           const spdk_proto_cfg* cfg, void* stream);

/* --- viscous terms (src/hydro.cpp:420-572), used when hydro/nu > 0 --------- */
/* src/prototypes.hpp:55 sd_rusanov_solver(U, F, dim): F at both interface points +=
 * 0.5(uR+uL) - 0.5(uR-uL) with uL = U at the right element's first flux point and
 * uR = U at the left element's last (U holds viscous fluxes) */
int spdk_sd_rusanov_solver(const spdk_sd* u, const spdk_sd* f, int dim, void* stream);
/* src/prototypes.hpp:37 compute_gradient(U, dU, h, dfp_to_sp, dim): dU (solution points)
 * = sum over the n+1 flux points along dim of U * dfp_to_sp / h, active elements only */
int spdk_compute_gradient(const spdk_sd* u, const spdk_sd* du, double h, const spdk_mat* dfp_to_sp, int dim,
                          const spdk_proto_cfg* cfg, void* stream);
/* src/prototypes.hpp:38 compute_viscous_flux(U, dU1, v1, dU2, v2, dU3, v3, sp_to_fp, nu, beta, dim):
 * at every flux point of direction dim (ghost elements included) the momentum
 * gradients du1/du2/du3 interpolated along dim and the viscous flux
 * (0, 2 nu du1 + beta div-part, nu (du1 + du2) ..., energy w.f) written over U;
 * v1 = 1+dim, (v2, v3) the cyclic momentum slots */
int spdk_compute_viscous_flux(const spdk_sd* u, const spdk_sd* du1, int v1, const spdk_sd* du2, int v2,
                              const spdk_sd* du3, int v3, const spdk_mat* sp_to_fp, double nu, double beta, int dim,
                              const spdk_proto_cfg* cfg, void* stream);

/* --- boundaries (src/boundary.cpp) -------------------------------------- */
/* src/prototypes.hpp:61 boundaries(comm, Boundaries{dim, type}, U): interface
 * flux point of the ghost elements of direction dim */
int spdk_boundaries_sd(const spdk_sd* u, int dim, int type, void* stream);
/* src/prototypes.hpp:62 boundaries(comm, FV_Boundaries{dim, type}, U, alignment, a_dim);
 * cell-centred arrays only (alignment 0; the staggered form serves the
 * induction solver) */
int spdk_boundaries_fv(const spdk_fv* u, int dim, int type, int alignment, int a_dim, void* stream);

/* --- finite-volume sub-grid (src/transforms.cpp) ------------------------- */
/* src/prototypes.hpp:66 face_integral(F_ader_fp, F, T, sp_to_cv, dim, t) */
int spdk_face_integral(const spdk_sd* f_fp, const spdk_fv* f, const spdk_sd* tmp, const spdk_mat* sp_to_cv,
                       int dim, int t, const spdk_proto_cfg* cfg, void* stream);
/* src/prototypes.hpp:68-71 fv_update_solution(U_old, U_new, U_cv, F_x, x_f, F_y, y_f, F_z, z_f, w, t, dt, update) */
int spdk_fv_update_solution(const spdk_fv* u_old, const spdk_fv* u_new, const spdk_sd* u_cv, const spdk_fv* fx,
                            const spdk_vec* x_f, const spdk_fv* fy, const spdk_vec* y_f, const spdk_fv* fz,
                            const spdk_vec* z_f, const spdk_vec* w, int t, double dt, int update,
                            const spdk_proto_cfg* cfg, void* stream);

/* --- trouble detection (src/trouble_detection.cpp) ----------------------- */
/* src/prototypes.hpp:74-77 detect_troubles(W_new, W_old, troubles, alpha_x, alpha_y, alpha_z,
 * X_dim, Y_dim, Z_dim, PAD, limit_mask); the dimension structs are replaced
 * by their FV centres and faces */
int spdk_detect_troubles(const spdk_fv* w_new, const spdk_fv* w_old, const spdk_fv* troubles,
                         const spdk_fv* alpha_x, const spdk_fv* alpha_y, const spdk_fv* alpha_z,
                         const spdk_vec* x_c, const spdk_vec* x_f, const spdk_vec* y_c, const spdk_vec* y_f,
                         const spdk_vec* z_c, const spdk_vec* z_f, int pad, int limit_mask,
                         const spdk_proto_cfg* cfg, void* stream);
/* src/prototypes.hpp:78-80 */
int spdk_apply_blending(const spdk_fv* troubles, const spdk_fv* theta, const spdk_proto_cfg* cfg, void* stream);
int spdk_blending_ring(const spdk_fv* theta_in, const spdk_fv* theta_out, const spdk_proto_cfg* cfg,
                       void* stream);
int spdk_theta_from_troubles(const spdk_fv* troubles, const spdk_fv* theta, void* stream);
/* src/prototypes.hpp:82-87 fallback_fluxes(W, theta, x_c, x_f, F_x, y_c, y_f, F_y, z_c, z_f, F_z, ader, w, dt) */
int spdk_fallback_fluxes(const spdk_fv* w_old, const spdk_fv* theta, const spdk_vec* x_c, const spdk_vec* x_f,
                         const spdk_fv* fx, const spdk_vec* y_c, const spdk_vec* y_f, const spdk_fv* fy,
                         const spdk_vec* z_c, const spdk_vec* z_f, const spdk_fv* fz, int ader,
                         const spdk_vec* w, double dt, const spdk_proto_cfg* cfg, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SPDK_PROTO_H */
