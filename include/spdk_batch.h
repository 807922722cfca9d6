/* Batched form (libspdk_cuda.so): many independent 2D hydro problems of
 * uneven sizes and orders advanced together. No counterpart in the
 * reference, which runs one problem per process.
 *
 * Problems are grouped by order p; every pass of an ADER step is one launch
 * per group that covers the tiles of all the group's problems (each block
 * looks up its problem in a table and runs the single-problem kernel body
 * on it), the groups run concurrently on their own streams, and the whole
 * step is captured once as a CUDA graph and replayed. Each problem keeps its
 * own dt (the step count is shared). The tile shape (elements per block) of
 * each group is chosen by spdk_batch_autotune, which times the candidates on
 * the batch itself.
 *
 * Supported: 2D, ADER, p in {2, 3, 5}, every element count a multiple of the
 * largest candidate tile that divides all of the group (tiles 1x1, 2x2 and,
 * for p <= 3, 4x4), all problems in one precision, fallback on or off for
 * all, no learned indicator. Results are bit-identical to stepping each
 * problem alone with spdk_hydro_step (labels included).
 */
#ifndef SPDK_BATCH_H
#define SPDK_BATCH_H

#include "spdk.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spdk_batch spdk_batch;

typedef struct spdk_batch_info {
    int n_problems;
    int n_groups;
    long long n_dof;           /* active solution points of all problems */
    int launches_per_step;     /* kernels one replayed step launches */
    int group_p[8];            /* order of each group */
    int group_tile[8];         /* tile edge (elements) of each group */
    int group_size[8];         /* problems in each group */
    size_t device_bytes;
} spdk_batch_info;

/* builds one spdk_hydro per configuration (same device, precision and
 * fallback setting for all) and the batched tables; tiles start at 2x2 */
int spdk_batch_create(const spdk_hydro_config* cfgs, int count, spdk_batch** out);
int spdk_batch_destroy(spdk_batch* b);
/* times every candidate tile of every group over `steps` steps and keeps the
 * fastest; the problems' state is restored afterwards (blocking) */
int spdk_batch_autotune(spdk_batch* b, int steps);
/* nsteps replays of the captured step on the batch's stream (asynchronous) */
int spdk_batch_steps(spdk_batch* b, int nsteps);
int spdk_batch_sync(spdk_batch* b);
int spdk_batch_get_info(spdk_batch* b, spdk_batch_info* info);
int spdk_batch_get_stream(spdk_batch* b, void** stream);
/* on = 1: every replayed step also writes each problem's per-element trouble
 * labels (1 where NAD/SED/PAD flagged any sub-cell of the element in any
 * slice of the step), read per member with spdk_hydro_read(
 * SPDK_FIELD_ELEMENT_TROUBLES) after spdk_batch_sync: the indicator's
 * training data from the batched run. Needs fallback = 1; blocking. */
int spdk_batch_record_labels(spdk_batch* b, int on);
/* the solver of problem i, for spdk_hydro_read / _get_dt after spdk_batch_sync
 * (owned by the batch: do not destroy or step it) */
int spdk_batch_member(spdk_batch* b, int i, spdk_hydro** h);

#ifdef __cplusplus
}
#endif
#endif /* SPDK_BATCH_H */
