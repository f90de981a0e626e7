/*
 * licom_batch.h - many tracer domains stepped together on one device.
 *
 * No counterpart in the reference, which advances one domain per MPI rank.
 * A batch holds existing domains (lt_create) of any sizes - ensemble members
 * of one grid, or regional domains of a serving pool - on the current device,
 * all of one precision.  One batch step advances every member by one tracer
 * step: the per-member surface, SSS-norm and halo kernels, and, in mixed
 * precision, ONE continuity launch and ONE persistent column launch over the
 * concatenated (member, tile) work list.  The steps are captured in a
 * CUDA graph (one per ping-pong parity) and replayed.
 *
 * Each member's state stays in its own arena; after a batch step the domain
 * API (lt_get_field, lt_tracer_content, lt_step, ...) sees the advanced state.
 * Do not step a member through its own stream while its batch is in flight.
 */
#ifndef LICOM_BATCH_H
#define LICOM_BATCH_H

#include "licom_tracer.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lt_batch lt_batch;

/* Launch shape of a batch step (what the autotuner chooses). */
typedef struct {
  int column_ctas_per_sm;   /* persistent CTAs of the column kernel per SM: 1..3 (mixed) */
  int continuity_tile_y;    /* rows of a continuity tile (32 x 4, 8 or 16 columns) */
  int use_graph;            /* 1: replay captured CUDA graphs, 0: launch directly */
} lt_batch_config;

/* members: n domains on the current device, all LT_PREC_MIXED or all
 * LT_PREC_FP64 (FP64 members run their own kernels inside the graph). */
int lt_batch_create(lt_domain* const* members, int n, lt_batch** out);
int lt_batch_destroy(lt_batch* b);
int lt_batch_size(lt_batch* b, int* n);
int lt_batch_get_config(lt_batch* b, lt_batch_config* cfg);
int lt_batch_set_config(lt_batch* b, const lt_batch_config* cfg);
/* Enqueue nsteps steps of every member on the batch's stream. */
int lt_batch_step(lt_batch* b, int nsteps);
/* Wait for the batch; LT_E_TIMEOUT if any member's column wait ran out. */
int lt_batch_sync(lt_batch* b);
/* Device time (ms) of the last lt_batch_step call, CUDA events. */
int lt_batch_last_ms(lt_batch* b, float* ms);
/* Autotuner: times every candidate launch shape for `trial_steps` steps (after
 * one untimed step), keeps the fastest and writes it to *chosen (may be NULL).
 * The members' states are restored afterwards, so tuning does not advance
 * them.  The choice is remembered for batches of the same member shapes. */
int lt_batch_autotune(lt_batch* b, int trial_steps, lt_batch_config* chosen);

#ifdef __cplusplus
}
#endif

#endif
