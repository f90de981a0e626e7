/*
 * licom_serve.h - a request server for tracer integrations on one device.
 *
 * No counterpart in the reference.  Requests (a domain described by the
 * seeded generators of licom_synth.h, a number of tracer steps and an arrival
 * time) are admitted while their arena fits the HBM budget, stay resident on
 * the device until done, and are advanced together: every scheduling
 * iteration steps all resident requests through one batch (licom_batch.h) by
 * the same number of steps - the smallest remaining count, at most
 * chunk_steps - so that requests leave exactly when they finish and freed
 * memory admits the next ones at the following iteration (continuous
 * batching).  While the device runs an iteration, the host builds the inputs
 * of newly arrived requests.  A request's result does not depend on what it
 * was batched with: the batched kernels compute each member exactly as a
 * domain stepped alone.
 */
#ifndef LICOM_SERVE_H
#define LICOM_SERVE_H

#include "licom_tracer.h"
#include "licom_synth.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lt_server lt_server;

typedef struct {
  size_t hbm_budget;     /* bytes the resident requests may hold; 0 = free memory at creation minus 8 GiB */
  int max_active;        /* resident requests at most; 0 = 512 */
  int chunk_steps;       /* largest step count of one iteration; 0 = 10 */
  int precision;         /* lt_precision of every request */
} lt_server_config;

typedef struct {
  lt_synth_config domain;  /* the request's domain (grid, fields, seed) */
  int steps;               /* tracer steps asked for (>= 1) */
  double arrival;          /* seconds on the server clock; the request is invisible before */
  int keep_state;          /* 1: keep the final AT on the host for lt_server_state */
} lt_request;

typedef enum { LT_REQ_PENDING = 0, LT_REQ_QUEUED = 1, LT_REQ_RESIDENT = 2, LT_REQ_DONE = 3, LT_REQ_REFUSED = -1 } lt_req_state;

typedef struct {
  int state;               /* lt_req_state */
  int steps_done;
  double arrival, admitted, finished;   /* server clock, seconds */
  double content[2];       /* global T and S content after the last step */
  long long cells;         /* nx*ny*km */
  size_t bytes;            /* device bytes of its arena */
} lt_request_status;

typedef struct {
  long long requests_done, requests_refused;
  long long iterations;
  double cell_steps;        /* cell-steps advanced */
  double busy_s;            /* device time of the iterations (CUDA events) */
  double wall_s;            /* server clock at the last iteration */
  double latency_p50, latency_p99, latency_max;   /* seconds, finished - arrival, over finished requests */
  int max_resident;
  size_t peak_bytes;
} lt_server_stats;

int lt_server_create(const lt_server_config* cfg, lt_server** out);
int lt_server_destroy(lt_server* s);
/* Seconds since the server was created. */
double lt_server_clock(lt_server* s);
int lt_server_submit(lt_server* s, const lt_request* r, int* id);
/* One scheduling iteration: queue what has arrived, admit what fits, step the
 * resident requests, retire the finished.  *busy = 1 if anything is still
 * pending, queued or resident. */
int lt_server_run_once(lt_server* s, int* busy);
/* Iterate until every submitted request is done or refused (waiting for
 * arrivals in between). */
int lt_server_drain(lt_server* s);
int lt_server_status(lt_server* s, int id, lt_request_status* st);
/* Final AT [2][km][ny+4][nx+4] of a finished request submitted with keep_state. */
int lt_server_state(lt_server* s, int id, double* host_at, size_t nbytes);
int lt_server_stats_get(lt_server* s, lt_server_stats* st);

#ifdef __cplusplus
}
#endif

#endif
