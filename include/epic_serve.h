/*
 * epic_serve.h -- served ensembles of independent EPIC simulations on one GPU.
 *
 * No counterpart in the reference (it runs one simulation per MPI job).  A
 * server keeps up to max_slots simulations on the device at once, each with
 * its own context and CUDA stream, so their kernels overlap on the GPU.
 * A slot that frees up takes the first queued request (in arrival order)
 * whose device memory fits in the server's share of the free HBM, so a large
 * request at the head does not hold back smaller ones behind it; a request
 * that arrives while others run starts without waiting for them (continuous
 * admission).  Contexts of finished requests are kept and
 * reused by later requests with the same configuration, so steady-state
 * serving allocates no device memory.  Initial states are generated on the
 * device (epic_gpu_init_state).
 */
#ifndef EPIC_SERVE_H
#define EPIC_SERVE_H

#include "epic_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct epic_request {
    epic_cfg       cfg;       /* grid, options, precision form            */
    epic_init_spec init;      /* initial state, generated on the device    */
    int32_t        steps;     /* full steps (epic_gpu_step) to run         */
    int32_t        tune;      /* 1: a new context runs epic_gpu_autotune first
                                 (timing-based launch shapes: fastest, but
                                 results then depend on the choice to the
                                 last bits); 0: fixed shapes, reproducible  */
} epic_request;

typedef struct epic_result {
    int64_t id;
    int32_t status;           /* EPIC_OK or the failing call's EPIC_ERR_*  */
    int32_t slot;             /* worker slot that ran it (-1: rejected)    */
    double  t_submit;         /* seconds since epic_srv_create             */
    double  t_start;          /* admitted (context acquired)               */
    double  t_done;
    int64_t parcel_steps;     /* sum over steps of parcels at step start   */
    int64_t n_parcels;        /* parcels after the last step               */
    double  t_final;          /* simulated time after the last step        */
    double  ke, enstrophy;    /* parcel_stats[1], [12] of the last step    */
    double  device_bytes;     /* admission estimate of the request         */
    char    message[160];     /* error message of a failed request         */
} epic_result;

typedef struct epic_server epic_server;

/* max_slots simulations at a time on the current device; the server admits
 * requests while their estimated memory stays below hbm_fraction of the
 * device memory that was free at creation. */
int epic_srv_create(int32_t max_slots, double hbm_fraction, epic_server** out);
/* Queue a request; *id identifies it.  A request larger than the server's
 * whole budget completes at once with status EPIC_ERR_CAPACITY. */
int epic_srv_submit(epic_server* srv, const epic_request* req, int64_t* id);
/* Block until request id has finished; fills *out (status included).  The
 * result is handed over: a second wait on the same id returns EPIC_ERR_ARG. */
int epic_srv_wait(epic_server* srv, int64_t id, epic_result* out);
int epic_srv_counts(epic_server* srv, int64_t* queued, int64_t* running, int64_t* done);

/* Admission order: the order in which a slot that frees up looks through the
 * queued requests for one that fits.  EPIC_SRV_ARRIVAL (the default) takes
 * them in arrival order; EPIC_SRV_SHORTEST_FIRST takes the smallest
 * estimated work first (cells x parcels per cell x steps, ties in arrival
 * order), which lowers the median time to completion when the offered load
 * exceeds the device, at the cost of the largest requests' wait.  Applies
 * to every later admission. */
#define EPIC_SRV_ARRIVAL 0
#define EPIC_SRV_SHORTEST_FIRST 1
int epic_srv_set_policy(epic_server* srv, int32_t policy);
/* Finish all queued work, then free every context. */
void epic_srv_destroy(epic_server* srv);

#ifdef __cplusplus
}
#endif

#endif
