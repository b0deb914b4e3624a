/* swl_b200 serving: a request loop that runs many shots on one GPU at once.
 *
 * Shot requests (2D or 3D session parameters, include/swl_session.h) are queued as they arrive.
 * The loop admits them in arrival order while their device memory fits the budget and the
 * active-shot limit allows.  A pool of host threads builds each admitted shot's FP64 model and
 * creates its engine on its own CUDA stream.  The loop then advances every running shot in
 * batches of CUDA-graph steps (swl2d_launch / swl3d_launch), so the batches of different shots
 * overlap on the device.  Receiver records are collected after every batch, and a shot's device
 * memory is released as soon as it completes, which lets the next queued shot in.
 *
 * No counterpart in the reference: its only concurrency is one UI worker thread per session
 * (include/SeisCommon/BackgroundRunner.hpp:13-52).  Admission follows its transactional memory
 * budget (src/two_d/MemoryBudget2D.hpp:12-38), applied per request against the server's budget.
 */
#ifndef SWL_SERVER_H
#define SWL_SERVER_H
#include "swl_session.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct swl_server swl_server;

typedef struct swl_server_config {
    int32_t device;        /* -1: the usable device with the most memory */
    int64_t memory_budget; /* device bytes the server may hold; 0: 85 % of the free memory at creation */
    int32_t max_active;    /* shots building or running at once; 0: only the budget limits */
    int32_t batch_steps;   /* RK4 steps per engine batch (default 64) */
    int32_t build_threads; /* host threads building models (default 4) */
    int32_t scheduler_threads; /* host threads driving the running shots' batches (default 4); each
                                * owns the shots it started: polls, records and relaunches them */
    int32_t persistent;        /* 1: the 2D shots of one precision and GSLS mechanism count advance
                                * together, one batch each, in ONE persistent launch per round
                                * (swl2d_queue_launch), driven by one host thread; 2: the same for the
                                * elastic 2D shots only; 0: each shot runs its own batches on its own
                                * stream.  3D shots always run on their own streams. */
    int32_t persistent_ctas;   /* resident CTAs per SM of a persistent launch (swl2d_queue_limit);
                                * default -1: all but one, leaving room for the 3D shots' kernels and
                                * the engine builds beside it */
} swl_server_config;

enum { SWL_SHOT_QUEUED = 0, SWL_SHOT_BUILDING = 1, SWL_SHOT_RUNNING = 2, SWL_SHOT_DONE = 3, SWL_SHOT_FAILED = 4 };

typedef struct swl_shot_status {
    int64_t id;
    int32_t dim, state, steps_done, total_steps, receivers, pad;
    int64_t samples, resident_bytes;
    double submit_s, start_s, finish_s; /* seconds since the server was created */
    double run_s;                       /* model built, first batch about to launch (0 before) */
    char error[256];
} swl_shot_status;

typedef struct swl_server_stats {
    int32_t queued, building, running, done, failed, peak_running;
    int64_t resident_bytes, peak_resident_bytes, memory_budget;
} swl_server_stats;

void swl_server_config_default(swl_server_config *c);
swl_status swl_server_create(const swl_server_config *c, swl_server **out);
/* Destroys the server; running shots are abandoned and their memory released. */
void swl_server_destroy(swl_server *s);
swl_status swl_server_submit2d(swl_server *s, const swl_params2d *p, int64_t *id);
swl_status swl_server_submit3d(swl_server *s, const swl_params3d *p, int64_t *id);
swl_status swl_server_status(swl_server *s, int64_t id, swl_shot_status *out);
/* Wait up to timeout_ms for a shot to finish (done or failed) that has not been reported yet;
 * *id = -1 on timeout. */
swl_status swl_server_next_finished(swl_server *s, int32_t timeout_ms, int64_t *id);
/* Records of a finished shot: 2D writes vx, vz (receivers x samples); 3D writes vx, vy, vz
 * (receivers x (steps + 1)).  Unused pointers may be null. */
swl_status swl_server_records(swl_server *s, int64_t id, double *vx, double *vy, double *vz);
/* Forget a finished shot (its records). */
swl_status swl_server_release(swl_server *s, int64_t id);
/* Block until every submitted shot has finished. */
swl_status swl_server_drain(swl_server *s);
swl_status swl_server_stats_get(swl_server *s, swl_server_stats *out);

#ifdef __cplusplus
}
#endif
#endif
