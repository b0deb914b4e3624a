/* swl_b200 multi-GPU serving: one request loop (include/swl_server.h) per device, and a front
 * that places every shot request on one of them by device-memory budget.
 *
 * Shots are independent, so a request stream shards over GPUs with no data-path exchange: each
 * request runs whole on the device it was placed on, and its records come back from that device's
 * server.  Placement charges every request its estimated resident bytes (the server's admission
 * estimate) against the device it goes to until it finishes, and sends it to the device with the
 * most budget left (worst fit: spreads the load and leaves the largest holes for large shots).
 * Ties go to the lower slot.  A request larger than every device's whole budget is refused.
 *
 * No counterpart in the reference: it selects one device per session
 * (src/common/ComputeDevices.cpp:16-40, the usable device with the most memory), which is what a
 * fleet of one device does.
 */
#ifndef SWL_FLEET_H
#define SWL_FLEET_H
#include "swl_server.h"
#ifdef __cplusplus
extern "C" {
#endif

#define SWL_FLEET_MAX_DEVICES 16

typedef struct swl_fleet swl_fleet;

typedef struct swl_fleet_config {
    int32_t n_devices;                        /* 0: every usable device */
    int32_t devices[SWL_FLEET_MAX_DEVICES];   /* device indices when n_devices > 0 */
    swl_server_config server;                 /* settings of every device's server (its device field is ignored) */
} swl_fleet_config;

/* Estimated device bytes of a request (what a server charges against its budget at admission). */
swl_status swl_request_bytes2d(const swl_params2d *p, int64_t *bytes);
swl_status swl_request_bytes3d(const swl_params3d *p, int64_t *bytes);
/* The placement rule alone, without devices: the slot (0..n-1) of the device a request of
 * `charge` bytes goes to, given each device's budget and the bytes already charged to it; -1 when
 * no device's whole budget can hold it. */
int32_t swl_fleet_choose(int32_t n, const int64_t *budgets, const int64_t *charged, int64_t charge);

void swl_fleet_config_default(swl_fleet_config *c);
swl_status swl_fleet_create(const swl_fleet_config *c, swl_fleet **out);
void swl_fleet_destroy(swl_fleet *f);
int32_t swl_fleet_size(const swl_fleet *f);               /* devices (slots) */
int32_t swl_fleet_device(const swl_fleet *f, int32_t slot); /* CUDA device index of a slot, or -1 */
/* Submit a request; *id is the fleet's id of the shot and *slot the device slot it was placed on. */
swl_status swl_fleet_submit2d(swl_fleet *f, const swl_params2d *p, int64_t *id, int32_t *slot);
swl_status swl_fleet_submit3d(swl_fleet *f, const swl_params3d *p, int64_t *id, int32_t *slot);
/* As the swl_server_* calls of the shot's device (the status's id is the fleet id). */
swl_status swl_fleet_status(swl_fleet *f, int64_t id, swl_shot_status *out, int32_t *slot);
swl_status swl_fleet_records(swl_fleet *f, int64_t id, double *vx, double *vy, double *vz);
swl_status swl_fleet_release(swl_fleet *f, int64_t id);
swl_status swl_fleet_drain(swl_fleet *f);
/* The server statistics of one slot, and the bytes the front has charged to it. */
swl_status swl_fleet_stats(swl_fleet *f, int32_t slot, swl_server_stats *out, int64_t *charged);

#ifdef __cplusplus
}
#endif
#endif
