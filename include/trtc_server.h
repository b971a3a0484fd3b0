/* trtc_server.h -- request server of libPyThrustRTC.so (thrustrtc_b200 addition, no
 * counterpart in the reference, whose calls are blocking and one at a time on stream 0).
 *
 * Requests work on the caller's device buffers and are served with continuous batching:
 * a request group starts when one of the server's streams is free and the temporary device
 * memory it needs fits in the budget next to the running groups; waiting requests of at most
 * coalesce_max_n elements with the same kind and element type are served together by one
 * segmented launch; larger ones run alone on the plain kernels.  Results equal those of the
 * single-request calls (bit-exact for sorts and integer scans/sums; float sums and scans
 * within rounding of a different summation order).
 *
 * Kinds: 0 Sort_By_Key (keys of `type` and uint32 values, sorted in place, ascending,
 * stable), 1 exclusive Plus scan (keys -> out), 2 Plus reduce (keys; result via
 * trtc_server_result).  Types: 4 int32, 5 uint32, 8 float, 6 int64, 7 uint64.
 * Buffers must stay valid until the request is done.  The server is thread-safe; calls
 * return -1 / NULL on failure (trtc_last_error() describes it). */
#ifndef TRTC_SERVER_H
#define TRTC_SERVER_H

#ifdef __cplusplus
extern "C" {
#endif

void* trtc_server_create(unsigned long long budget_bytes, int num_streams, unsigned long long coalesce_max_n);
/* returns the request id (> 0) */
long long trtc_server_submit(void* srv, int kind, int type, void* keys, void* values, void* out,
                             unsigned long long n);
/* retires finished groups and launches waiting requests; returns the number of requests
 * still queued or running */
int trtc_server_poll(void* srv);
/* state: 0 queued, 1 running, 2 done, -1 error; times in seconds since the server started
 * (submission, and completion as seen by the poll that retired it) */
int trtc_server_info(void* srv, long long id, double* t_submit, double* t_done, double* result);
/* a finished reduce's sum: the element's bytes in the low bytes of *out8 */
int trtc_server_result(void* srv, long long id, void* out8);
double trtc_server_now(void* srv);
/* drops the records of finished requests */
void trtc_server_forget_done(void* srv);
void trtc_server_destroy(void* srv);

#ifdef __cplusplus
}
#endif

#endif /* TRTC_SERVER_H */
