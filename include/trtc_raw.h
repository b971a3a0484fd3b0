/* trtc_raw.h -- raw-pointer entry points of libPyThrustRTC.so (thrustrtc_b200 additions).
 *
 * These have no counterpart in the reference's python/api.h: they run the same nvcc-built
 * kernels on caller-owned device buffers of the built-in element types, on a caller-chosen
 * CUDA stream (void* = cudaStream_t, NULL = legacy default stream), without the object
 * model.  They back the benchmark, the batched and serving paths, and direct C users.
 * Element type codes: 0 int8, 1 uint8, 2 int16, 3 uint16, 4 int32, 5 uint32, 6 int64,
 * 7 uint64, 8 float, 9 double.  Operator codes: 0 Plus, 1 Maximum, 2 Minimum.
 * int results: 0 success, -1 failure (trtc_last_error() describes it).  Calls that return
 * a count or value synchronise the stream; the others are asynchronous, and trtc_raw_sync()
 * synchronises and reports any device-side error (e.g. an exceeded bounded wait).
 */
#ifndef TRTC_RAW_H
#define TRTC_RAW_H

#ifdef __cplusplus
extern "C" {
#endif

const char* trtc_last_error(void);
/* number of thrustrtc_b200 kernels launched by this process */
unsigned long long trtc_launch_count(void);
/* optional per-launch timing: while enabled (on != 0; enabling or disabling discards old
 * records) each launch of this library records a CUDA event on its stream.  count()
 * synchronises those events and returns the number of timed launches (-1 on failure);
 * get() returns the kernel name and its device time in milliseconds. */
void trtc_timing_enable(int on);
int trtc_timing_count(void);
int trtc_timing_get(int i, char* name, unsigned long long name_cap, float* ms);
/* caps the size of any one device allocation the library makes for a call (temporaries and
 * DVVector storage; 0 removes the cap).  An allocation above the cap fails the way an
 * out-of-memory one does (the call returns its failure value, before any kernel runs, and
 * leaves its inputs untouched); for capacity planning and for tests of those failure paths. */
void trtc_set_alloc_limit(unsigned long long bytes);
/* counters of the NVRTC kernel cache since the process started: out[0] NVRTC compilations,
 * out[1] kernels taken from the persistent cubin cache (TRTC_CACHE_DIR, else
 * ~/.cache/thrustrtc_b200; TRTC_JIT_DISK_CACHE=0 turns it off), out[2] kernels found already
 * loaded in this process.  No reference counterpart (its cache has no counters). */
void trtc_jit_cache_stats(unsigned long long* out);
/* synchronises `stream`; 0, or -1 when a kernel reported an error */
int trtc_raw_sync(void* stream);

/* stable radix sort in place; same order as TRTC_Sort with Less (descending=0) or Greater */
int trtc_raw_sort(int key_type, void* keys, unsigned long long n, int descending, void* stream);
/* pairs: values of `value_size` bytes move with their keys */
int trtc_raw_sort_by_key(int key_type, void* keys, void* values, unsigned long long value_size,
                         unsigned long long n, int descending, void* stream);
/* index selected by TRTC_Min_Element's reduction tree (~0ull on failure); synchronous */
unsigned long long trtc_raw_min_element(int type, const void* in, unsigned long long n, void* stream);

/* inclusive (exclusive=0) or exclusive scan with host-side init (NULL: zero) */
int trtc_raw_scan(int type, int op, int exclusive, const void* in, void* out, unsigned long long n,
                  const void* init, void* stream);
/* trtc_raw_scan without any allocation.  No counterpart in the reference, which allocates
 * scan workspace on every call.  For callers that cannot allocate device memory while they
 * run: code inside a memory-pool or allocator callback (an allocation would re-enter the
 * allocator), a framework that has reserved the device's memory for its own allocator (a
 * cudaMalloc would fail), or a real-time loop that cannot take cudaMalloc's device-wide
 * synchronisation.  It runs the two-phase kernel trtc_raw_scan runs for these types; integer
 * results are identical to trtc_raw_scan's, float results agree within rounding (a float
 * look-back may group tile totals differently from one run to the next).  Accepts int32 (4),
 * uint32 (5) and float (8), op 0 Plus / 1 Maximum / 2 Minimum, 1 <= n <= 2^28 elements; other
 * sizes, types or operators return -1 with a message in trtc_last_error() and launch
 * nothing.  The look-back scratch is a 256 KiB array in the library's static device memory,
 * held by every GPU context that loads the library until the process exits; the call makes
 * no cudaMalloc, cudaFree, pinned host allocation or memory-pool allocation.  The first call
 * in a CUDA context does a one-time set-up (it looks up the scratch array's device address
 * with that context current); make that first call before any stream capture.  Every call
 * shares the one scratch array of its context, which keeps the last call's contents, so
 * calls that overlap on the device (other streams, other host threads) race: issue them in
 * one stream or synchronise in between.  status_dev: NULL, or a caller-owned device word that
 * must be zero before the call; a device-side failure (an expired bounded wait) ORs a
 * nonzero code into it.  Asynchronous with respect to the host. */
int trtc_raw_scan_noalloc(int type, int op, int exclusive, const void* in, void* out, unsigned long long n,
                          const void* init, unsigned int* status_dev, void* stream);
/* reduction to host memory (init may be NULL); synchronous */
int trtc_raw_reduce(int type, int op, const void* in, unsigned long long n, const void* init, void* result_host,
                    void* stream);
/* reduction left in device memory at *result_dev (library-owned, valid until the next call) */
int trtc_raw_reduce_async(int type, int op, const void* in, unsigned long long n, const void* init,
                          void** result_dev, void* stream);
/* segmented scan, EqualTo keys / Plus values */
int trtc_raw_scan_by_key(int key_type, int value_type, int exclusive, const void* keys, const void* values,
                         void* out, unsigned long long n, const void* init, void* stream);
/* stable compactions; return the number of elements written (~0ull on failure) */
unsigned long long trtc_raw_remove_copy(int type, const void* in, void* out, unsigned long long n,
                                        const void* value, void* stream);
unsigned long long trtc_raw_unique_copy(int type, const void* in, void* out, unsigned long long n, void* stream);

/* Batched segmented sort + scan (no reference counterpart; the reference needs one sort call
 * and one scan call per segment).  Segment i is keys/values[offsets[i], offsets[i+1]) with
 * `offsets` a device array of nseg + 1 ascending element indices.  Each segment is stably
 * sorted by key (ascending or descending, same order as trtc_raw_sort_by_key on it alone),
 * its 4-byte values move with the keys, and scan_out receives the exclusive Plus scan
 * (uint32 wrap-around) of each segment's sorted values.  Key types 4 (int32), 5 (uint32),
 * 8 (float), 6 (int64), 7 (uint64); n and nseg below 2^32.  One persistent launch over all
 * segments; the caller passes a device workspace of at least
 * trtc_raw_segmented_workspace_bytes(key_type, n, nseg) bytes, and the call allocates nothing
 * else (it can be captured in a CUDA graph after a first, uncaptured call of the same key
 * type has set the kernels up). */
unsigned long long trtc_raw_segmented_workspace_bytes(int key_type, unsigned long long n, unsigned long long nseg);
int trtc_raw_segmented_sort_scan(int key_type, void* keys, void* values, void* scan_out,
                                 const unsigned long long* offsets, unsigned long long nseg, unsigned long long n,
                                 void* workspace, unsigned long long workspace_bytes, int descending, void* stream);
/* Size classes of the batched kernel: segments of at most `warp_small` (0 or 32) keys are
 * sorted by one warp with a bitonic network (no digit counters), at most 32 x items keys by
 * one warp with 8-bit radix passes, at most 64 / 128 x items keys by a group of two / four
 * warps, at most 256 x items keys by a whole CTA on chip, longer ones by a whole CTA through
 * global memory; items is 8 or 16.  Per key type, the shape
 * (items, warp_small) comes from a tuning table: compiled-in defaults (16, 32), a table loaded
 * from the file named by TRTC_SEG_TUNING_FILE at the first batched call, a table passed to
 * trtc_raw_segmented_tuning_load, or the autotuner.
 * The autotuner times the four shapes on random keys with these segment offsets and keeps the
 * fastest for this key type; returns its items per thread, or -1.  Allocates its own
 * scratch; synchronous. */
int trtc_raw_segmented_autotune(int key_type, const unsigned long long* offsets, unsigned long long nseg,
                                unsigned long long n, void* stream);
/* the tuning table as versioned JSON (written into out, at most cap bytes with the final NUL);
 * returns the full length */
unsigned long long trtc_raw_segmented_tuning_json(char* out, unsigned long long cap);
/* replaces the entries named in a table of that JSON form; 0, or -1 for another format or
 * version or an unsupported shape */
int trtc_raw_segmented_tuning_load(const char* json);

/* Test hook for the bounded device waits: one inclusive Plus scan of int32 (n >= 4 * 8192)
 * with a kernel built so that tile 2 never publishes its look-back word and every wait gives
 * up after 4096 polls.  The waits behind tile 2 run out, the kernel records the error and
 * finishes; the call returns -1 with "look-back wait exceeded its bound" in
 * trtc_last_error(), and the library stays usable (out holds garbage).  Synchronous. */
int trtc_test_scan_lookback_timeout(const int* in, int* out, unsigned long long n, void* stream);

/* diagnostics: copies the sort control block of the last sort on `stream` */
unsigned long long trtc_debug_sort_ctrl(void* host, unsigned long long bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TRTC_RAW_H */
