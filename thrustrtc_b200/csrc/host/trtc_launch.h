// trtc_launch.h -- entry points of the nvcc-built (built-in type / operator) kernels.
#pragma once
#include <string>
#include <cstddef>
#include <cuda_runtime.h>

namespace trtc_host {

// compaction selector codes (same values as trtc::CompactMode)
enum : int { COMPACT_NOT_EQUAL = 2, COMPACT_UNIQUE = 5 };

// radix sort of built-in key types; vals may be null; vsize = payload bytes per element
bool sort_raw(int key_tc, void* keys, void* vals, size_t vsize, size_t n, bool desc, cudaStream_t s);
bool sort_raw_narrow(int key_tc, void* keys, void* vals, size_t vsize, size_t n, bool desc, cudaStream_t s);
bool sort_raw_32(int key_tc, void* keys, void* vals, size_t vsize, size_t n, bool desc, cudaStream_t s);
bool sort_raw_64(int key_tc, void* keys, void* vals, size_t vsize, size_t n, bool desc, cudaStream_t s);
// index of the minimum in the reference's Min_Element tree order (synchronous)
bool min_element_raw(int tc, const void* keys, size_t n, cudaStream_t s, unsigned long long* idx);

// mode 0 inclusive, 1 exclusive with *init; in/out same type
bool scan_raw(int tc, int op, int mode, const void* in, void* out, size_t n, const void* init, cudaStream_t s);
// init may be null; result written to host memory (synchronous)
bool reduce_raw(int tc, int op, const void* in, size_t n, const void* init, void* result_host, cudaStream_t s);
// kernel-only variant: result left in device memory at *result_dev (asynchronous)
bool reduce_raw_async(int tc, int op, const void* in, size_t n, const void* init, void** result_dev, cudaStream_t s);
// segmented scan, EqualTo keys / Plus values; mode 0 inclusive, 1 exclusive with *init (or 0)
bool scan_by_key_raw(int key_tc, int val_tc, int mode, const void* keys, const void* vals, void* out, size_t n,
                     const void* init, cudaStream_t s);
// compaction with built-in selectors: CM_NOT_EQUAL (value) or CM_UNIQUE; count is synchronous
bool compact_raw(int tc, int mode, const void* in, void* out, size_t n, const void* value, cudaStream_t s,
                 unsigned long long* count);

// batched segmented sort + exclusive scan (launch_segmented.cu); 4-byte values
size_t segmented_workspace_bytes(int tc, size_t n, size_t nseg);
int segmented_tuned_items(int tc);
bool segmented_sort_scan_raw(int tc, void* keys, void* vals, void* scan, const unsigned long long* off, size_t nseg,
                             size_t n, void* ws, size_t ws_bytes, bool desc, cudaStream_t s);
bool segmented_autotune(int tc, const unsigned long long* off, size_t nseg, size_t n, cudaStream_t s, int* chosen);
std::string segmented_tuning_json();
bool segmented_tuning_load(const char* json);

}  // namespace trtc_host
