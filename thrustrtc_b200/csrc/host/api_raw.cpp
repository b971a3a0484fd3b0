// api_raw.cpp -- raw-pointer C ABI (include/trtc_raw.h): built-in element types on device
// buffers the caller owns, on a caller-chosen stream.  The object-model ABI of
// include/thrustrtc_b200.h is layered on the same launchers.
#include <cstring>
#include "trtc_jit.h"
#include "trtc_launch.h"
#include "trtc_runtime.h"

using namespace trtc_host;

static inline cudaStream_t S(void* s) { return (cudaStream_t)s; }

extern "C" {

const char* trtc_last_error() { return last_error(); }

unsigned long long trtc_launch_count() { return launch_count(); }

void trtc_timing_enable(int on) { ktimer_enable(on != 0); }
int trtc_timing_count() { return ktimer_count(); }
int trtc_timing_get(int i, char* name, unsigned long long name_cap, float* ms) {
    std::string nm;
    float t = 0.f;
    if (!ktimer_get(i, nm, t)) return -1;
    if (name && name_cap) {
        const size_t c = nm.size() < name_cap - 1 ? nm.size() : (size_t)name_cap - 1;
        memcpy(name, nm.data(), c);
        name[c] = 0;
    }
    if (ms) *ms = t;
    return 0;
}

// Copies the sort control block of `stream` (histograms, plan, NaN flag, rotation count of
// the last sort on that stream) to host memory; for diagnostics.  Returns bytes copied.
unsigned long long trtc_debug_sort_ctrl(void* host, unsigned long long bytes, void* stream) {
    void* c = sort_ctrl_ws(S(stream), 1 << 16);
    if (!c || !host) return 0;
    if (!TRTC_CUDA(cudaMemcpyAsync(host, c, (size_t)bytes, cudaMemcpyDeviceToHost, S(stream)))) return 0;
    if (!TRTC_CUDA(cudaStreamSynchronize(S(stream)))) return 0;
    return bytes;
}

void trtc_set_alloc_limit(unsigned long long bytes) { set_alloc_limit(bytes); }

void trtc_jit_cache_stats(unsigned long long* out) {
    if (out) jit_cache_stats(out);
}

int trtc_raw_sync(void* stream) {
    if (!ensure_device()) return -1;
    return check_device_errors(S(stream), "stream") ? 0 : -1;
}

int trtc_raw_sort(int key_tc, void* keys, unsigned long long n, int descending, void* stream) {
    if (!ensure_device()) return -1;
    return sort_raw(key_tc, keys, nullptr, 0, (size_t)n, descending != 0, S(stream)) ? 0 : -1;
}

int trtc_raw_sort_by_key(int key_tc, void* keys, void* values, unsigned long long value_size, unsigned long long n,
                         int descending, void* stream) {
    if (!ensure_device()) return -1;
    if (!values || value_size == 0) { set_error("sort_by_key: no values"); return -1; }
    return sort_raw(key_tc, keys, values, (size_t)value_size, (size_t)n, descending != 0, S(stream)) ? 0 : -1;
}

unsigned long long trtc_raw_min_element(int tc, const void* in, unsigned long long n, void* stream) {
    if (!ensure_device()) return ~0ull;
    unsigned long long idx = 0;
    return min_element_raw(tc, in, (size_t)n, S(stream), &idx) ? idx : ~0ull;
}

int trtc_raw_scan(int tc, int op, int exclusive, const void* in, void* out, unsigned long long n, const void* init,
                  void* stream) {
    if (!ensure_device()) return -1;
    if (exclusive && !init) {
        static const unsigned long long zero[2] = {0, 0};
        init = zero;
    }
    return scan_raw(tc, op, exclusive ? 1 : 0, in, out, (size_t)n, init, S(stream)) ? 0 : -1;
}

int trtc_raw_reduce(int tc, int op, const void* in, unsigned long long n, const void* init, void* result_host,
                    void* stream) {
    if (!ensure_device()) return -1;
    return reduce_raw(tc, op, in, (size_t)n, init, result_host, S(stream)) ? 0 : -1;
}

int trtc_raw_reduce_async(int tc, int op, const void* in, unsigned long long n, const void* init, void** result_dev,
                          void* stream) {
    if (!ensure_device()) return -1;
    return reduce_raw_async(tc, op, in, (size_t)n, init, result_dev, S(stream)) ? 0 : -1;
}

int trtc_raw_scan_by_key(int key_tc, int val_tc, int exclusive, const void* keys, const void* vals, void* out,
                         unsigned long long n, const void* init, void* stream) {
    if (!ensure_device()) return -1;
    return scan_by_key_raw(key_tc, val_tc, exclusive ? 1 : 0, keys, vals, out, (size_t)n, init, S(stream)) ? 0 : -1;
}

unsigned long long trtc_raw_remove_copy(int tc, const void* in, void* out, unsigned long long n, const void* value,
                                        void* stream) {
    if (!ensure_device()) return ~0ull;
    unsigned long long c = 0;
    return compact_raw(tc, COMPACT_NOT_EQUAL, in, out, (size_t)n, value, S(stream), &c) ? c : ~0ull;
}

unsigned long long trtc_raw_unique_copy(int tc, const void* in, void* out, unsigned long long n, void* stream) {
    if (!ensure_device()) return ~0ull;
    unsigned long long c = 0;
    return compact_raw(tc, COMPACT_UNIQUE, in, out, (size_t)n, nullptr, S(stream), &c) ? c : ~0ull;
}

unsigned long long trtc_raw_segmented_workspace_bytes(int key_type, unsigned long long n, unsigned long long nseg) {
    return segmented_workspace_bytes(key_type, (size_t)n, (size_t)nseg);
}

int trtc_raw_segmented_sort_scan(int key_type, void* keys, void* values, void* scan_out,
                                 const unsigned long long* offsets, unsigned long long nseg, unsigned long long n,
                                 void* workspace, unsigned long long workspace_bytes, int descending, void* stream) {
    if (!ensure_device()) return -1;
    return segmented_sort_scan_raw(key_type, keys, values, scan_out, offsets, (size_t)nseg, (size_t)n, workspace,
                                   (size_t)workspace_bytes, descending != 0, S(stream)) ? 0 : -1;
}

int trtc_raw_segmented_autotune(int key_type, const unsigned long long* offsets, unsigned long long nseg,
                                unsigned long long n, void* stream) {
    int chosen = 0;
    return segmented_autotune(key_type, offsets, (size_t)nseg, (size_t)n, S(stream), &chosen) ? chosen : -1;
}

unsigned long long trtc_raw_segmented_tuning_json(char* out, unsigned long long cap) {
    const std::string j = segmented_tuning_json();
    if (out && cap) {
        const size_t c = j.size() < cap - 1 ? j.size() : (size_t)cap - 1;
        memcpy(out, j.data(), c);
        out[c] = 0;
    }
    return j.size();
}

int trtc_raw_segmented_tuning_load(const char* json) { return segmented_tuning_load(json) ? 0 : -1; }

}  // extern "C"
