// trtc_runtime.h -- host runtime shared by the launchers, the JIT engine and the C ABI.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

namespace trtc_host {

// element type codes shared by the raw C ABI and the oracle
enum TypeCode : int {
    TC_I8 = 0, TC_U8 = 1, TC_I16 = 2, TC_U16 = 3, TC_I32 = 4, TC_U32 = 5,
    TC_I64 = 6, TC_U64 = 7, TC_F32 = 8, TC_F64 = 9, TC_NONE = -1
};
enum OpCode : int { OP_PLUS = 0, OP_MAX = 1, OP_MIN = 2 };

int type_code_of(const std::string& elem_cls);   // -1 if not a built-in arithmetic type
size_t type_size(int tc);

// ---- errors: the last failure of this thread, and the device-side error word
void set_error(const std::string& msg);
const char* last_error();
bool cuda_ok(cudaError_t e, const char* what);
#define TRTC_CUDA(call) ::trtc_host::cuda_ok((call), #call)

bool ensure_device();                 // initialises the CUDA context once
uint32_t* device_error_word();        // mapped host word that kernels report into
bool check_device_errors(cudaStream_t s, const char* what);  // syncs s, reads + clears the word

// ---- launch accounting (kernels of this library launched so far)
void count_launch(unsigned n = 1);
unsigned long long launch_count();

// ---- optional per-launch timing (off by default).  While enabled, launchers record a CUDA
// event on the launching stream after each kernel (ktimer_mark(name)); a mark with an empty
// name only opens an interval.  The duration of a named mark is the time since the previous
// mark on the same stream.
void ktimer_enable(bool on);          // also discards recorded marks
void ktimer_mark(const char* name, cudaStream_t s);
int ktimer_count();                   // synchronises the recorded events
bool ktimer_get(int i, std::string& name, float& ms);

// ---- per-stream look-back workspace
struct LookbackWs {
    uint32_t* flags = nullptr;
    void* agg = nullptr;
    void* incl = nullptr;
    unsigned long long* packed = nullptr;  // flag + value words for values of <= 4 bytes
    unsigned long long* tile_ctr = nullptr;
    unsigned long long* result = nullptr;  // device scalar (count / total)
    size_t tiles_cap = 0;
    size_t value_cap = 0;                  // bytes per agg/incl entry capacity
    uint32_t epoch = 0;
    // reduce helpers
    void* partials = nullptr;
    int* partial_has = nullptr;
    uint32_t* done_ctr = nullptr;
    size_t partials_cap = 0;
    // sort control block
    void* sort_ctrl = nullptr;
};
// Reserves room for `tiles` tiles of `value_size`-byte values; returns the workspace with
// its flag epoch advanced for one launch.
LookbackWs* lookback_ws(cudaStream_t s, size_t tiles, size_t value_size, uint32_t* epoch8);
LookbackWs* reduce_ws(cudaStream_t s, size_t partials, size_t value_size);
void* sort_ctrl_ws(cudaStream_t s, size_t bytes);

// cap on the size of any one temporary or vector allocation (0: none); an allocation above it
// fails like an out-of-memory one, before anything is launched
void set_alloc_limit(unsigned long long bytes);
// L2 prefetch distance, in tiles, of the kernels that claim tiles in order: `tiles` (the
// persistent kernels pass half their grid; the sort's digit pass 1.5 tiles per SM), or 0 when
// TRTC_TILE_PREFETCH=0 is set in the environment
unsigned tile_prefetch_ahead(size_t tiles);
// stream-ordered temporaries (cached by the CUDA memory pool)
void* tmp_alloc(size_t bytes, cudaStream_t s);
void tmp_free(void* p, cudaStream_t s);
// DVVector storage (a pool of its own that keeps up to 8 GiB of freed vectors mapped);
// vector_free waits for the device like cudaFree
void* vector_alloc(size_t bytes);
void vector_free(void* p);

int sm_count();

}  // namespace trtc_host
