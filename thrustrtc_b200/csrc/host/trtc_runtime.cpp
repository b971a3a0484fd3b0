// trtc_runtime.cpp -- device init, error reporting, workspaces, stream-ordered temporaries.
#include "trtc_runtime.h"

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace trtc_host {

static thread_local std::string t_last_error;
static std::atomic<unsigned long long> g_launches{0};

void set_error(const std::string& msg) {
    t_last_error = msg;
    fprintf(stderr, "[thrustrtc_b200] %s\n", msg.c_str());
}
const char* last_error() { return t_last_error.c_str(); }

bool cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(std::string(what) + " failed: " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
    return false;
}

void count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

namespace {
struct KtMark { std::string name; cudaEvent_t ev; cudaStream_t s; };
std::atomic<bool> g_kt_on{false};
std::mutex g_kt_mu;
std::vector<KtMark> g_kt;
std::vector<cudaEvent_t> g_kt_free;
std::vector<std::pair<std::string, float>> g_kt_done;
}  // namespace

void ktimer_enable(bool on) {
    std::lock_guard<std::mutex> lk(g_kt_mu);
    for (auto& m : g_kt) g_kt_free.push_back(m.ev);
    g_kt.clear();
    g_kt_done.clear();
    g_kt_on.store(on, std::memory_order_relaxed);
}

void ktimer_mark(const char* name, cudaStream_t s) {
    if (!g_kt_on.load(std::memory_order_relaxed)) return;
    std::lock_guard<std::mutex> lk(g_kt_mu);
    cudaEvent_t e;
    if (!g_kt_free.empty()) { e = g_kt_free.back(); g_kt_free.pop_back(); }
    else if (cudaEventCreate(&e) != cudaSuccess) return;
    if (cudaEventRecord(e, s) != cudaSuccess) { g_kt_free.push_back(e); return; }
    g_kt.push_back({name, e, s});
}

int ktimer_count() {
    std::lock_guard<std::mutex> lk(g_kt_mu);
    // resolve pending marks into (name, ms) pairs
    for (size_t i = 0; i < g_kt.size(); i++) {
        if (cudaEventSynchronize(g_kt[i].ev) != cudaSuccess) return -1;
        if (g_kt[i].name.empty()) continue;
        for (size_t j = i; j-- > 0;) {
            if (g_kt[j].s != g_kt[i].s) continue;
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, g_kt[j].ev, g_kt[i].ev) == cudaSuccess) g_kt_done.push_back({g_kt[i].name, ms});
            break;
        }
    }
    for (auto& m : g_kt) g_kt_free.push_back(m.ev);
    g_kt.clear();
    return (int)g_kt_done.size();
}

bool ktimer_get(int i, std::string& name, float& ms) {
    std::lock_guard<std::mutex> lk(g_kt_mu);
    if (i < 0 || (size_t)i >= g_kt_done.size()) return false;
    name = g_kt_done[i].first;
    ms = g_kt_done[i].second;
    return true;
}

int type_code_of(const std::string& c) {
    if (c == "int8_t" || c == "char" || c == "signed char") return TC_I8;
    if (c == "uint8_t" || c == "unsigned char" || c == "bool") return c == "bool" ? TC_NONE : TC_U8;
    if (c == "int16_t" || c == "short") return TC_I16;
    if (c == "uint16_t" || c == "unsigned short") return TC_U16;
    if (c == "int32_t" || c == "int") return TC_I32;
    if (c == "uint32_t" || c == "unsigned int" || c == "unsigned") return TC_U32;
    if (c == "int64_t" || c == "long long") return TC_I64;
    if (c == "uint64_t" || c == "unsigned long long" || c == "size_t") return TC_U64;
    if (c == "float") return TC_F32;
    if (c == "double") return TC_F64;
    return TC_NONE;
}

size_t type_size(int tc) {
    static const size_t sz[] = {1, 1, 2, 2, 4, 4, 8, 8, 4, 8};
    return (tc >= 0 && tc <= 9) ? sz[tc] : 0;
}

static std::mutex g_mu;
static bool g_inited = false;
static bool g_init_ok = false;
static uint32_t* g_err_host = nullptr;
static uint32_t* g_err_dev = nullptr;
static int g_sms = 0;
static cudaMemPool_t g_vec_pool = nullptr;
// freed DVVector storage kept mapped for the next vectors; above this the pool gives memory
// back to the device at the next synchronisation
static const uint64_t kVectorCacheBytes = 8ull << 30;

bool ensure_device() {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_inited) return g_init_ok;
    g_inited = true;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) {
        cudaGetLastError();
        set_error("no CUDA device is available");
        return false;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    if (!TRTC_CUDA(cudaHostAlloc((void**)&g_err_host, sizeof(uint32_t), cudaHostAllocMapped))) return false;
    *g_err_host = 0;
    if (!TRTC_CUDA(cudaHostGetDevicePointer((void**)&g_err_dev, g_err_host, 0))) return false;
    // keep freed temporaries cached in the default pool instead of returning them
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    // DVVector storage: a pool of its own, so that creating and destroying vectors reuses
    // mapped memory instead of mapping and unmapping device pages in cudaMalloc / cudaFree
    // (TRTC_VECTOR_POOL=0 keeps one cudaMalloc per vector, e.g. for CUDA IPC export)
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    const char* vp = getenv("TRTC_VECTOR_POOL");
    if (vp && std::string(vp) == "0") {
        g_vec_pool = nullptr;
    } else if (cudaMemPoolCreate(&g_vec_pool, &props) == cudaSuccess) {
        uint64_t thr = kVectorCacheBytes;
        cudaMemPoolSetAttribute(g_vec_pool, cudaMemPoolAttrReleaseThreshold, &thr);
    } else {
        cudaGetLastError();
        g_vec_pool = nullptr;
    }
    g_init_ok = true;
    return true;
}

int sm_count() { return g_sms > 0 ? g_sms : 148; }

uint32_t* device_error_word() { return g_err_dev; }

bool check_device_errors(cudaStream_t s, const char* what) {
    if (!TRTC_CUDA(cudaStreamSynchronize(s))) return false;
    if (!TRTC_CUDA(cudaGetLastError())) return false;
    if (g_err_host && *(volatile uint32_t*)g_err_host) {
        const uint32_t e = *(volatile uint32_t*)g_err_host;
        *(volatile uint32_t*)g_err_host = 0;
        char buf[200];
        snprintf(buf, sizeof(buf), "%s: device reported error 0x%x (%s%s%s)", what, e,
                 (e & 1u) ? "look-back wait exceeded its bound; " : "",
                 (e & 4u) ? "bulk tile copy did not complete within its bound; " : "",
                 (e & 2u) ? "inconsistent sort plan" : "");
        set_error(buf);
        return false;
    }
    return true;
}

// ---------------------------------------------------------------- workspaces
static std::map<cudaStream_t, LookbackWs*> g_ws;

static LookbackWs* ws_for(cudaStream_t s) {
    auto it = g_ws.find(s);
    if (it != g_ws.end()) return it->second;
    LookbackWs* w = new LookbackWs();
    g_ws[s] = w;
    return w;
}

LookbackWs* lookback_ws(cudaStream_t s, size_t tiles, size_t value_size, uint32_t* epoch8) {
    std::lock_guard<std::mutex> lk(g_mu);
    LookbackWs* w = ws_for(s);
    if (value_size < 8) value_size = 8;
    const bool grow = tiles > w->tiles_cap || value_size > w->value_cap;
    if (grow || w->epoch >= (1u << 28)) {
        // the old arrays may still be in use by queued work on this stream
        cudaStreamSynchronize(s);
        if (grow) {
            size_t cap = tiles > w->tiles_cap ? tiles : w->tiles_cap;
            if (cap < 1024) cap = 1024;
            size_t vcap = value_size > w->value_cap ? value_size : w->value_cap;
            cudaFree(w->flags); cudaFree(w->agg); cudaFree(w->incl); cudaFree(w->packed);
            if (!TRTC_CUDA(cudaMalloc(&w->flags, cap * 4)) || !TRTC_CUDA(cudaMalloc(&w->agg, cap * vcap)) ||
                !TRTC_CUDA(cudaMalloc(&w->incl, cap * vcap)) || !TRTC_CUDA(cudaMalloc(&w->packed, cap * 8))) {
                w->tiles_cap = 0;
                return nullptr;
            }
            w->tiles_cap = cap;
            w->value_cap = vcap;
        }
        if (!w->tile_ctr) {
            if (!TRTC_CUDA(cudaMalloc(&w->tile_ctr, 16)) || !TRTC_CUDA(cudaMalloc(&w->result, 16))) return nullptr;
        }
        cudaMemset(w->flags, 0, w->tiles_cap * 4);
        cudaMemset(w->packed, 0, w->tiles_cap * 8);
        cudaMemset(w->tile_ctr, 0, 16);
        cudaDeviceSynchronize();
        w->epoch = 0;
    }
    w->epoch += 1;
    *epoch8 = w->epoch * 8u;
    return w;
}

LookbackWs* reduce_ws(cudaStream_t s, size_t partials, size_t value_size) {
    std::lock_guard<std::mutex> lk(g_mu);
    LookbackWs* w = ws_for(s);
    if (value_size < 8) value_size = 8;
    if (partials * value_size > w->partials_cap || !w->done_ctr) {
        cudaStreamSynchronize(s);
        cudaFree(w->partials); cudaFree(w->partial_has);
        const size_t cap = partials < 4096 ? 4096 : partials;
        if (!TRTC_CUDA(cudaMalloc(&w->partials, cap * 16)) || !TRTC_CUDA(cudaMalloc(&w->partial_has, cap * 4)))
            return nullptr;
        w->partials_cap = cap * 16;
        if (!w->done_ctr) {
            if (!TRTC_CUDA(cudaMalloc(&w->done_ctr, 16))) return nullptr;
            cudaMemset(w->done_ctr, 0, 16);
        }
        if (!w->result) {
            if (!TRTC_CUDA(cudaMalloc(&w->result, 16))) return nullptr;
        }
        cudaDeviceSynchronize();
    }
    return w;
}

void* sort_ctrl_ws(cudaStream_t s, size_t bytes) {
    std::lock_guard<std::mutex> lk(g_mu);
    LookbackWs* w = ws_for(s);
    if (!w->sort_ctrl) {
        if (!TRTC_CUDA(cudaMalloc(&w->sort_ctrl, bytes))) return nullptr;
    }
    return w->sort_ctrl;
}

unsigned tile_prefetch_ahead(size_t tiles) {
    static const bool on = [] {
        const char* e = getenv("TRTC_TILE_PREFETCH");
        return !(e && std::string(e) == "0");
    }();
    return on ? (unsigned)tiles : 0u;
}

// ---------------------------------------------------------------- allocation cap
static std::atomic<unsigned long long> g_alloc_limit{0};
void set_alloc_limit(unsigned long long bytes) { g_alloc_limit.store(bytes, std::memory_order_relaxed); }

static bool within_alloc_limit(size_t bytes, const char* what) {
    const unsigned long long lim = g_alloc_limit.load(std::memory_order_relaxed);
    if (lim == 0 || bytes <= lim) return true;
    set_error(std::string(what) + ": allocation of " + std::to_string(bytes) + " bytes exceeds the limit of " +
              std::to_string(lim) + " bytes (trtc_set_alloc_limit)");
    return false;
}

void* tmp_alloc(size_t bytes, cudaStream_t s) {
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    if (!within_alloc_limit(bytes, "temporary")) return nullptr;
    if (!TRTC_CUDA(cudaMallocAsync(&p, bytes, s))) return nullptr;
    return p;
}
void tmp_free(void* p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

void* vector_alloc(size_t bytes) {
    void* p = nullptr;
    if (!within_alloc_limit(bytes, "vector")) return nullptr;
    if (!g_vec_pool) return TRTC_CUDA(cudaMalloc(&p, bytes)) ? p : nullptr;
    // ordered on the legacy default stream, like the copy or memset that fills the vector
    if (cudaMallocFromPoolAsync(&p, bytes, g_vec_pool, 0) == cudaSuccess) return p;
    cudaGetLastError();
    // out of memory: give the cached blocks of both pools back to the device, then retry once
    cudaDeviceSynchronize();
    int dev = 0;
    cudaMemPool_t def;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&def, dev) == cudaSuccess)
        cudaMemPoolTrimTo(def, 0);
    cudaMemPoolTrimTo(g_vec_pool, 0);
    p = nullptr;
    return TRTC_CUDA(cudaMallocFromPoolAsync(&p, bytes, g_vec_pool, 0)) ? p : nullptr;
}
void vector_free(void* p) {
    if (!p) return;
    if (!g_vec_pool) {
        cudaFree(p);
        return;
    }
    // cudaFree waits for all work on the device before the memory can be reused; keep that
    // for work on other streams that may still read the vector
    cudaDeviceSynchronize();
    cudaFreeAsync(p, 0);
}

}  // namespace trtc_host
