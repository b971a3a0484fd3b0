// trtc_server.cu -- a request server over the hot path: Sort_By_Key, exclusive scan and
// reduce requests arrive one by one and are served with continuous batching.
//
//   * admission: a request group is launched only when the device memory its temporaries
//     need fits in the server's budget next to the groups already running;
//   * coalescing: requests of at most `coalesce_max_n` elements of the same kind and element
//     type that are waiting together are served by one segmented launch (each request is a
//     segment with its own arrays); larger requests run alone on the plain kernels;
//   * overlap: groups run on a fixed set of non-blocking streams, so requests that arrive
//     while others are on the GPU start as soon as a stream and the memory are free;
//   * temporaries come from the CUDA stream-ordered memory pool (kept resident by the
//     library's release threshold); the request inputs and outputs are the client's device
//     buffers.
// No counterpart in the reference, which serves one blocking call at a time on stream 0.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "../device/trtc_segmented.cuh"
#include "trtc_launch.h"
#include "trtc_runtime.h"

namespace trtc_host {

using namespace trtc;

namespace {

enum : int { REQ_SORT_BY_KEY = 0, REQ_EXCL_SCAN = 1, REQ_REDUCE = 2 };
enum : int { ST_QUEUED = 0, ST_RUNNING = 1, ST_DONE = 2, ST_ERROR = -1 };
constexpr size_t MAX_GROUP = 4096;  // requests per coalesced launch

struct Req {
    long long id;
    int kind, type;
    void *k, *v, *out;
    size_t n;
    double t_submit = 0, t_done = 0;
    int state = ST_QUEUED;
    double result = 0;          // reduce: the sum, converted to double
    unsigned long long raw = 0;  // reduce: the sum's bytes (little-endian, element size)
    size_t temp = 0;
};

struct Slot {  // one stream and its pinned staging
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;
    SegItem* h_items = nullptr;           // pinned
    unsigned long long* h_res = nullptr;  // pinned result words (reduce)
    bool busy = false;
    std::vector<long long> ids;
    size_t temp = 0;
    void* dev = nullptr;  // group temporaries (one stream-ordered allocation)
};

size_t esize(int t) { return (t == TC_I64 || t == TC_U64 || t == TC_F64) ? 8 : 4; }
size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

template <class T>
double as_double(unsigned long long w) {
    T t;
    memcpy(&t, &w, sizeof(T));
    return (double)t;
}

}  // namespace

class Server {
public:
    Server(size_t budget, int nstreams, size_t coalesce_max)
        : budget_(budget), coalesce_max_(coalesce_max), t0_(std::chrono::steady_clock::now()) {
        slots_.resize(nstreams < 1 ? 1 : nstreams);
        for (auto& sl : slots_) {
            ok_ = ok_ && TRTC_CUDA(cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking)) &&
                  TRTC_CUDA(cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming)) &&
                  TRTC_CUDA(cudaHostAlloc((void**)&sl.h_items, MAX_GROUP * sizeof(SegItem), cudaHostAllocDefault)) &&
                  TRTC_CUDA(cudaHostAlloc((void**)&sl.h_res, MAX_GROUP * 8, cudaHostAllocDefault));
        }
    }
    ~Server() {
        for (auto& sl : slots_) {
            if (sl.s) cudaStreamSynchronize(sl.s);
            if (sl.dev) cudaFreeAsync(sl.dev, sl.s);
            if (sl.s) { cudaStreamSynchronize(sl.s); cudaStreamDestroy(sl.s); }
            if (sl.ev) cudaEventDestroy(sl.ev);
            if (sl.h_items) cudaFreeHost(sl.h_items);
            if (sl.h_res) cudaFreeHost(sl.h_res);
        }
    }
    bool ok() const { return ok_; }
    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
    }

    long long submit(int kind, int type, void* k, void* v, void* out, size_t n) {
        std::lock_guard<std::mutex> lk(mu_);
        if (kind < 0 || kind > 2) { set_error("server: unknown request kind"); return -1; }
        if (!(type == TC_U32 || type == TC_I32 || type == TC_F32 || type == TC_I64 || type == TC_U64)) {
            set_error("server: element type must be int32, uint32, float, int64 or uint64");
            return -1;
        }
        if (n == 0 || !k || (kind == REQ_SORT_BY_KEY && !v) || (kind == REQ_EXCL_SCAN && !out)) {
            set_error("server: empty request or missing buffer");
            return -1;
        }
        Req r;
        r.id = next_id_++;
        r.kind = kind; r.type = type; r.k = k; r.v = v; r.out = out; r.n = n;
        r.temp = temp_bytes(r);
        if (r.temp > budget_) { set_error("server: request needs more temporary memory than the budget"); return -1; }
        r.t_submit = now();
        reqs_[r.id] = r;
        queue_.push_back(r.id);
        return r.id;
    }

    // Retires finished groups, then launches queued requests while streams and memory allow.
    // Returns the number of requests queued or running, or -1 on a failure.
    int poll() {
        std::lock_guard<std::mutex> lk(mu_);
        for (auto& sl : slots_) {
            if (!sl.busy) continue;
            const cudaError_t q = cudaEventQuery(sl.ev);
            if (q == cudaErrorNotReady) continue;
            if (!cuda_ok(q, "server: group") || !check_device_errors(sl.s, "server")) { fail_group(sl); return -1; }
            retire(sl);
        }
        while (!queue_.empty()) {
            Slot* free_slot = nullptr;
            for (auto& sl : slots_) if (!sl.busy) { free_slot = &sl; break; }
            if (!free_slot) break;
            if (!launch_next(*free_slot)) break;
        }
        int active = (int)queue_.size();
        for (auto& sl : slots_) if (sl.busy) active += (int)sl.ids.size();
        return failed_ ? -1 : active;
    }

    int info(long long id, double* ts, double* td, double* res) {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = reqs_.find(id);
        if (it == reqs_.end()) { set_error("server: unknown request"); return ST_ERROR; }
        if (ts) *ts = it->second.t_submit;
        if (td) *td = it->second.t_done;
        if (res) *res = it->second.result;
        return it->second.state;
    }

    bool raw_result(long long id, unsigned long long* out) {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = reqs_.find(id);
        if (it == reqs_.end() || it->second.state != ST_DONE) { set_error("server: no result for this request"); return false; }
        *out = it->second.raw;
        return true;
    }

    void forget_done() {
        std::lock_guard<std::mutex> lk(mu_);
        for (auto it = reqs_.begin(); it != reqs_.end();)
            it = (it->second.state == ST_DONE) ? reqs_.erase(it) : std::next(it);
    }

private:
    size_t temp_bytes(const Req& r) const {
        const size_t e = esize(r.type);
        if (r.kind == REQ_SORT_BY_KEY) {
            // plain radix sort: two temp key and value arrays + status; segmented: one of each,
            // plus (float keys) the NaN-rotation tree slots (16 bytes per 128 keys + 4 per request)
            if (r.n > coalesce_max_) return 2 * r.n * (e + 4) + (r.n / 1024 + 1) * 4096;
            return a256(r.n * (e + 4)) + (r.type == TC_F32 ? r.n / 8 + 96 : 0);
        }
        return 4096;
    }

    void retire(Slot& sl) {
        const double t = now();
        for (size_t i = 0; i < sl.ids.size(); i++) {
            Req& r = reqs_[sl.ids[i]];
            r.state = ST_DONE;
            r.t_done = t;
            if (r.kind == REQ_REDUCE) {
                r.raw = sl.h_res[i];
                if (esize(r.type) == 4) r.raw &= 0xFFFFFFFFull;
                switch (r.type) {
                    case TC_U32: r.result = as_double<uint32_t>(sl.h_res[i]); break;
                    case TC_I32: r.result = as_double<int32_t>(sl.h_res[i]); break;
                    case TC_F32: r.result = as_double<float>(sl.h_res[i]); break;
                    case TC_I64: r.result = as_double<long long>(sl.h_res[i]); break;
                    default: r.result = as_double<unsigned long long>(sl.h_res[i]); break;
                }
            }
        }
        if (sl.dev) { cudaFreeAsync(sl.dev, sl.s); sl.dev = nullptr; }
        used_ -= sl.temp;
        sl.temp = 0;
        sl.ids.clear();
        sl.busy = false;
    }

    void fail_group(Slot& sl) {
        for (long long id : sl.ids) reqs_[id].state = ST_ERROR;
        used_ -= sl.temp;
        sl.temp = 0;
        sl.ids.clear();
        sl.busy = false;
        failed_ = true;
    }

    bool launch_next(Slot& sl) {
        const long long head = queue_.front();
        const Req& h = reqs_[head];
        if (used_ + h.temp > budget_) return false;  // admission: wait for memory
        std::vector<long long> group{head};
        size_t temp = h.temp;
        if (h.n <= coalesce_max_) {
            // coalesce queued requests of the same kind and type (in arrival order)
            for (size_t i = 1; i < queue_.size() && group.size() < MAX_GROUP; i++) {
                const Req& r = reqs_[queue_[i]];
                if (r.kind != h.kind || r.type != h.type || r.n > coalesce_max_) continue;
                if (used_ + temp + r.temp > budget_) break;
                group.push_back(r.id);
                temp += r.temp;
            }
        }
        // remove the group from the queue (the head alone: O(1), so a long backlog of plain
        // requests costs no host time per launch)
        if (group.size() == 1) {
            queue_.pop_front();
        } else {
            std::deque<long long> rest;
            size_t gi = 0;
            for (long long id : queue_) {
                if (gi < group.size() && id == group[gi]) { gi++; continue; }
                rest.push_back(id);
            }
            queue_.swap(rest);
        }
        sl.ids = group;
        sl.temp = temp;
        used_ += temp;
        sl.busy = true;
        for (long long id : group) reqs_[id].state = ST_RUNNING;
        const bool ok = (group.size() == 1 && h.n > coalesce_max_) ? run_plain(sl, reqs_[head]) : run_group(sl);
        if (!ok || !TRTC_CUDA(cudaEventRecord(sl.ev, sl.s))) { fail_group(sl); return false; }
        return true;
    }

    bool run_plain(Slot& sl, Req& r) {
        switch (r.kind) {
            case REQ_SORT_BY_KEY: return sort_raw(r.type, r.k, r.v, 4, r.n, false, sl.s);
            case REQ_EXCL_SCAN: {
                unsigned long long zero = 0;
                return scan_raw(r.type, OP_PLUS, 1, r.k, r.out, r.n, &zero, sl.s);
            }
            default: {
                void* res = nullptr;
                return reduce_raw_async(r.type, OP_PLUS, r.k, r.n, nullptr, &res, sl.s) &&
                       TRTC_CUDA(cudaMemcpyAsync(sl.h_res, res, esize(r.type), cudaMemcpyDeviceToHost, sl.s));
            }
        }
    }

    // one segmented launch for the whole group: items array (H2D from pinned staging),
    // control block, temporaries, results (reduce)
    bool run_group(Slot& sl) {
        const size_t g = sl.ids.size();
        const Req& h = reqs_[sl.ids[0]];
        const size_t e = esize(h.type);
        // largest first (the queue order of the persistent kernel)
        std::vector<long long> order(sl.ids);
        std::sort(order.begin(), order.end(), [&](long long a, long long b) { return reqs_[a].n > reqs_[b].n; });
        sl.ids = order;
        size_t tn = 0;
        for (size_t i = 0; i < g; i++) {
            const Req& r = reqs_[order[i]];
            SegItem it;
            it.k = r.k;
            it.v = r.v;
            it.out = (r.kind == REQ_EXCL_SCAN) ? r.out : nullptr;
            it.n = r.n;
            it.toff = tn;
            if (r.kind == REQ_SORT_BY_KEY) tn += r.n;
            sl.h_items[i] = it;
        }
        const size_t items_bytes = a256(g * sizeof(SegItem));
        const size_t ctrl_bytes = a256(sizeof(SegCtrl));
        const size_t res_bytes = a256(g * 8);
        const size_t tk_bytes = a256(tn * e), tv_bytes = a256(tn * 4);
        // float sorts: per-request NaN-rotation counts and Min_Element tree slots
        const bool fsort = h.kind == REQ_SORT_BY_KEY && h.type == TC_F32;
        const size_t rot_bytes = fsort ? a256(g * 4) : 0;
        const size_t tree_bytes = fsort ? a256(seg_tree_slots(tn, g) * sizeof(SegMinSlot<float>)) : 0;
        const size_t bytes = items_bytes + ctrl_bytes + res_bytes + tk_bytes + tv_bytes + rot_bytes + tree_bytes;
        if (!TRTC_CUDA(cudaMallocAsync(&sl.dev, bytes, sl.s))) { sl.dev = nullptr; return false; }
        unsigned char* p = (unsigned char*)sl.dev;
        SegItem* d_items = (SegItem*)p;
        SegCtrl* ctrl = (SegCtrl*)(p + items_bytes);
        unsigned long long* d_res = (unsigned long long*)(p + items_bytes + ctrl_bytes);
        void* tk = p + items_bytes + ctrl_bytes + res_bytes;
        void* tv = (unsigned char*)tk + tk_bytes;
        uint32_t* rot = (uint32_t*)((unsigned char*)tv + tv_bytes);
        void* tree = (unsigned char*)rot + rot_bytes;
        if (h.kind == REQ_REDUCE)
            for (size_t i = 0; i < g; i++) sl.h_items[i].out = d_res + i;
        if (!TRTC_CUDA(cudaMemcpyAsync(d_items, sl.h_items, g * sizeof(SegItem), cudaMemcpyHostToDevice, sl.s)) ||
            !TRTC_CUDA(cudaMemsetAsync(ctrl, 0, sizeof(SegCtrl), sl.s)) ||
            !TRTC_CUDA(cudaMemsetAsync(d_res, 0, g * 8, sl.s)))
            return false;
        const int sms = sm_count();
        const unsigned grid = (unsigned)std::min<size_t>(g, (size_t)sms * 2);
        switch (h.kind) {
            case REQ_SORT_BY_KEY: {
                if (!group_sort(h.type, d_items, g, ctrl, tk, tv, rot, tree, grid, sl.s)) return false;
                break;
            }
            case REQ_EXCL_SCAN: {
                switch (h.type) {
                    case TC_U32: seg_scan_list_kernel<uint32_t, 8><<<grid, 256, 0, sl.s>>>(d_items, g, ctrl); break;
                    case TC_I32: seg_scan_list_kernel<int32_t, 8><<<grid, 256, 0, sl.s>>>(d_items, g, ctrl); break;
                    case TC_F32: seg_scan_list_kernel<float, 8><<<grid, 256, 0, sl.s>>>(d_items, g, ctrl); break;
                    case TC_I64: seg_scan_list_kernel<long long, 4><<<grid, 256, 0, sl.s>>>(d_items, g, ctrl); break;
                    default: seg_scan_list_kernel<unsigned long long, 4><<<grid, 256, 0, sl.s>>>(d_items, g, ctrl); break;
                }
                count_launch();
                break;
            }
            default: {
                switch (h.type) {
                    case TC_U32: seg_reduce_list_kernel<uint32_t><<<grid, 256, 0, sl.s>>>(d_items, g, ctrl); break;
                    case TC_I32: seg_reduce_list_kernel<int32_t><<<grid, 256, 0, sl.s>>>(d_items, g, ctrl); break;
                    case TC_F32: seg_reduce_list_kernel<float><<<grid, 256, 0, sl.s>>>(d_items, g, ctrl); break;
                    case TC_I64: seg_reduce_list_kernel<long long><<<grid, 256, 0, sl.s>>>(d_items, g, ctrl); break;
                    default: seg_reduce_list_kernel<unsigned long long><<<grid, 256, 0, sl.s>>>(d_items, g, ctrl); break;
                }
                count_launch();
                if (!TRTC_CUDA(cudaMemcpyAsync(sl.h_res, d_res, g * 8, cudaMemcpyDeviceToHost, sl.s))) return false;
                break;
            }
        }
        return TRTC_CUDA(cudaGetLastError());
    }

    template <class K>
    static bool group_sort_k(SegItem* items, size_t g, SegCtrl* ctrl, void* tk, void* tv, uint32_t* rot, void* tree,
                             unsigned grid, cudaStream_t s) {
        constexpr int ITEMS = 8;
        typedef typename RadixKey<K>::B KB;
        constexpr size_t smem = seg_sort_scan_smem<K, uint32_t, ITEMS>();
        // 2 CTAs per SM: a group ends with its longest request, sorted by one CTA through
        // global memory, which runs faster with the larger register budget (measured: the
        // 4-CTA build of the batch kernel cut the serving capacity from 19,750 to 16,350/s)
        auto kernel = seg_sort_scan_kernel<K, uint32_t, unsigned long long, false, ITEMS, 2>;
        static bool attr = false;
        if (!attr) {
            if (!TRTC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
                return false;
            attr = true;
        }
        constexpr bool FK = is_same<K, float>::value;
        if constexpr (FK) {
            // the reference's NaN rotation per request (as its own Sort_By_Key call applies it)
            seg_rot_kernel<K, unsigned long long><<<grid, 256, 0, s>>>(nullptr, nullptr, items, g,
                                                                       (SegMinSlot<K>*)tree, rot);
            count_launch();
        }
        kernel<<<grid, 256, smem, s>>>(nullptr, nullptr, nullptr, (KB*)tk, (uint32_t*)tv, nullptr, nullptr, g, ctrl,
                                       items, 32u);
        count_launch();
        if constexpr (FK) {
            seg_rotate_kernel<K, uint32_t, unsigned long long, false><<<grid, 256, 0, s>>>(
                nullptr, nullptr, nullptr, (KB*)tk, (uint32_t*)tv, nullptr, items, g, rot);
            count_launch();
        }
        return true;
    }

    static bool group_sort(int type, SegItem* items, size_t g, SegCtrl* ctrl, void* tk, void* tv, uint32_t* rot,
                           void* tree, unsigned grid, cudaStream_t s) {
        switch (type) {
            case TC_U32: return group_sort_k<uint32_t>(items, g, ctrl, tk, tv, rot, tree, grid, s);
            case TC_I32: return group_sort_k<int32_t>(items, g, ctrl, tk, tv, rot, tree, grid, s);
            case TC_F32: return group_sort_k<float>(items, g, ctrl, tk, tv, rot, tree, grid, s);
            case TC_I64: return group_sort_k<int64_t>(items, g, ctrl, tk, tv, rot, tree, grid, s);
            default: return group_sort_k<uint64_t>(items, g, ctrl, tk, tv, rot, tree, grid, s);
        }
    }

    std::mutex mu_;
    size_t budget_, coalesce_max_, used_ = 0;
    std::chrono::steady_clock::time_point t0_;
    std::vector<Slot> slots_;
    std::deque<long long> queue_;
    std::unordered_map<long long, Req> reqs_;
    long long next_id_ = 1;
    bool ok_ = true, failed_ = false;
};

}  // namespace trtc_host

using trtc_host::Server;

extern "C" {

void* trtc_server_create(unsigned long long budget_bytes, int num_streams, unsigned long long coalesce_max_n) {
    if (!trtc_host::ensure_device()) return nullptr;
    Server* s = new Server((size_t)budget_bytes, num_streams, (size_t)coalesce_max_n);
    if (!s->ok()) { delete s; return nullptr; }
    return s;
}

long long trtc_server_submit(void* srv, int kind, int type, void* keys, void* values, void* out,
                             unsigned long long n) {
    return static_cast<Server*>(srv)->submit(kind, type, keys, values, out, (size_t)n);
}

int trtc_server_poll(void* srv) { return static_cast<Server*>(srv)->poll(); }

int trtc_server_info(void* srv, long long id, double* t_submit, double* t_done, double* result) {
    return static_cast<Server*>(srv)->info(id, t_submit, t_done, result);
}

int trtc_server_result(void* srv, long long id, void* out8) {
    return static_cast<Server*>(srv)->raw_result(id, (unsigned long long*)out8) ? 0 : -1;
}

double trtc_server_now(void* srv) { return static_cast<Server*>(srv)->now(); }

void trtc_server_forget_done(void* srv) { static_cast<Server*>(srv)->forget_done(); }

void trtc_server_destroy(void* srv) { delete static_cast<Server*>(srv); }

}  // extern "C"
