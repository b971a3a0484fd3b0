// trtc_jit.cpp -- NVRTC engine, struct registry, layout reflection and JIT kernel cache.
#include "trtc_jit.h"
#include "trtc_runtime.h"

#include <cuda.h>
#include <dlfcn.h>
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <set>
#include <sstream>
#include <unordered_map>

namespace trtc_host {

extern const int g_num_device_headers;
extern const char* const g_device_header_names[];
extern const char* const g_device_header_sources[];

size_t round_up(size_t x, size_t a) { return a <= 1 ? x : (x + a - 1) / a * a; }

// ------------------------------------------------------------------ context state
static std::recursive_mutex g_jit_mu;
static bool g_verbose = false, g_kernel_debug = false;
static std::vector<std::string> g_code_blocks;
static std::vector<std::string> g_include_dirs;
static std::vector<std::pair<std::string, std::string>> g_user_headers;
static std::vector<std::pair<std::string, ViewBuf>> g_constants;
static std::string g_struct_header;
static std::set<std::string> g_struct_names;
static std::string g_nvrtc_path;

void jit_set_verbose(bool v) { g_verbose = v; }
void jit_set_kernel_debug(bool v) { g_kernel_debug = v; }
bool jit_kernel_debug() { return g_kernel_debug; }
void jit_add_code_block(const std::string& code) {
    std::lock_guard<std::recursive_mutex> lk(g_jit_mu);
    g_code_blocks.push_back(code);
}
void jit_add_include_dir(const std::string& dir) {
    std::lock_guard<std::recursive_mutex> lk(g_jit_mu);
    g_include_dirs.push_back(dir);
}
void jit_add_built_in_header(const std::string& name, const std::string& content) {
    std::lock_guard<std::recursive_mutex> lk(g_jit_mu);
    g_user_headers.emplace_back(name, content);
}
void jit_set_nvrtc_path(const std::string& path) { g_nvrtc_path = path; }

static unsigned long long fnv1a(const std::string& s, unsigned long long h = 1469598103934665603ull) {
    for (unsigned char c : s) { h ^= c; h *= 1099511628211ull; }
    return h;
}

std::string jit_add_struct(const std::string& body) {
    std::lock_guard<std::recursive_mutex> lk(g_jit_mu);
    char name[40];
    snprintf(name, sizeof(name), "_S_%016llx", fnv1a(body));
    if (g_struct_names.insert(name).second) {
        g_struct_header += std::string("struct ") + name + "\n{\n    typedef " + name + " CurType;\n" + body + "};\n";
    }
    return name;
}

void jit_add_constant_object(const std::string& name, const DeviceViewable& obj) {
    std::lock_guard<std::recursive_mutex> lk(g_jit_mu);
    g_code_blocks.push_back("__constant__ " + obj.name_view_cls() + " " + name + ";\n");
    g_constants.emplace_back(name, obj.view());
}

// ------------------------------------------------------------------ layouts
static std::unordered_map<std::string, Layout> g_layouts;

static void init_scalar_layouts() {
    static bool done = false;
    if (done) return;
    done = true;
    const char* n1[] = {"bool", "char", "signed char", "unsigned char", "int8_t", "uint8_t"};
    const char* n2[] = {"short", "unsigned short", "int16_t", "uint16_t"};
    const char* n4[] = {"int", "unsigned int", "unsigned", "int32_t", "uint32_t", "float"};
    const char* n8[] = {"long", "unsigned long", "long long", "unsigned long long", "int64_t", "uint64_t",
                        "size_t", "double"};
    for (auto s : n1) g_layouts[s] = Layout{1, 1};
    for (auto s : n2) g_layouts[s] = Layout{2, 2};
    for (auto s : n4) g_layouts[s] = Layout{4, 4};
    for (auto s : n8) g_layouts[s] = Layout{8, 8};
    g_layouts["cuFloatComplex"] = Layout{8, 8};
    g_layouts["cuDoubleComplex"] = Layout{16, 16};
    g_layouts["trtc::Nothing"] = Layout{1, 1};
}

void layout_register(const std::string& n, const Layout& l) {
    std::lock_guard<std::recursive_mutex> lk(g_jit_mu);
    init_scalar_layouts();
    g_layouts[n] = l;
}

static std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\n"), b = s.find_last_not_of(" \t\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

static bool probe_layout(const std::string& type_name, Layout& out);

bool layout_of(const std::string& type_name_in, Layout& out) {
    std::lock_guard<std::recursive_mutex> lk(g_jit_mu);
    init_scalar_layouts();
    const std::string t = trim(type_name_in);
    auto it = g_layouts.find(t);
    if (it != g_layouts.end()) { out = it->second; return true; }
    // Pair<A, B> with a top-level comma
    if (t.compare(0, 5, "Pair<") == 0 && t.back() == '>') {
        const std::string inner = t.substr(5, t.size() - 6);
        int depth = 0;
        for (size_t i = 0; i < inner.size(); i++) {
            if (inner[i] == '<') depth++;
            else if (inner[i] == '>') depth--;
            else if (inner[i] == ',' && depth == 0) {
                Layout a, b;
                if (layout_of(inner.substr(0, i), a) && layout_of(inner.substr(i + 1), b)) {
                    StructLayout sl;
                    sl.add(a);
                    sl.add(b);
                    out = sl.finish();
                    g_layouts[t] = out;
                    return true;
                }
                break;
            }
        }
    }
    if (probe_layout(t, out)) { g_layouts[t] = out; return true; }
    return false;
}

// ------------------------------------------------------------------ NVRTC + driver entry points
typedef nvrtcResult (*PFN_nvrtcCreateProgram)(nvrtcProgram*, const char*, const char*, int, const char* const*,
                                              const char* const*);
typedef nvrtcResult (*PFN_nvrtcCompileProgram)(nvrtcProgram, int, const char* const*);
typedef nvrtcResult (*PFN_nvrtcGetProgramLogSize)(nvrtcProgram, size_t*);
typedef nvrtcResult (*PFN_nvrtcGetProgramLog)(nvrtcProgram, char*);
typedef nvrtcResult (*PFN_nvrtcGetCUBINSize)(nvrtcProgram, size_t*);
typedef nvrtcResult (*PFN_nvrtcGetCUBIN)(nvrtcProgram, char*);
typedef nvrtcResult (*PFN_nvrtcDestroyProgram)(nvrtcProgram*);
typedef nvrtcResult (*PFN_nvrtcAddNameExpression)(nvrtcProgram, const char*);
typedef nvrtcResult (*PFN_nvrtcGetLoweredName)(nvrtcProgram, const char*, const char**);
typedef const char* (*PFN_nvrtcGetErrorString)(nvrtcResult);
typedef nvrtcResult (*PFN_nvrtcVersion)(int*, int*);

static struct Nvrtc {
    bool tried = false, ok = false;
    PFN_nvrtcCreateProgram create;
    PFN_nvrtcCompileProgram compile;
    PFN_nvrtcGetProgramLogSize log_size;
    PFN_nvrtcGetProgramLog log;
    PFN_nvrtcGetCUBINSize cubin_size;
    PFN_nvrtcGetCUBIN cubin;
    PFN_nvrtcDestroyProgram destroy;
    PFN_nvrtcAddNameExpression add_name;
    PFN_nvrtcGetLoweredName lowered;
    PFN_nvrtcGetErrorString err_str;
    PFN_nvrtcVersion version;  // optional
} g_nv;

static bool load_nvrtc() {
    if (g_nv.tried) return g_nv.ok;
    g_nv.tried = true;
    std::vector<std::string> cands;
    if (!g_nvrtc_path.empty()) cands.push_back(g_nvrtc_path);
    if (const char* e = getenv("TRTC_NVRTC_PATH")) cands.push_back(e);
    cands.push_back("libnvrtc.so.12");
    cands.push_back("libnvrtc.so");
    cands.push_back("/usr/local/cuda/lib64/libnvrtc.so.12");
    cands.push_back("/usr/local/cuda/lib64/libnvrtc.so");
    void* h = nullptr;
    for (auto& c : cands)
        if ((h = dlopen(c.c_str(), RTLD_NOW | RTLD_LOCAL))) break;
    if (!h) { set_error("NVRTC library not found (set TRTC_NVRTC_PATH)"); return false; }
#define TRTC_SYM(field, name) g_nv.field = (decltype(g_nv.field))dlsym(h, name)
    TRTC_SYM(create, "nvrtcCreateProgram");
    TRTC_SYM(compile, "nvrtcCompileProgram");
    TRTC_SYM(log_size, "nvrtcGetProgramLogSize");
    TRTC_SYM(log, "nvrtcGetProgramLog");
    TRTC_SYM(cubin_size, "nvrtcGetCUBINSize");
    TRTC_SYM(cubin, "nvrtcGetCUBIN");
    TRTC_SYM(destroy, "nvrtcDestroyProgram");
    TRTC_SYM(add_name, "nvrtcAddNameExpression");
    TRTC_SYM(lowered, "nvrtcGetLoweredName");
    TRTC_SYM(err_str, "nvrtcGetErrorString");
    TRTC_SYM(version, "nvrtcVersion");
#undef TRTC_SYM
    g_nv.ok = g_nv.create && g_nv.compile && g_nv.cubin && g_nv.add_name && g_nv.lowered;
    if (!g_nv.ok) set_error("NVRTC library lacks required entry points");
    return g_nv.ok;
}

typedef CUresult (*PFN_cuModuleLoadData_t)(CUmodule*, const void*);
typedef CUresult (*PFN_cuModuleGetFunction_t)(CUfunction*, CUmodule, const char*);
typedef CUresult (*PFN_cuModuleGetGlobal_t)(CUdeviceptr*, size_t*, CUmodule, const char*);
typedef CUresult (*PFN_cuLaunchKernel_t)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                                          unsigned, CUstream, void**, void**);
typedef CUresult (*PFN_cuFuncSetAttribute_t)(CUfunction, CUfunction_attribute, int);
typedef CUresult (*PFN_cuOccupancyMaxPotentialBlockSize_t)(int*, int*, CUfunction, CUoccupancyB2DSize, size_t, int);

static struct Drv {
    bool tried = false, ok = false;
    PFN_cuModuleLoadData_t load;
    PFN_cuModuleGetFunction_t get_function;
    PFN_cuModuleGetGlobal_t get_global;
    PFN_cuLaunchKernel_t launch;
    PFN_cuFuncSetAttribute_t set_attr;
    PFN_cuOccupancyMaxPotentialBlockSize_t occupancy;
} g_drv;

static bool load_driver() {
    if (g_drv.tried) return g_drv.ok;
    g_drv.tried = true;
    if (!ensure_device()) return false;
    cudaFree(0);  // the primary context becomes current for driver calls
    auto get = [](const char* name, void** fp) {
        cudaDriverEntryPointQueryResult q;
        return cudaGetDriverEntryPoint(name, fp, cudaEnableDefault, &q) == cudaSuccess &&
               q == cudaDriverEntryPointSuccess && *fp;
    };
    g_drv.ok = get("cuModuleLoadData", (void**)&g_drv.load) && get("cuModuleGetFunction", (void**)&g_drv.get_function) &&
               get("cuModuleGetGlobal", (void**)&g_drv.get_global) && get("cuLaunchKernel", (void**)&g_drv.launch) &&
               get("cuFuncSetAttribute", (void**)&g_drv.set_attr) &&
               get("cuOccupancyMaxPotentialBlockSize", (void**)&g_drv.occupancy);
    if (!g_drv.ok) set_error("CUDA driver entry points unavailable");
    return g_drv.ok;
}

int jit_ptx_arch() {
    if (!ensure_device()) return -1;
    int dev = 0, ma = 0, mi = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&ma, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&mi, cudaDevAttrComputeCapabilityMinor, dev);
    return ma * 10 + mi;
}

static std::string arch_option() {
    const int a = jit_ptx_arch();
    char buf[48];
    // architecture-specific features (sm_90a, sm_100a) where the GPU has them
    snprintf(buf, sizeof(buf), "--gpu-architecture=sm_%d%s", a, a >= 90 ? "a" : "");
    return buf;
}

static const char* k_stub_headers[][2] = {
    {"cstdint", "#pragma once\n"},
    {"stdint.h", "#pragma once\n"},
    {"cfloat",
     "#pragma once\n#define FLT_MAX 3.402823466e+38F\n#define FLT_MIN 1.175494351e-38F\n"
     "#define DBL_MAX 1.7976931348623158e+308\n#define DBL_MIN 2.2250738585072014e-308\n"},
    {"cuComplex.h", "#pragma once\n"},
    {"built_in.h", "#pragma once\n"},
};

static std::string compose_source(const std::vector<std::string>& headers, const std::string& extra) {
    std::string src = "#define TRTC_JIT 1\n#include \"trtc_builtins.cuh\"\n"
                      "typedef float2 cuFloatComplex;\ntypedef double2 cuDoubleComplex;\n";
    for (auto& c : g_code_blocks) src += c;
    src += g_struct_header;
    for (auto& h : headers) src += "#include \"" + h + "\"\n";
    src += extra;
    return src;
}

// ------------------------------------------------------------------ persistent cubin cache
// Compiled cubins persist across processes under cache_dir() (TRTC_CACHE_DIR, else
// ~/.cache/thrustrtc_b200), so a kernel string costs its NVRTC compilation once per machine,
// not once per process (the reference keeps such a cache in an unqlite file,
// internal/impl_context.inl:404-648).  An entry is three files named by a 128-bit hash of its
// key: <id>.cubin, <id>.name (the kernel's lowered name) and <id>.key, the key itself.  The
// key holds everything the cubin depends on -- the cache format, a digest of the device
// headers embedded in this library and of the headers the caller added, NVRTC's version, the
// architecture, the kernel's name expression and the full source -- and an entry is used only
// when its stored key equals the key exactly, so neither a hash collision nor an entry written
// by another build of the library is ever loaded.  The key file is written last, each file by
// a rename, so a reader sees a complete entry or none.  TRTC_JIT_DISK_CACHE=0 turns the cache
// off; so do include directories (jit_add_include_dir), whose files the key does not track.
static std::string cache_dir() {
    const char* e = getenv("TRTC_CACHE_DIR");
    std::string d;
    if (e && *e) d = e;
    else {
        const char* home = getenv("HOME");
        d = std::string(home ? home : "/tmp") + "/.cache/thrustrtc_b200";
    }
    return d;
}

static std::atomic<unsigned long long> g_cache_compiles{0}, g_cache_disk_hits{0}, g_cache_mem_hits{0};

void jit_cache_stats(unsigned long long out[3]) {
    out[0] = g_cache_compiles.load();
    out[1] = g_cache_disk_hits.load();
    out[2] = g_cache_mem_hits.load();
}

static bool disk_cache_on() {
    const char* e = getenv("TRTC_JIT_DISK_CACHE");
    if (e && e[0] == '0' && e[1] == 0) return false;
    return g_include_dirs.empty();
}

static std::string hex64(unsigned long long v) {
    char b[20];
    snprintf(b, sizeof(b), "%016llx", v);
    return b;
}

// digest of the device headers embedded in the library (fixed for a build)
static const std::string& embedded_headers_digest() {
    static std::string d;
    if (d.empty()) {
        unsigned long long h = fnv1a("trtc embedded headers");
        for (int i = 0; i < g_num_device_headers; i++) {
            h = fnv1a(g_device_header_names[i], h);
            h = fnv1a(std::string("\n") + g_device_header_sources[i], h);
        }
        d = hex64(h);
    }
    return d;
}

// digest of the headers added by jit_add_built_in_header (they replace or add to the stubs)
static std::string user_headers_digest() {
    unsigned long long h = fnv1a("trtc user headers");
    for (auto& u : g_user_headers) {
        h = fnv1a(u.first, h);
        h = fnv1a("\n" + u.second, h);
    }
    return hex64(h);
}

static std::string nvrtc_version_str() {
    int ma = 0, mi = 0;
    if (load_nvrtc() && g_nv.version && g_nv.version(&ma, &mi) == NVRTC_SUCCESS)
        return std::to_string(ma) + "." + std::to_string(mi);
    return "unknown";
}

static std::string cache_key(const std::string& src, const std::string& name_expr) {
    return "thrustrtc_b200 cubin cache 2\ndevice headers " + embedded_headers_digest() + "\nuser headers " +
           user_headers_digest() + "\nnvrtc " + nvrtc_version_str() + "\n" + arch_option() + "\nname " + name_expr +
           "\n" + src;
}

static bool read_file(const std::string& path, std::string& out) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    return true;
}

// writes `data` to `path` through a temporary file and a rename
static bool write_file_atomic(const std::string& path, const std::string& data) {
    const std::string tmp = path + ".tmp" + std::to_string((unsigned long long)getpid());
    {
        std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
        if (!f) return false;
        f.write(data.data(), (std::streamsize)data.size());
        f.close();
        if (!f) { remove(tmp.c_str()); return false; }
    }
    if (rename(tmp.c_str(), path.c_str()) != 0) { remove(tmp.c_str()); return false; }
    return true;
}

static void mkdirs(const std::string& p) {
    std::string cur;
    std::stringstream ss(p);
    std::string part;
    if (!p.empty() && p[0] == '/') cur = "/";
    while (std::getline(ss, part, '/')) {
        if (part.empty()) continue;
        cur += part + "/";
        mkdir(cur.c_str(), 0755);
    }
}

// compiles `src`, returns cubin and the lowered names of `name_exprs`
static bool nvrtc_compile(const std::string& src, const std::vector<std::string>& name_exprs, std::string& cubin,
                          std::vector<std::string>& lowered) {
    if (!load_nvrtc()) return false;
    std::vector<const char*> hn, hs;
    for (int i = 0; i < g_num_device_headers; i++) {
        hn.push_back(g_device_header_names[i]);
        hs.push_back(g_device_header_sources[i]);
    }
    for (auto& h : k_stub_headers) {
        bool user = false;
        for (auto& u : g_user_headers) user = user || u.first == h[0];
        if (!user) { hn.push_back(h[0]); hs.push_back(h[1]); }
    }
    for (auto& u : g_user_headers) { hn.push_back(u.first.c_str()); hs.push_back(u.second.c_str()); }
    nvrtcProgram prog;
    nvrtcResult r = g_nv.create(&prog, src.c_str(), "trtc_jit.cu", (int)hn.size(), hs.data(), hn.data());
    if (r != NVRTC_SUCCESS) { set_error("nvrtcCreateProgram failed"); return false; }
    for (auto& ne : name_exprs) g_nv.add_name(prog, ne.c_str());
    std::vector<std::string> opts = {arch_option(), "-std=c++17", "-default-device"};
    for (auto& d : g_include_dirs) opts.push_back("-I" + d);
    std::vector<const char*> o;
    for (auto& s : opts) o.push_back(s.c_str());
    r = g_nv.compile(prog, (int)o.size(), o.data());
    if (r != NVRTC_SUCCESS || g_verbose) {
        size_t ls = 0;
        g_nv.log_size(prog, &ls);
        std::string log(ls, '\0');
        if (ls) g_nv.log(prog, &log[0]);
        if (r != NVRTC_SUCCESS || g_verbose) {
            fprintf(stderr, "[thrustrtc_b200] NVRTC %s:\n%s\n", r == NVRTC_SUCCESS ? "log" : "compile error", log.c_str());
            if (r != NVRTC_SUCCESS) {
                // number the source lines like the reference's verbose mode
                std::stringstream ss(src);
                std::string line;
                int ln = 1;
                if (g_verbose || g_kernel_debug)
                    while (std::getline(ss, line)) fprintf(stderr, "%d\t%s\n", ln++, line.c_str());
            }
        }
        if (r != NVRTC_SUCCESS) {
            g_nv.destroy(&prog);
            set_error("NVRTC compilation failed: " + log.substr(0, 2000));
            return false;
        }
    }
    size_t cs = 0;
    g_nv.cubin_size(prog, &cs);
    cubin.assign(cs, '\0');
    g_nv.cubin(prog, &cubin[0]);
    lowered.clear();
    for (auto& ne : name_exprs) {
        const char* ln = nullptr;
        if (g_nv.lowered(prog, ne.c_str(), &ln) != NVRTC_SUCCESS || !ln) {
            g_nv.destroy(&prog);
            set_error("NVRTC: no lowered name for " + ne);
            return false;
        }
        lowered.push_back(ln);
    }
    g_nv.destroy(&prog);
    return true;
}

// The cubin of `src` and, when `name_expr` is given, the lowered name of that kernel: from the
// disk cache when it holds an entry of exactly this key, else compiled by NVRTC and stored.
// `from_disk` (optional) tells the caller the cubin came from the cache; `read_disk` false skips
// the lookup (a cached cubin that the driver refused is compiled again and replaced).
static bool cubin_for(const std::string& src, const std::string& name_expr, std::string& cubin, std::string& lowered,
                      bool* from_disk = nullptr, bool read_disk = true) {
    const bool disk = disk_cache_on();
    if (from_disk) *from_disk = false;
    std::string key, base;
    if (disk) {
        key = cache_key(src, name_expr);
        base = cache_dir() + "/" + hex64(fnv1a(key)) + hex64(fnv1a(key, 0x84222325cbf29ce4ull));
        std::string stored;
        if (read_disk && read_file(base + ".key", stored) && stored == key && read_file(base + ".cubin", cubin) &&
            !cubin.empty() && (name_expr.empty() || (read_file(base + ".name", lowered) && !lowered.empty()))) {
            g_cache_disk_hits++;
            if (from_disk) *from_disk = true;
            return true;
        }
    }
    std::vector<std::string> names, low;
    if (!name_expr.empty()) names.push_back("&" + name_expr);
    if (!nvrtc_compile(src, names, cubin, low)) return false;
    g_cache_compiles++;
    lowered = name_expr.empty() ? std::string() : low[0];
    if (disk) {
        // a failed store only costs the next process a compilation
        mkdirs(cache_dir());
        if (write_file_atomic(base + ".cubin", cubin) && write_file_atomic(base + ".name", lowered))
            write_file_atomic(base + ".key", key);
    }
    return true;
}

struct CachedModule {
    CUmodule mod = nullptr;
    CUfunction fn = nullptr;
};
static std::unordered_map<std::string, CachedModule> g_kernels;

static bool upload_constants(CUmodule mod) {
    for (auto& c : g_constants) {
        CUdeviceptr p;
        size_t sz;
        if (g_drv.get_global(&p, &sz, mod, c.first.c_str()) == CUDA_SUCCESS)
            cudaMemcpy((void*)p, c.second.data(), c.second.size() < sz ? c.second.size() : sz, cudaMemcpyHostToDevice);
    }
    return true;
}

bool jit_get_kernel(const std::vector<std::string>& headers, const std::string& extra, const std::string& name_expr,
                    const std::string& c_name, JitFunction& out) {
    std::lock_guard<std::recursive_mutex> lk(g_jit_mu);
    if (!load_driver()) return false;
    const std::string src = compose_source(headers, extra);
    const std::string key = src + "\n//" + name_expr + "|" + c_name + "|" + arch_option() + "|" + user_headers_digest();
    auto it = g_kernels.find(key);
    if (it != g_kernels.end()) {
        g_cache_mem_hits++;
        out.func = it->second.fn;
        return true;
    }
    std::string cubin, lname;
    bool from_disk = false;
    if (!cubin_for(src, name_expr, cubin, lname, &from_disk)) return false;
    CachedModule m;
    CUresult cr = g_drv.load(&m.mod, cubin.data());
    if (cr != CUDA_SUCCESS && from_disk) {
        if (!cubin_for(src, name_expr, cubin, lname, nullptr, false)) return false;
        cr = g_drv.load(&m.mod, cubin.data());
    }
    if (cr != CUDA_SUCCESS) { set_error("cuModuleLoadData failed"); return false; }
    if (name_expr.empty()) lname = c_name;
    cr = g_drv.get_function(&m.fn, m.mod, lname.c_str());
    if (cr != CUDA_SUCCESS) { set_error("cuModuleGetFunction failed for " + lname); return false; }
    upload_constants(m.mod);
    g_kernels[key] = m;
    out.func = m.fn;
    return true;
}

bool jit_launch(const JitFunction& f, dim_type grid, dim_type block, unsigned smem, cudaStream_t s,
                const std::vector<ViewBuf>& params) {
    if (!load_driver()) return false;
    if (grid.x == 0 || grid.y == 0 || grid.z == 0) return true;
    std::vector<void*> args(params.size());
    for (size_t i = 0; i < params.size(); i++) args[i] = (void*)params[i].data();
    if (smem > 48 * 1024) g_drv.set_attr((CUfunction)f.func, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem);
    const CUresult r = g_drv.launch((CUfunction)f.func, grid.x, grid.y, grid.z, block.x, block.y, block.z, smem,
                                    (CUstream)s, args.data(), nullptr);
    if (r != CUDA_SUCCESS) {
        char b[64];
        snprintf(b, sizeof(b), "cuLaunchKernel failed (%d)", (int)r);
        set_error(b);
        return false;
    }
    count_launch();
    if (g_kernel_debug && !check_device_errors(s, "JIT kernel")) return false;
    return true;
}

int jit_block_size(const JitFunction& f, unsigned smem) {
    if (!load_driver()) return 256;
    int minGrid = 0, bs = 256;
    if (g_drv.occupancy(&minGrid, &bs, (CUfunction)f.func, nullptr, smem, 0) != CUDA_SUCCESS) return 256;
    return bs > 0 ? bs : 256;
}

// Evaluates constant expressions (sizeof, alignof, __builtin_offsetof) in device code:
// compiled into a __device__ array, read back through the module's global.
bool jit_probe_values(const std::vector<std::string>& exprs, std::vector<unsigned long long>& out) {
    std::lock_guard<std::recursive_mutex> lk(g_jit_mu);
    if (!load_driver()) return false;
    std::string extra = "extern \"C\" __global__ void __trtc_probe() {}\n"
                        "__device__ unsigned long long __trtc_probe_values[" + std::to_string(exprs.size()) + "] = {";
    for (size_t i = 0; i < exprs.size(); i++) extra += (i ? ", " : "") + std::string("(unsigned long long)(") + exprs[i] + ")";
    extra += "};\n";
    const std::string src = compose_source({}, extra);
    std::string cubin, unused;
    if (!cubin_for(src, std::string(), cubin, unused)) return false;
    CUmodule mod;
    if (g_drv.load(&mod, cubin.data()) != CUDA_SUCCESS) return false;
    CUdeviceptr p;
    size_t sz;
    if (g_drv.get_global(&p, &sz, mod, "__trtc_probe_values") != CUDA_SUCCESS) return false;
    out.assign(exprs.size(), 0);
    return cudaMemcpy(out.data(), (void*)p, exprs.size() * 8, cudaMemcpyDeviceToHost) == cudaSuccess;
}

static bool probe_layout(const std::string& type_name, Layout& out) {
    std::vector<unsigned long long> v;
    if (!jit_probe_values({"sizeof(" + type_name + ")", "alignof(" + type_name + ")"}, v)) return false;
    out.size = (size_t)v[0];
    out.align = (size_t)v[1];
    return out.size > 0;
}

}  // namespace trtc_host
