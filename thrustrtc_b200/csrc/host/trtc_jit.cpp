// trtc_jit.cpp -- NVRTC engine, struct registry, layout reflection and JIT kernel cache.
#include "trtc_jit.h"
#include "trtc_runtime.h"

#include <cuda.h>
#include <dlfcn.h>
#include <nvrtc.h>
#include <sys/stat.h>

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
    const std::string key = src + "\n//" + name_expr + "|" + c_name + "|" + arch_option();
    auto it = g_kernels.find(key);
    if (it != g_kernels.end()) { out.func = it->second.fn; return true; }
    char hbuf[32];
    snprintf(hbuf, sizeof(hbuf), "%016llx", fnv1a(key));
    const std::string dir = cache_dir();
    const std::string cpath = dir + "/" + hbuf + ".cubin", npath = dir + "/" + hbuf + ".name";
    std::string cubin, lname;
    {
        std::ifstream fc(cpath, std::ios::binary), fn(npath);
        if (fc && fn) {
            cubin.assign(std::istreambuf_iterator<char>(fc), std::istreambuf_iterator<char>());
            std::getline(fn, lname);
        }
    }
    if (cubin.empty() || lname.empty()) {
        std::vector<std::string> lowered;
        std::vector<std::string> names;
        if (!name_expr.empty()) names.push_back("&" + name_expr);
        if (!nvrtc_compile(src, names, cubin, lowered)) return false;
        lname = name_expr.empty() ? c_name : lowered[0];
        mkdirs(dir);
        std::ofstream fc(cpath + ".tmp", std::ios::binary), fn(npath + ".tmp");
        if (fc && fn) {
            fc.write(cubin.data(), (std::streamsize)cubin.size());
            fn << lname << "\n";
            fc.close();
            fn.close();
            rename((cpath + ".tmp").c_str(), cpath.c_str());
            rename((npath + ".tmp").c_str(), npath.c_str());
        }
    }
    CachedModule m;
    CUresult cr = g_drv.load(&m.mod, cubin.data());
    if (cr != CUDA_SUCCESS) { set_error("cuModuleLoadData failed"); return false; }
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
    std::string cubin;
    std::vector<std::string> lowered;
    if (!nvrtc_compile(src, {}, cubin, lowered)) return false;
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
