// trtc_context.cpp -- context functions and the generic JIT launchers TRTC_Kernel / TRTC_For
// (TRTCContext.h:13-71).  A TRTC_Kernel is `extern "C" __global__ void saxpy(<view types>
// <param names>) { body }`; a TRTC_For runs `body` once per index of [begin, end) with the
// index named `name_iter` -- the same contract as the reference (TRTCContext.cpp:204-246,
// internal/impl_context.inl:554-898), compiled by NVRTC for the device's sm_XXa.
#include "thrustrtc_cpp.h"
#include "trtc_jit.h"
#include "trtc_runtime.h"

using namespace trtc_host;

void set_libnvrtc_path(const char* path) { jit_set_nvrtc_path(path ? path : ""); }
bool TRTC_Try_Init() { return ensure_device(); }
int TRTC_Get_PTX_Arch() { return jit_ptx_arch(); }
void TRTC_Set_Verbose(bool verbose) { jit_set_verbose(verbose); }
void TRTC_Set_Kernel_Debug(bool kernel_debug) { jit_set_kernel_debug(kernel_debug); }

size_t TRTC_Size_Of(const char* cls) {
    Layout l;
    return layout_of(cls, l) ? l.size : (size_t)(-1);
}

// Offsets of the named members: reflected by NVRTC for arbitrary structs.
bool TRTC_Query_Struct(const char* name_struct, const std::vector<const char*>& name_members, size_t* offsets) {
    Layout l;
    if (!layout_of(name_struct, l)) return false;
    if (name_members.empty()) { offsets[0] = 1; return true; }
    if (name_members.size() == 1) { offsets[0] = 0; offsets[1] = l.size; return true; }
    std::vector<std::string> exprs;
    for (auto m : name_members) exprs.push_back(std::string("__builtin_offsetof(") + name_struct + ", " + m + ")");
    exprs.push_back(std::string("sizeof(") + name_struct + ")");
    std::vector<unsigned long long> v;
    if (!jit_probe_values(exprs, v)) return false;
    for (size_t i = 0; i < v.size(); i++) offsets[i] = (size_t)v[i];
    return true;
}

void TRTC_Add_Include_Dir(const char* path) { jit_add_include_dir(path); }
void TRTC_Add_Built_In_Header(const char* name, const char* content) { jit_add_built_in_header(name, content); }
void TRTC_Add_Code_Block(const char* code) { jit_add_code_block(code); }
void TRTC_Add_Inlcude_Filename(const char* fn) { jit_add_code_block(std::string("#include \"") + fn + "\"\n"); }
void TRTC_Add_Constant_Object(const char* name, const DeviceViewable& obj) { jit_add_constant_object(name, obj); }
std::string TRTC_Add_Struct(const char* struct_body) { return jit_add_struct(struct_body); }

void TRTC_Wait() {
    if (ensure_device()) check_device_errors((cudaStream_t)0, "wait");
}

static std::string kernel_source(const std::vector<std::string>& names, const DeviceViewable** args,
                                 const std::string& prefix_params, const std::string& body) {
    std::string s = "extern \"C\" __global__ void saxpy(" + prefix_params;
    for (size_t i = 0; i < names.size(); i++) {
        if (i > 0 || !prefix_params.empty()) s += ", ";
        s += args[i]->name_view_cls() + " " + names[i];
    }
    s += ")\n{\n" + body + "\n}\n";
    return s;
}

TRTC_Kernel::TRTC_Kernel(const std::vector<const char*>& param_names, const char* code_body) {
    for (auto p : param_names) m_param_names.push_back(p);
    m_code_body = code_body;
}

static bool get_saxpy(const std::vector<std::string>& names, const DeviceViewable** args, const std::string& prefix,
                      const std::string& body, JitFunction& f) {
    return jit_get_kernel({}, kernel_source(names, args, prefix, body), "", "saxpy", f);
}

bool TRTC_Kernel::calc_optimal_block_size(const DeviceViewable** args, int& sizeBlock, unsigned sharedMemBytes) {
    JitFunction f;
    if (!get_saxpy(m_param_names, args, "", m_code_body, f)) return false;
    sizeBlock = jit_block_size(f, sharedMemBytes);
    return true;
}

bool TRTC_Kernel::calc_number_blocks(const DeviceViewable** args, int sizeBlock, int& numBlocks, unsigned sharedMemBytes) {
    JitFunction f;
    if (!get_saxpy(m_param_names, args, "", m_code_body, f)) return false;
    int per_sm = 2048 / (sizeBlock > 0 ? sizeBlock : 256);
    if (per_sm < 1) per_sm = 1;
    (void)sharedMemBytes;
    numBlocks = sm_count() * per_sm;
    return true;
}

bool TRTC_Kernel::launch(dim_type gridDim, dim_type blockDim, const DeviceViewable** args, unsigned sharedMemBytes) {
    JitFunction f;
    if (!get_saxpy(m_param_names, args, "", m_code_body, f)) return false;
    std::vector<ViewBuf> params;
    for (size_t i = 0; i < m_param_names.size(); i++) params.push_back(args[i]->view());
    return jit_launch(f, gridDim, blockDim, sharedMemBytes, (cudaStream_t)0, params);
}

TRTC_For::TRTC_For(const std::vector<const char*>& param_names, const char* name_iter, const char* code_body) {
    for (auto p : param_names) m_param_names.push_back(p);
    m_name_iter = name_iter;
    m_code_body = code_body;
}

bool TRTC_For::launch(size_t begin, size_t end, const DeviceViewable** args) {
    if (end <= begin) return true;
    const std::string body = "    size_t " + m_name_iter + " = threadIdx.x + (size_t)blockIdx.x * blockDim.x + _trtc_begin;\n"
                             "    if (" + m_name_iter + " >= _trtc_end) return;\n" + m_code_body;
    JitFunction f;
    if (!get_saxpy(m_param_names, args, "size_t _trtc_begin, size_t _trtc_end", body, f)) return false;
    std::vector<ViewBuf> params;
    ViewBuf b(8), e(8);
    memcpy(b.data(), &begin, 8);
    memcpy(e.data(), &end, 8);
    params.push_back(b);
    params.push_back(e);
    for (size_t i = 0; i < m_param_names.size(); i++) params.push_back(args[i]->view());
    const int bs = jit_block_size(f, 0);
    const size_t blocks = (end - begin + bs - 1) / bs;
    return jit_launch(f, dim_type{(unsigned)blocks, 1, 1}, dim_type{(unsigned)bs, 1, 1}, 0, (cudaStream_t)0, params);
}

bool TRTC_For::launch_n(size_t n, const DeviceViewable** args) { return launch(0, n, args); }
