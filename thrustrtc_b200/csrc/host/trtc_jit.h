// trtc_jit.h -- NVRTC path: user Functor / view structs slotted into the kernel templates.
//
// The reference compiles every kernel from strings at run time (TRTC_Kernel / TRTC_For,
// internal/impl_context.inl:554-898).  Here only the instantiations that involve user code
// or non-contiguous views are compiled at run time, by NVRTC for sm_100a, from the same
// device headers the nvcc-built kernels use (embedded in the library).  Kernels are cached
// in memory and on disk (keyed by a hash of the full source).
#pragma once
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "thrustrtc_cpp.h"

namespace trtc_host {

struct Layout {
    size_t size = 1;
    size_t align = 1;
};
size_t round_up(size_t x, size_t a);
// layout of a named device type: scalars, Pair<,>, registered view / functor structs, and
// (when a GPU is present) an NVRTC reflection probe for anything else
bool layout_of(const std::string& type_name, Layout& out);
void layout_register(const std::string& type_name, const Layout& l);

// incremental struct layout (members in declaration order, C++ alignment rules)
struct StructLayout {
    size_t size = 0, align = 1;
    std::vector<size_t> offsets;
    size_t add(const Layout& m) {
        const size_t off = round_up(size, m.align);
        offsets.push_back(off);
        size = off + m.size;
        if (m.align > align) align = m.align;
        return off;
    }
    Layout finish() const {
        Layout l;
        if (offsets.empty()) { l.size = 1; l.align = 1; return l; }
        l.align = align;
        l.size = round_up(size, align);
        return l;
    }
};

// context state shared with TRTC_Add_* (TRTCContext.h:18-39)
void jit_set_verbose(bool v);
void jit_set_kernel_debug(bool v);
bool jit_kernel_debug();
void jit_add_code_block(const std::string& code);
void jit_add_include_dir(const std::string& dir);
void jit_add_built_in_header(const std::string& name, const std::string& content);
void jit_add_constant_object(const std::string& name, const DeviceViewable& obj);
std::string jit_add_struct(const std::string& struct_body);  // returns the struct's name
void jit_set_nvrtc_path(const std::string& path);
int jit_ptx_arch();

struct JitFunction {
    void* func = nullptr;   // CUfunction
};

// Compiles (or fetches from cache) the translation unit made of the common prelude, the
// user code blocks and structs, `#include`s of `headers` and `extra`; returns the kernel
// whose NVRTC name expression is `name_expr` ("&trtc::kernel<...>" form is added here), or
// the extern "C" function named `c_name` when name_expr is empty.
bool jit_get_kernel(const std::vector<std::string>& headers, const std::string& extra, const std::string& name_expr,
                    const std::string& c_name, JitFunction& out);
// Launches with each parameter given as its raw bytes.
bool jit_launch(const JitFunction& f, dim_type grid, dim_type block, unsigned smem, cudaStream_t s,
                const std::vector<ViewBuf>& params);
// Maximal resident-CTA-friendly block size for a JIT kernel (occupancy API).
int jit_block_size(const JitFunction& f, unsigned smem);
// Device-side values of constant expressions (sizeof / alignof / __builtin_offsetof ...).
bool jit_probe_values(const std::vector<std::string>& exprs, std::vector<unsigned long long>& out);
// persistent cubin cache counters: NVRTC compilations, disk-cache hits, in-process hits
void jit_cache_stats(unsigned long long out[3]);

}  // namespace trtc_host
