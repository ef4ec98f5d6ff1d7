// jit.cu — the deferred volume / expression kernel with the AdditionalCompute expressions compiled
// to straight-line device code at run time (NVRTC), in place of the bytecode interpreter.
//
// The reference walks each expression's tree per particle and step (TrajectoryIntegrator.hpp:
// 539-627); the engine compiles it to postfix bytecode (expr.cpp).  Here the bytecode of a run's
// expressions becomes one C++ function: every operand is a named float, every operation the
// interpreter's operation in the same order (a op b with the same operands, the same library
// calls), compiled with --fmad=false like the rest of the device code, so the values are the
// interpreter's.  The kernel around it is deferred_extras (granite_kernels.cuh), compiled from the
// package's own headers.  libnvrtc is opened at run time; where it or the headers are missing, or
// the compile fails, the caller keeps the interpreter (GR_JIT=0 forces that).
#include <dlfcn.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <utility>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <nvrtc.h>

#include "expr.h"
#include "jit.h"

namespace granite_b200 {

namespace {

struct Nvrtc {
    bool ok = false;
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
    std::string why;
};

Nvrtc load_nvrtc() {
    Nvrtc n;
    void *h = nullptr;
    for (const char *name : {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"}) {
        h = dlopen(name, RTLD_NOW | RTLD_LOCAL);
        if (h) break;
    }
    if (!h) {
        n.why = "libnvrtc not found";
        return n;
    }
    n.create = reinterpret_cast<decltype(n.create)>(dlsym(h, "nvrtcCreateProgram"));
    n.compile = reinterpret_cast<decltype(n.compile)>(dlsym(h, "nvrtcCompileProgram"));
    n.log_size = reinterpret_cast<decltype(n.log_size)>(dlsym(h, "nvrtcGetProgramLogSize"));
    n.log = reinterpret_cast<decltype(n.log)>(dlsym(h, "nvrtcGetProgramLog"));
    n.cubin_size = reinterpret_cast<decltype(n.cubin_size)>(dlsym(h, "nvrtcGetCUBINSize"));
    n.cubin = reinterpret_cast<decltype(n.cubin)>(dlsym(h, "nvrtcGetCUBIN"));
    n.destroy = reinterpret_cast<decltype(n.destroy)>(dlsym(h, "nvrtcDestroyProgram"));
    n.ok = n.create && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.destroy;
    if (!n.ok) n.why = "libnvrtc lacks an entry point";
    return n;
}

Nvrtc &nvrtc() {
    static Nvrtc n = load_nvrtc();
    return n;
}

// Directory of this library's sources (csrc next to libgranite_b200.so) and CUDA's headers.
std::string source_dir() {
    Dl_info info{};
    if (!dladdr(reinterpret_cast<const void *>(&source_dir), &info) || !info.dli_fname) return "";
    std::string p = info.dli_fname;
    const size_t slash = p.rfind('/');
    return (slash == std::string::npos ? std::string(".") : p.substr(0, slash)) + "/csrc";
}

std::string cuda_include_dir() {
    for (const char *env : {"CUDA_HOME", "CUDA_PATH"}) {
        const char *v = std::getenv(env);
        if (v && *v) return std::string(v) + "/include";
    }
    return "/usr/local/cuda/include";
}

bool readable(const std::string &path) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::fclose(f);
    return true;
}

std::string float_literal(float v) {
    unsigned u;
    std::memcpy(&u, &v, sizeof u);
    char buf[48];
    std::snprintf(buf, sizeof buf, "__int_as_float(0x%08x)", u);
    return buf;
}

// One expression as statements over named floats; the stack of the interpreter becomes the
// list of names (eval_program's operand order: s1 is the operand pushed first).
bool emit_expression(const Program &p, int e, std::string &out) {
    std::vector<std::string> st;
    int t = 0;
    auto fresh = [&](const std::string &rhs) {
        const std::string name = "e" + std::to_string(e) + "_" + std::to_string(t++);
        out += "        const float " + name + " = " + rhs + ";\n";
        st.push_back(name);
    };
    for (int k = 0; k < p.len; ++k) {
        const Instr in = p.code[k];
        if (in.op == OP_REF) {
            if (in.arg < 0 || in.arg >= REF_COUNT) return false;
            fresh("ref[" + std::to_string(in.arg) + "]");
            continue;
        }
        if (in.op == OP_CONST) {
            fresh(float_literal(in.value));
            continue;
        }
        const bool binary = in.op == OP_ADD || in.op == OP_SUB || in.op == OP_MUL || in.op == OP_DIV ||
                            in.op == OP_RSUB || in.op == OP_RDIV || in.op == OP_ATAN2 || in.op == OP_RATAN2;
        if (binary) {
            if (st.size() < 2) return false;
            const std::string s0 = st.back();
            st.pop_back();
            const std::string s1 = st.back();
            st.pop_back();
            switch (in.op) {
                case OP_ADD: fresh(s1 + " + " + s0); break;
                case OP_SUB: fresh(s1 + " - " + s0); break;
                case OP_MUL: fresh(s1 + " * " + s0); break;
                case OP_DIV: fresh(s1 + " / " + s0); break;
                case OP_RSUB: fresh(s0 + " - " + s1); break;
                case OP_RDIV: fresh(s0 + " / " + s1); break;
                case OP_ATAN2: fresh("atan2f(" + s1 + ", " + s0 + ")"); break;
                default: fresh("atan2f(" + s0 + ", " + s1 + ")"); break;
            }
            continue;
        }
        if (st.empty()) return false;
        const std::string s0 = st.back();
        st.pop_back();
        const char *fn = nullptr;
        switch (in.op) {
            case OP_SQRT: fn = "sqrtf"; break;
            case OP_EXP: fn = "expf"; break;
            case OP_LOG: fn = "logf"; break;
            case OP_SIN: fn = "sinf"; break;
            case OP_COS: fn = "cosf"; break;
            case OP_TAN: fn = "tanf"; break;
            case OP_ASIN: fn = "asinf"; break;
            case OP_ACOS: fn = "acosf"; break;
            case OP_ATAN: fn = "atanf"; break;
            default: fn = nullptr; break;   // the interpreter's default: the operand unchanged
        }
        fresh(fn ? std::string(fn) + "(" + s0 + ")" : s0);
    }
    out += "        return " + (st.empty() ? std::string("0.f") : st.back()) + ";\n";
    return true;
}

struct Cached {
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kernel = nullptr;
    std::string why;
};

std::mutex g_mu;
std::map<std::string, Cached> g_cache;

}  // namespace

std::string jit_source(const Program *progs, const JitOptions &o, int dim) {
    const int nexpr = o.nexpr;
    std::string src = "#define GR_JIT_OPTIONS 1\n";
    const std::pair<const char *, int> opts[] = {{"nvol", o.nvol}, {"nexpr", o.nexpr}, {"ncon", o.ncon},
                                                 {"volume_mode", o.volume_mode}, {"constants_mode", o.constants_mode},
                                                 {"curvature_mode", o.curvature_mode}, {"dyn_any", o.dyn_any}};
    for (const auto &kv : opts) src += "#define GR_JIT_" + std::string(kv.first) + " " + std::to_string(kv.second) + "\n";
    src += "#include \"granite_kernels.cuh\"\nnamespace granite_b200 {\nstruct JitCode {\n";
    src += "    __device__ __forceinline__ float eval(int e, const float (&ref)[19]) const {\n";
    for (int e = 0; e < nexpr; ++e) {
        src += "      if (e == " + std::to_string(e) + ") {\n";
        if (!emit_expression(progs[e], e, src)) return "";
        src += "      }\n";
    }
    src += "      return 0.f;\n    }\n};\n}  // namespace granite_b200\n";
    src += "extern \"C\" __global__ void __launch_bounds__(256, 3) gr_jit_deferred_extras(\n"
           "    const __grid_constant__ granite_b200::KParams P, int rec, int irec, int k_end, int all) {\n";
    src += "    granite_b200::deferred_extras<" + std::to_string(dim) +
           ">(P, granite_b200::JitCode{}, rec, irec, k_end, all);\n}\n";
    return src;
}

cudaKernel_t jit_deferred_kernel(const Program *progs, const JitOptions &o, int dim, std::string &why) {
    const char *env = std::getenv("GR_JIT");
    if (env && env[0] == '0') {
        why = "GR_JIT=0";
        return nullptr;
    }
    const std::string src = jit_source(progs, o, dim);
    if (src.empty()) {
        why = "expression code not translatable";
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_cache.find(src);
    if (it != g_cache.end()) {
        why = it->second.why;
        return it->second.kernel;
    }
    Cached &c = g_cache[src];
    Nvrtc &n = nvrtc();
    const std::string dir = source_dir(), cuda_inc = cuda_include_dir();
    if (!n.ok) {
        c.why = n.why;
    } else if (dir.empty() || !readable(dir + "/granite_kernels.cuh") || !readable(cuda_inc + "/cuda_fp16.h")) {
        c.why = "device headers not found";
    } else {
        nvrtcProgram prog = nullptr;
        if (n.create(&prog, src.c_str(), "gr_jit_extras.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
            c.why = "nvrtcCreateProgram failed";
        } else {
            const std::string inc1 = "-I" + dir, inc2 = "-I" + cuda_inc;
            const char *opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "--fmad=false", inc1.c_str(),
                                  inc2.c_str()};
            const nvrtcResult rc = n.compile(prog, 5, opts);
            if (rc != NVRTC_SUCCESS) {
                size_t ls = 0;
                n.log_size(prog, &ls);
                std::string log(ls, '\0');
                if (ls) n.log(prog, &log[0]);
                c.why = "nvrtc compile failed: " + log.substr(0, 400);
            } else {
                size_t size = 0;
                n.cubin_size(prog, &size);
                std::vector<char> cubin(size);
                n.cubin(prog, cubin.data());
                if (cudaLibraryLoadData(&c.lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) != cudaSuccess ||
                    cudaLibraryGetKernel(&c.kernel, c.lib, "gr_jit_deferred_extras") != cudaSuccess) {
                    cudaGetLastError();
                    c.kernel = nullptr;
                    c.why = "loading the compiled kernel failed";
                }
            }
            n.destroy(&prog);
        }
    }
    why = c.why;
    return c.kernel;
}

}  // namespace granite_b200
