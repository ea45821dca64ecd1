// Layout-specialized compilation of the fused substep kernel with NVRTC.
//
// The reference compiles every quantized field access into its own LLVM IR
// with the bit offsets and scales as constants (codegen_llvm_quant.cpp).
// Here the same happens at aq_sim_create: the kernel template of
// aq_kernels.cuh is compiled for sm_100a with the record layout given as a
// constexpr aq_layout, so that slot kinds, bit offsets, shifts and scales
// fold away.  libnvrtc is opened with dlopen and the driver API is reached
// through cudaGetDriverEntryPoint, so libaq.so carries no link-time
// dependency on either; if NVRTC is missing or compilation fails, the
// simulator falls back to the nvcc-built generic kernel (and reports so).
#include <cuda.h>
#include <dlfcn.h>
#include <nvrtc.h>
#include <stdio.h>
#include <string.h>

#include <stdlib.h>

#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "aq_common.cuh"
#include "aq_jit.h"

// Header sources embedded at build time (autoquantizer_b200/build.py).
#include "aq_jit_sources.inc"

namespace aq {

namespace {

struct Nvrtc {
  void* h = nullptr;
  nvrtcResult (*create)(nvrtcProgram*, const char*, const char*, int, const char* const*, const char* const*);
  nvrtcResult (*compile)(nvrtcProgram, int, const char* const*);
  nvrtcResult (*log_size)(nvrtcProgram, size_t*);
  nvrtcResult (*log)(nvrtcProgram, char*);
  nvrtcResult (*cubin_size)(nvrtcProgram, size_t*);
  nvrtcResult (*cubin)(nvrtcProgram, char*);
  nvrtcResult (*add_name)(nvrtcProgram, const char*);
  nvrtcResult (*lowered)(nvrtcProgram, const char*, const char**);
  nvrtcResult (*destroy)(nvrtcProgram*);
  bool ok = false;
};

struct Driver {
  CUresult (*load)(CUmodule*, const void*) = nullptr;
  CUresult (*getfn)(CUfunction*, CUmodule, const char*) = nullptr;
  CUresult (*launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                     void**, void**) = nullptr;
  CUresult (*setattr)(CUfunction, CUfunction_attribute, int) = nullptr;
  CUresult (*occ)(int*, CUfunction, int, size_t) = nullptr;
  bool ok = false;
};

std::mutex g_mu;
Nvrtc g_nv;
Driver g_dr;
bool g_init = false;
std::unordered_map<std::string, CUfunction> g_cache;

template <class F>
bool sym(void* h, const char* n, F& f) {
  f = reinterpret_cast<F>(dlsym(h, n));
  return f != nullptr;
}

template <class F>
bool drv(const char* n, F& f) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(n, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
    return false;
  f = reinterpret_cast<F>(p);
  return true;
}

void init_once() {
  if (g_init) return;
  g_init = true;
  const char* names[] = {"/usr/local/cuda/lib64/libnvrtc.so.12", "libnvrtc.so.12", "libnvrtc.so"};
  for (const char* n : names) {
    g_nv.h = dlopen(n, RTLD_NOW | RTLD_LOCAL);
    if (g_nv.h) break;
  }
  if (g_nv.h) {
    g_nv.ok = sym(g_nv.h, "nvrtcCreateProgram", g_nv.create) && sym(g_nv.h, "nvrtcCompileProgram", g_nv.compile) &&
              sym(g_nv.h, "nvrtcGetProgramLogSize", g_nv.log_size) && sym(g_nv.h, "nvrtcGetProgramLog", g_nv.log) &&
              sym(g_nv.h, "nvrtcGetCUBINSize", g_nv.cubin_size) && sym(g_nv.h, "nvrtcGetCUBIN", g_nv.cubin) &&
              sym(g_nv.h, "nvrtcAddNameExpression", g_nv.add_name) &&
              sym(g_nv.h, "nvrtcGetLoweredName", g_nv.lowered) && sym(g_nv.h, "nvrtcDestroyProgram", g_nv.destroy);
  }
  g_dr.ok = drv("cuModuleLoadData", g_dr.load) && drv("cuModuleGetFunction", g_dr.getfn) &&
            drv("cuLaunchKernel", g_dr.launch) && drv("cuFuncSetAttribute", g_dr.setattr) &&
            drv("cuOccupancyMaxActiveBlocksPerMultiprocessor", g_dr.occ);
}

void fmt_f32(std::string& s, float v) {
  char b[64];
  snprintf(b, sizeof b, "%af", (double)v);
  s += b;
}

void fmt_f64(std::string& s, double v) {
  char b[64];
  snprintf(b, sizeof b, "%a", v);
  s += b;
}

}  // namespace

std::string jit_layout_source(const aq_layout& L) {
  std::string s;
  char b[256];
  snprintf(b, sizeof b,
           "struct JitLayout {\n  static constexpr bool kRegRecord = %s;\n  static constexpr int kWords = %d;\n"
           "  static constexpr int kMinBlocks = %d;\n",
           jit_reg_record(L) ? "true" : "false", L.n_words, jit_reg_record(L) ? kJitRegRecordMinBlocks : kJitSlotMinBlocks);
  s += b;
  s += "  static __device__ __forceinline__ aq_layout get(const aq_layout&) {\n    return aq_layout{";
  snprintf(b, sizeof b, "%d, %d, %d, %d, %d, %d, {0, 0}, {", L.n_slots, L.n_words, L.total_bits, L.compute_f64,
           L.use_dithering, L.n_groups);
  s += b;
  for (int i = 0; i < AQ_MAX_SLOTS; ++i) {
    const aq_slot& S = L.slot[i];
    snprintf(b, sizeof b, "{%d, %d, %d, %d, %d, %d, %d, %d, ", S.kind, S.bits, S.is_signed, S.exp_bits, S.bit_offset,
             S.exp_offset, S.group, S.exp_first);
    s += b;
    fmt_f32(s, S.scale_f32);
    s += ", ";
    fmt_f32(s, S.inv_scale_f32);
    s += ", ";
    fmt_f32(s, S.offset_f32);
    s += ", 0.0f, ";
    fmt_f64(s, S.scale_f64);
    s += ", ";
    fmt_f64(s, S.inv_scale_f64);
    s += ", ";
    fmt_f64(s, S.offset_f64);
    s += ", 0.0}";
    s += i + 1 < AQ_MAX_SLOTS ? ",\n" : "";
  }
  s += "}};\n  }\n};\n";
  return s;
}

bool jit_available() {
  std::lock_guard<std::mutex> g(g_mu);
  init_once();
  return g_nv.ok && g_dr.ok;
}

void* jit_k_step(int D, bool HF, bool HM, bool f64, bool col, bool sparse, const aq_layout& L, std::string* err) {
  std::lock_guard<std::mutex> g(g_mu);
  init_once();
  if (!g_nv.ok || !g_dr.ok) {
    if (err) *err = g_nv.ok ? "driver entry points unavailable" : "libnvrtc not found";
    return nullptr;
  }
  char name[160];
  snprintf(name, sizeof name, "aq::k_step<%d, %s, %s, %s, aq::JitLayout, %s, %s>", D, HF ? "true" : "false",
           HM ? "true" : "false", f64 ? "double" : "float", col ? "true" : "false", sparse ? "true" : "false");
  std::string src = "#include \"aq_kernels.cuh\"\nnamespace aq {\n";
  src += jit_layout_source(L);
  src += "}\n";
  // AQ_JIT_SOURCE_DIR (environment, kernel development): compile from the
  // aq_kernels.cuh found in this folder (and the headers it includes from
  // there) instead of the copies embedded in the library at build time
  const char* sdir = getenv("AQ_JIT_SOURCE_DIR");
  const bool from_dir = sdir && *sdir;
  std::string key = std::string(name) + "\n" + src;
  if (const char* e = getenv("AQ_JIT_DEFINES")) key += std::string("\n") + e;
  if (from_dir) key += std::string("\n") + sdir;
  auto hit = g_cache.find(key);
  if (hit != g_cache.end()) return (void*)hit->second;

  nvrtcProgram prog;
  if (g_nv.create(&prog, src.c_str(), "aq_jit_step.cu", from_dir ? 0 : kAqJitHeaderCount,
                  from_dir ? nullptr : kAqJitHeaderSrc, from_dir ? nullptr : kAqJitHeaderName) != NVRTC_SUCCESS) {
    if (err) *err = "nvrtcCreateProgram failed";
    return nullptr;
  }
  g_nv.add_name(prog, name);
  // AQ_JIT_DEFINES (environment): extra -D options, e.g.
  // "AQ_STEP_MIN_BLOCKS(R,LA)=4", separated by spaces (tuning experiments)
  std::vector<std::string> extra;
  if (const char* e = getenv("AQ_JIT_DEFINES")) {
    std::string s(e), tok;
    for (size_t i = 0; i <= s.size(); ++i) {
      if (i == s.size() || s[i] == ' ') {
        if (!tok.empty()) extra.push_back("-D" + tok);
        tok.clear();
      } else {
        tok += s[i];
      }
    }
  }
  if (from_dir) extra.push_back(std::string("-I") + sdir);
  extra.push_back("-DAQ_CH=" + std::to_string(AQ_CH));  // the launch's CTA size
  std::vector<const char*> opts = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo", "-DAQ_JIT=1"};
  for (const std::string& x : extra) opts.push_back(x.c_str());
  const nvrtcResult rc = g_nv.compile(prog, (int)opts.size(), opts.data());
  if (rc != NVRTC_SUCCESS) {
    size_t n = 0;
    g_nv.log_size(prog, &n);
    std::string log(n, '\0');
    if (n) g_nv.log(prog, &log[0]);
    if (err) *err = "nvrtc: " + log.substr(0, 2000);
    g_nv.destroy(&prog);
    return nullptr;
  }
  size_t cn = 0;
  g_nv.cubin_size(prog, &cn);
  std::string cubin(cn, '\0');
  g_nv.cubin(prog, &cubin[0]);
  const char* lowered = nullptr;
  g_nv.lowered(prog, name, &lowered);
  std::string lname = lowered ? lowered : "";
  g_nv.destroy(&prog);
  CUmodule mod;
  CUfunction fn;
  if (g_dr.load(&mod, cubin.data()) != CUDA_SUCCESS || g_dr.getfn(&fn, mod, lname.c_str()) != CUDA_SUCCESS) {
    if (err) *err = "cuModuleLoadData/cuModuleGetFunction failed";
    return nullptr;
  }
  g_cache[key] = fn;
  return (void*)fn;
}

int jit_set_smem(void* fn, int bytes) {
  return g_dr.setattr((CUfunction)fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, bytes) == CUDA_SUCCESS
             ? AQ_OK
             : AQ_E_CUDA;
}

int jit_occupancy(void* fn, int block, size_t smem, int* out) {
  return g_dr.occ(out, (CUfunction)fn, block, smem) == CUDA_SUCCESS ? AQ_OK : AQ_E_CUDA;
}

int jit_launch(void* fn, unsigned grid, unsigned block, size_t smem, cudaStream_t st, void** args) {
  return g_dr.launch((CUfunction)fn, grid, 1, 1, block, 1, 1, (unsigned)smem, (CUstream)st, args, nullptr) ==
                 CUDA_SUCCESS
             ? AQ_OK
             : AQ_E_CUDA;
}

}  // namespace aq
