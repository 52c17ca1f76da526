// Run-time specialisation of kernels with NVRTC.
//
// A kernel whose hot loop indexes with run-time strides spends issue slots on address
// arithmetic that constants would fold into the loads' immediates. jit::kernel compiles such a
// kernel's source once per (context, options, entry point) with the strides as -D constants,
// for the device's own architecture (sm_XYa, real code: no PTX JIT at load), and caches the
// loaded function for the life of the process. NVRTC is opened with dlopen, the driver's module
// calls through the runtime's entry-point query, so the library neither links against them nor
// fails to load without them: jit::kernel then returns nullptr and the caller launches its
// ahead-of-time build of the same code. A failed compile or load is remembered and not retried;
// at most kMaxModules are built per process.
//
// The cache key holds the context's unique id (cuCtxGetId), so a cudaDeviceReset, which
// destroys the modules with the context, leads to a fresh compile rather than a stale handle.
// Loading a module is not a stream operation: callers pass build = false while their stream is
// being captured, and the ahead-of-time kernel runs until a call outside capture has built it.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>
#include <stdio.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "pct_internal.h"

namespace pct {
namespace jit {
namespace {

struct Nvrtc {
  bool ok = false;
  decltype(&nvrtcCreateProgram) create = nullptr;
  decltype(&nvrtcCompileProgram) compile = nullptr;
  decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
  decltype(&nvrtcGetCUBIN) cubin = nullptr;
  decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
  decltype(&nvrtcGetProgramLog) log = nullptr;
  decltype(&nvrtcDestroyProgram) destroy = nullptr;
};

struct Driver {
  bool ok = false;
  PFN_cuModuleLoadData_v2000 load = nullptr;
  PFN_cuModuleGetFunction_v2000 get = nullptr;
  PFN_cuLaunchKernel_v4000 launch = nullptr;
  PFN_cuCtxGetCurrent_v4000 ctx = nullptr;
  PFN_cuCtxGetId_v12000 ctx_id = nullptr;
};

const Nvrtc &nvrtc() {
  static Nvrtc n = [] {
    Nvrtc r;
    void *h = nullptr;
    for (const char *name : {"libnvrtc.so.12", "libnvrtc.so"})
      if ((h = dlopen(name, RTLD_NOW | RTLD_LOCAL)) != nullptr) break;
    if (!h) return r;
    r.create = reinterpret_cast<decltype(r.create)>(dlsym(h, "nvrtcCreateProgram"));
    r.compile = reinterpret_cast<decltype(r.compile)>(dlsym(h, "nvrtcCompileProgram"));
    r.cubin_size = reinterpret_cast<decltype(r.cubin_size)>(dlsym(h, "nvrtcGetCUBINSize"));
    r.cubin = reinterpret_cast<decltype(r.cubin)>(dlsym(h, "nvrtcGetCUBIN"));
    r.log_size = reinterpret_cast<decltype(r.log_size)>(dlsym(h, "nvrtcGetProgramLogSize"));
    r.log = reinterpret_cast<decltype(r.log)>(dlsym(h, "nvrtcGetProgramLog"));
    r.destroy = reinterpret_cast<decltype(r.destroy)>(dlsym(h, "nvrtcDestroyProgram"));
    r.ok = r.create && r.compile && r.cubin_size && r.cubin && r.log_size && r.log && r.destroy;
    return r;
  }();
  return n;
}

template <typename F>
bool entry(const char *name, int version, F *fn) {
  void *p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPointByVersion(name, &p, version, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !p)
    return false;
  *fn = reinterpret_cast<F>(p);
  return true;
}

const Driver &driver() {
  static Driver d = [] {
    Driver r;
    r.ok = entry("cuModuleLoadData", 2000, &r.load) && entry("cuModuleGetFunction", 2000, &r.get) &&
           entry("cuLaunchKernel", 4000, &r.launch) && entry("cuCtxGetCurrent", 4000, &r.ctx) &&
           entry("cuCtxGetId", 12000, &r.ctx_id);
    return r;
  }();
  return d;
}

// Compiled modules stay loaded for the life of their context; past this many (distinct
// geometries) new ones are not built and callers use their ahead-of-time kernels.
constexpr int kMaxModules = 64;

std::mutex g_mu;
std::map<std::string, CUfunction> g_cache;  // nullptr entries: failed, not retried
int g_modules = 0;

// Compiles `source` for the current device and returns the loaded `entry_name`, or nullptr.
CUfunction build(const char *source, const char *file_name, const std::vector<std::string> &options,
                 const char *entry_name) {
  const Nvrtc &n = nvrtc();
  const Driver &d = driver();
  int dev = 0, major = 0, minor = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev) != cudaSuccess)
    return nullptr;
  nvrtcProgram prog;
  if (n.create(&prog, source, file_name, 0, nullptr, nullptr) != NVRTC_SUCCESS) return nullptr;
  std::vector<std::string> opts = options;
  opts.push_back("--gpu-architecture=sm_" + std::to_string(major) + std::to_string(minor) + "a");
  opts.push_back("-std=c++17");
  std::vector<const char *> argv;
  for (const std::string &o : opts) argv.push_back(o.c_str());
  CUfunction fn = nullptr;
  if (n.compile(prog, (int)argv.size(), argv.data()) == NVRTC_SUCCESS) {
    size_t size = 0;
    if (n.cubin_size(prog, &size) == NVRTC_SUCCESS && size > 0) {
      std::vector<char> image(size);
      CUmodule mod = nullptr;
      if (n.cubin(prog, image.data()) == NVRTC_SUCCESS &&
          d.load(&mod, image.data()) == CUDA_SUCCESS && d.get(&fn, mod, entry_name) != CUDA_SUCCESS)
        fn = nullptr;  // the module stays loaded for the life of the context
    }
  } else {
    size_t ls = 0;
    if (n.log_size(prog, &ls) == NVRTC_SUCCESS && ls > 1) {
      std::string log(ls, '\0');
      if (n.log(prog, &log[0]) == NVRTC_SUCCESS)
        fprintf(stderr, "pct_b200: run-time compile of %s failed:\n%s\n", file_name, log.c_str());
    }
  }
  n.destroy(&prog);
  return fn;
}

}  // namespace

void *kernel(const char *source, const char *file_name, const std::vector<std::string> &options,
             const char *entry_name, bool build_allowed) {
  if (!nvrtc().ok || !driver().ok) return nullptr;
  CUcontext ctx = nullptr;  // the runtime's context, current once the caller has used the device
  unsigned long long ctx_id = 0;
  if (driver().ctx(&ctx) != CUDA_SUCCESS || !ctx || driver().ctx_id(ctx, &ctx_id) != CUDA_SUCCESS)
    return nullptr;
  std::string key = std::to_string(ctx_id) + '|' + file_name + '|' + entry_name;
  for (const std::string &o : options) key += '|' + o;
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_cache.find(key);
  if (it != g_cache.end()) return it->second;
  if (!build_allowed || g_modules >= kMaxModules) return nullptr;
  CUfunction fn = build(source, file_name, options, entry_name);
  g_cache[key] = fn;
  if (fn) ++g_modules;
  return fn;
}

cudaError_t launch(void *fn, unsigned grid, unsigned block, cudaStream_t stream, void **args) {
  if (!fn || !driver().ok) return cudaErrorInvalidDeviceFunction;
  const CUresult r = driver().launch(static_cast<CUfunction>(fn), grid, 1, 1, block, 1, 1, 0,
                                     stream, args, nullptr);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorLaunchFailure;
}

}  // namespace jit
}  // namespace pct
