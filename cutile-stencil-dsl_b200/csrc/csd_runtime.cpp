// libcsd: host runtime of the B200 stencil backend.
//
// * JIT: NVRTC compiles a generated stencil module for sm_100a; cubins are
//   cached on disk by a hash of source + headers + options + NVRTC version.
// * Loading/launching through the CUDA driver API, which is resolved with
//   dlopen("libcuda.so.1") so the library itself loads on machines without a
//   GPU driver (CPU-only tests check the exported symbols).
// * TMA descriptors are encoded per launch with cuTensorMapEncodeTiled.
//
// No per-launch allocation: the only device memory this file allocates is
// one 4-byte error word per device, on first use.
#include <dlfcn.h>
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/csd.h"

// ---------------------------------------------------------------------------
// Minimal driver API surface (types from the CUDA driver API documentation)
// ---------------------------------------------------------------------------
typedef int CUresult;
typedef int CUdevice;
typedef struct CUctx_st* CUcontext;
typedef struct CUmod_st* CUmodule;
typedef struct CUfunc_st* CUfunction;
typedef struct CUstream_st* CUstream;
typedef unsigned long long CUdeviceptr;

enum {
  CU_FUNC_ATTRIBUTE_NUM_REGS_ = 4,
  CU_FUNC_ATTRIBUTE_LOCAL_SIZE_BYTES_ = 3,
  CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES_ = 8,
  CU_DEVICE_ATTRIBUTE_MULTIPROCESSOR_COUNT_ = 16,
};
enum {
  TMAP_FLOAT32 = 7,  // CU_TENSOR_MAP_DATA_TYPE_FLOAT32
  TMAP_FLOAT64 = 8,  // CU_TENSOR_MAP_DATA_TYPE_FLOAT64
};

struct Driver {
  bool ok = false;
  std::string why;
  CUresult (*cuInit)(unsigned);
  CUresult (*cuDeviceGet)(CUdevice*, int);
  CUresult (*cuDeviceGetAttribute)(int*, int, CUdevice);
  CUresult (*cuCtxGetCurrent)(CUcontext*);
  CUresult (*cuCtxSetCurrent)(CUcontext);
  CUresult (*cuCtxGetDevice)(CUdevice*);
  CUresult (*cuDevicePrimaryCtxRetain)(CUcontext*, CUdevice);
  CUresult (*cuModuleLoadData)(CUmodule*, const void*);
  CUresult (*cuModuleUnload)(CUmodule);
  CUresult (*cuModuleGetFunction)(CUfunction*, CUmodule, const char*);
  CUresult (*cuModuleGetGlobal)(CUdeviceptr*, size_t*, CUmodule, const char*);
  CUresult (*cuMemcpyDtoH)(void*, CUdeviceptr, size_t);
  CUresult (*cuMemcpyHtoD)(CUdeviceptr, const void*, size_t);
  CUresult (*cuMemAlloc)(CUdeviceptr*, size_t);
  CUresult (*cuFuncSetAttribute)(CUfunction, int, int);
  CUresult (*cuFuncGetAttribute)(int*, int, CUfunction);
  CUresult (*cuOccupancyMaxActiveBlocksPerMultiprocessor)(int*, CUfunction, int, size_t);
  CUresult (*cuLaunchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                             unsigned, CUstream, void**, void**);
  CUresult (*cuTensorMapEncodeTiled)(void*, int, unsigned, void*, const unsigned long long*,
                                     const unsigned long long*, const unsigned*, const unsigned*,
                                     int, int, int, int);
  CUresult (*cuGetErrorString)(CUresult, const char**);
  CUresult (*cuCtxSynchronize)(void);
  CUresult (*cuCtxGetId)(CUcontext, unsigned long long*);  // optional (driver >= 12.0)
};

static thread_local std::string g_last_error;
static std::mutex g_mu;

static int fail(int code, const char* fmt, ...) {
  char buf[2048];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

static void load_driver(Driver& d);

static Driver& drv() {
  static Driver d;
  static std::once_flag once;
  std::call_once(once, [] { load_driver(d); });
  return d;
}

static void load_driver(Driver& d) {
  void* h = dlopen("libcuda.so.1", RTLD_NOW | RTLD_GLOBAL);
  if (!h) h = dlopen("libcuda.so", RTLD_NOW | RTLD_GLOBAL);
  if (!h) {
    d.why = "libcuda.so.1 not found (no NVIDIA driver)";
    return;
  }
#define CSD_SYM(field, name)                                                    \
  d.field = reinterpret_cast<decltype(d.field)>(dlsym(h, name));                \
  if (!d.field) {                                                               \
    d.why = std::string("driver symbol missing: ") + name;                      \
    return;                                                                     \
  }
  CSD_SYM(cuInit, "cuInit");
  CSD_SYM(cuDeviceGet, "cuDeviceGet");
  CSD_SYM(cuDeviceGetAttribute, "cuDeviceGetAttribute");
  CSD_SYM(cuCtxGetCurrent, "cuCtxGetCurrent");
  CSD_SYM(cuCtxSetCurrent, "cuCtxSetCurrent");
  CSD_SYM(cuCtxGetDevice, "cuCtxGetDevice");
  CSD_SYM(cuDevicePrimaryCtxRetain, "cuDevicePrimaryCtxRetain");
  CSD_SYM(cuModuleLoadData, "cuModuleLoadData");
  CSD_SYM(cuModuleUnload, "cuModuleUnload");
  CSD_SYM(cuModuleGetFunction, "cuModuleGetFunction");
  CSD_SYM(cuModuleGetGlobal, "cuModuleGetGlobal_v2");
  CSD_SYM(cuMemcpyDtoH, "cuMemcpyDtoH_v2");
  CSD_SYM(cuMemcpyHtoD, "cuMemcpyHtoD_v2");
  CSD_SYM(cuMemAlloc, "cuMemAlloc_v2");
  CSD_SYM(cuFuncSetAttribute, "cuFuncSetAttribute");
  CSD_SYM(cuFuncGetAttribute, "cuFuncGetAttribute");
  CSD_SYM(cuOccupancyMaxActiveBlocksPerMultiprocessor, "cuOccupancyMaxActiveBlocksPerMultiprocessor");
  CSD_SYM(cuLaunchKernel, "cuLaunchKernel");
  CSD_SYM(cuTensorMapEncodeTiled, "cuTensorMapEncodeTiled");
  CSD_SYM(cuGetErrorString, "cuGetErrorString");
  CSD_SYM(cuCtxSynchronize, "cuCtxSynchronize");
#undef CSD_SYM
  d.cuCtxGetId = reinterpret_cast<decltype(d.cuCtxGetId)>(dlsym(h, "cuCtxGetId"));
  if (d.cuInit(0) != 0) {
    d.why = "cuInit failed (no usable device)";
    return;
  }
  d.ok = true;
}

static int cu_fail(CUresult r, const char* what) {
  const char* s = "unknown";
  if (drv().cuGetErrorString) drv().cuGetErrorString(r, &s);
  return fail(CSD_ELAUNCH, "%s failed: CUDA error %d (%s)", what, r, s ? s : "?");
}

// Make sure a context is current (torch normally made the primary one current).
static int ensure_context(CUdevice* dev_out) {
  Driver& d = drv();
  if (!d.ok) return fail(CSD_ENODEV, "%s", d.why.c_str());
  CUcontext ctx = nullptr;
  d.cuCtxGetCurrent(&ctx);
  if (!ctx) {
    CUdevice dev;
    CUresult r = d.cuDeviceGet(&dev, 0);
    if (r) return cu_fail(r, "cuDeviceGet");
    r = d.cuDevicePrimaryCtxRetain(&ctx, dev);
    if (r) return cu_fail(r, "cuDevicePrimaryCtxRetain");
    r = d.cuCtxSetCurrent(ctx);
    if (r) return cu_fail(r, "cuCtxSetCurrent");
  }
  CUdevice dev;
  CUresult r = d.cuCtxGetDevice(&dev);
  if (r) return cu_fail(r, "cuCtxGetDevice");
  if (dev_out) *dev_out = dev;
  return CSD_OK;
}

// ---------------------------------------------------------------------------
// Per-device state: SM count and the error word
// ---------------------------------------------------------------------------
struct DeviceState {
  int sms = 0;
  CUdeviceptr err = 0;
};
static std::unordered_map<int, DeviceState> g_devices;

static int device_state(CUdevice dev, DeviceState** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceState& st = g_devices[dev];
  if (st.sms == 0) {
    CUresult r = drv().cuDeviceGetAttribute(&st.sms, CU_DEVICE_ATTRIBUTE_MULTIPROCESSOR_COUNT_, dev);
    if (r) return cu_fail(r, "cuDeviceGetAttribute");
  }
  if (st.err == 0) {
    CUresult r = drv().cuMemAlloc(&st.err, 16);
    if (r) return cu_fail(r, "cuMemAlloc(error word)");
    int zero[4] = {0, 0, 0, 0};
    r = drv().cuMemcpyHtoD(st.err, zero, sizeof(zero));
    if (r) return cu_fail(r, "cuMemcpyHtoD(error word)");
  }
  *out = &st;
  return CSD_OK;
}

// ---------------------------------------------------------------------------
// JIT compile with a disk cache
// ---------------------------------------------------------------------------
static unsigned long long fnv1a(const std::string& s, unsigned long long h = 1469598103934665603ull) {
  for (unsigned char c : s) {
    h ^= c;
    h *= 1099511628211ull;
  }
  return h;
}

static std::vector<std::string> split_opts(const char* options) {
  std::vector<std::string> v;
  if (!options) return v;
  std::string cur;
  for (const char* p = options; *p; ++p) {
    if (*p == '\n') {
      if (!cur.empty()) v.push_back(cur);
      cur.clear();
    } else {
      cur += *p;
    }
  }
  if (!cur.empty()) v.push_back(cur);
  return v;
}

static bool read_file(const std::string& path, std::string* out) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  std::stringstream ss;
  ss << f.rdbuf();
  *out = ss.str();
  return true;
}

// An ELF image (the only thing NVRTC's cubin output can be).
static bool cubin_ok(const std::string& b) {
  return b.size() >= 64 && (unsigned char)b[0] == 0x7f && b[1] == 'E' && b[2] == 'L' && b[3] == 'F';
}

// Integrity record of a cached cubin: its size and FNV-1a hash.
static std::string cubin_sum(const std::string& b) {
  char s[64];
  snprintf(s, sizeof(s), "%zu %016llx\n", b.size(), fnv1a(b));
  return s;
}

static int jit_compile(const char* src, int n_headers, const char* const* headers,
                       const char* const* header_names, const char* options, const char* cache_dir,
                       std::string* cubin, std::string* path_out, std::string* log_out) {
  if (!src) return fail(CSD_EINVAL, "null source");
  int major = 0, minor = 0;
  nvrtcVersion(&major, &minor);
  std::string key = src;
  for (int i = 0; i < n_headers; ++i) {
    key += "\n//header:";
    key += header_names[i];
    key += "\n";
    key += headers[i];
  }
  key += "\n//opts:";
  key += options ? options : "";
  key += "\n//nvrtc:" + std::to_string(major) + "." + std::to_string(minor);
  char hex[32];
  snprintf(hex, sizeof(hex), "%016llx", fnv1a(key));
  std::string path, sumpath;
  if (cache_dir && *cache_dir) {
    mkdir(cache_dir, 0755);
    path = std::string(cache_dir) + "/" + hex + ".cubin";
    sumpath = std::string(cache_dir) + "/" + hex + ".sum";
    std::string logpath = std::string(cache_dir) + "/" + hex + ".log";
    std::string sum;
    // A cache entry is used only when it is an ELF image whose size and
    // checksum match the record written with it; a truncated, overwritten or
    // half-written entry is compiled again and replaced.
    if (read_file(path, cubin) && read_file(sumpath, &sum) && cubin_ok(*cubin) &&
        sum == cubin_sum(*cubin)) {
      if (path_out) *path_out = path;
      if (log_out) read_file(logpath, log_out);
      return CSD_OK;
    }
    cubin->clear();
  }
  nvrtcProgram prog;
  nvrtcResult rr = nvrtcCreateProgram(&prog, src, "stencil.cu", n_headers, headers, header_names);
  if (rr != NVRTC_SUCCESS) return fail(CSD_ECOMPILE, "nvrtcCreateProgram: %s", nvrtcGetErrorString(rr));
  std::vector<std::string> opts = split_opts(options);
  std::vector<const char*> argv;
  for (auto& o : opts) argv.push_back(o.c_str());
  rr = nvrtcCompileProgram(prog, (int)argv.size(), argv.data());
  size_t log_size = 0;
  nvrtcGetProgramLogSize(prog, &log_size);
  std::string log(log_size, '\0');
  if (log_size) nvrtcGetProgramLog(prog, &log[0]);
  log.resize(strlen(log.c_str()));  // drop the terminating NUL
  if (log_out) *log_out = log;
  if (rr != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    return fail(CSD_ECOMPILE, "NVRTC compilation failed: %s\n%s", nvrtcGetErrorString(rr), log.c_str());
  }
  size_t n = 0;
  rr = nvrtcGetCUBINSize(prog, &n);
  if (rr != NVRTC_SUCCESS || n == 0) {
    nvrtcDestroyProgram(&prog);
    return fail(CSD_ECOMPILE, "nvrtcGetCUBINSize: %s (use a real sm_XXa architecture)",
                nvrtcGetErrorString(rr));
  }
  cubin->assign(n, '\0');
  nvrtcGetCUBIN(prog, &(*cubin)[0]);
  nvrtcDestroyProgram(&prog);
  if (!path.empty()) {
    std::string tmp = path + ".tmp" + std::to_string(getpid());
    {
      std::ofstream f(tmp, std::ios::binary);
      f.write(cubin->data(), (std::streamsize)cubin->size());
    }
    rename(tmp.c_str(), path.c_str());
    {
      std::string stmp = sumpath + ".tmp" + std::to_string(getpid());
      {
        std::ofstream f(stmp, std::ios::binary);
        f << cubin_sum(*cubin);
      }
      rename(stmp.c_str(), sumpath.c_str());
    }
    std::ofstream lf(std::string(cache_dir) + "/" + hex + ".log");
    lf << log;
    if (path_out) *path_out = path;
  }
  return CSD_OK;
}

// ---------------------------------------------------------------------------
// Modules and kernels
// ---------------------------------------------------------------------------
struct csd_module {
  CUmodule mod = nullptr;
  CUdevice dev = 0;
};

struct csd_kernel {
  csd_module* module = nullptr;
  CUfunction fn[2] = {nullptr, nullptr};  // [CSD_LOADER_TMA], [CSD_LOADER_LDG]
  csd_kernel_desc desc;
  int blocks_per_sm[2] = {0, 0};
  std::string name;
};

extern "C" {

int csd_internal_fail(int code, const char* msg) { return fail(code, "%s", msg); }

// Unique id of the calling thread's current CUDA context (0: none current, or
// the driver cannot say).  Lets callers notice that a device's context was
// destroyed and re-created (cudaDeviceReset) since they cached an address.
unsigned long long csd_internal_ctx_id(void) {
  Driver& d = drv();
  if (!d.ok || !d.cuCtxGetId) return 0;
  CUcontext c = nullptr;
  if (d.cuCtxGetCurrent(&c) != 0 || !c) return 0;
  unsigned long long id = 0;
  return d.cuCtxGetId(c, &id) == 0 ? id : 0;
}

int csd_version(void) { return 101; }

size_t csd_grid_size(void) { return sizeof(csd_grid); }

const char* csd_last_error(void) { return g_last_error.c_str(); }

int csd_compile(const char* src, int n_headers, const char* const* headers,
                const char* const* header_names, const char* options, const char* cache_dir,
                char* cubin_path, size_t path_len, char* log, size_t log_len) {
  std::string cubin, path, lg;
  int rc = jit_compile(src, n_headers, headers, header_names, options, cache_dir, &cubin, &path, &lg);
  if (cubin_path && path_len) {
    snprintf(cubin_path, path_len, "%s", path.c_str());
  }
  if (log && log_len) snprintf(log, log_len, "%s", lg.c_str());
  return rc;
}

int csd_module_load(const char* src, int n_headers, const char* const* headers,
                    const char* const* header_names, const char* options, const char* cache_dir,
                    csd_module** out) {
  if (!out) return fail(CSD_EINVAL, "null output handle");
  CUdevice dev;
  int rc = ensure_context(&dev);
  if (rc) return rc;
  std::string cubin, path, log;
  rc = jit_compile(src, n_headers, headers, header_names, options, cache_dir, &cubin, &path, &log);
  if (rc) return rc;
  CUmodule mod;
  CUresult r = drv().cuModuleLoadData(&mod, cubin.data());
  if (r) return cu_fail(r, "cuModuleLoadData");
  csd_module* m = new csd_module();
  m->mod = mod;
  m->dev = dev;
  *out = m;
  return CSD_OK;
}

int csd_module_load_image(const void* image, size_t size, csd_module** out) {
  if (!out || !image) return fail(CSD_EINVAL, "null argument");
  // an ELF cubin starts with 0x7f 'E' 'L' 'F'; anything else (PTX text, a
  // truncated file) is refused before the driver sees it
  const unsigned char* b = static_cast<const unsigned char*>(image);
  if (size < 64 || b[0] != 0x7f || b[1] != 'E' || b[2] != 'L' || b[3] != 'F')
    return fail(CSD_EINVAL, "not a cubin image (%zu bytes)", size);
  CUdevice dev;
  int rc = ensure_context(&dev);
  if (rc) return rc;
  CUmodule mod;
  CUresult r = drv().cuModuleLoadData(&mod, image);
  if (r) return cu_fail(r, "cuModuleLoadData");
  csd_module* m = new csd_module();
  m->mod = mod;
  m->dev = dev;
  *out = m;
  return CSD_OK;
}

int csd_module_unload(csd_module* m) {
  if (!m) return CSD_OK;
  if (m->mod && drv().ok) drv().cuModuleUnload(m->mod);
  delete m;
  return CSD_OK;
}

int csd_kernel_get(csd_module* m, const char* name, csd_kernel** out) {
  if (!m || !name || !out) return fail(CSD_EINVAL, "null argument");
  Driver& d = drv();
  csd_kernel* k = new csd_kernel();
  k->module = m;
  k->name = name;
  std::string n = name;
  CUresult r = d.cuModuleGetFunction(&k->fn[CSD_LOADER_TMA], m->mod, (n + "_tma").c_str());
  if (r) {
    delete k;
    return fail(CSD_ENOSYM, "kernel %s_tma not found in module", name);
  }
  r = d.cuModuleGetFunction(&k->fn[CSD_LOADER_LDG], m->mod, (n + "_ldg").c_str());
  if (r) {
    delete k;
    return fail(CSD_ENOSYM, "kernel %s_ldg not found in module", name);
  }
  CUdeviceptr dp;
  size_t sz;
  r = d.cuModuleGetGlobal(&dp, &sz, m->mod, (n + "_desc").c_str());
  if (r || sz != sizeof(csd_kernel_desc)) {
    delete k;
    return fail(CSD_ENOSYM, "descriptor %s_desc not found (size %zu)", name, (size_t)sz);
  }
  r = d.cuMemcpyDtoH(&k->desc, dp, sizeof(csd_kernel_desc));
  if (r) {
    delete k;
    return cu_fail(r, "cuMemcpyDtoH(desc)");
  }
  if (k->desc.magic != CSD_DESC_MAGIC) {
    delete k;
    return fail(CSD_ENOSYM, "bad descriptor magic for %s", name);
  }
  for (int l = 0; l < 2; ++l) {
    r = d.cuFuncSetAttribute(k->fn[l], CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES_,
                             k->desc.smem_bytes);
    if (r) {
      delete k;
      return cu_fail(r, "cuFuncSetAttribute(max dynamic smem)");
    }
    r = d.cuOccupancyMaxActiveBlocksPerMultiprocessor(&k->blocks_per_sm[l], k->fn[l],
                                                      k->desc.threads, (size_t)k->desc.smem_bytes);
    if (r) {
      delete k;
      return cu_fail(r, "cuOccupancyMaxActiveBlocksPerMultiprocessor");
    }
    if (k->blocks_per_sm[l] < 1) k->blocks_per_sm[l] = 1;
  }
  *out = k;
  return CSD_OK;
}

int csd_kernel_describe(const csd_kernel* k, csd_kernel_desc* out) {
  if (!k || !out) return fail(CSD_EINVAL, "null argument");
  *out = k->desc;
  return CSD_OK;
}

int csd_kernel_resources(csd_kernel* k, int* regs, int* local_bytes, int* blocks_per_sm) {
  if (!k) return fail(CSD_EINVAL, "null kernel");
  Driver& d = drv();
  if (regs) d.cuFuncGetAttribute(regs, CU_FUNC_ATTRIBUTE_NUM_REGS_, k->fn[CSD_LOADER_TMA]);
  if (local_bytes) d.cuFuncGetAttribute(local_bytes, CU_FUNC_ATTRIBUTE_LOCAL_SIZE_BYTES_, k->fn[CSD_LOADER_TMA]);
  if (blocks_per_sm) *blocks_per_sm = k->blocks_per_sm[CSD_LOADER_TMA];
  return CSD_OK;
}

// Map an N-D array (halo included) to the engine's (Z, Y, X) view.
static void view3(const csd_field& f, long long dims[3], const int halo_in[3], int halo[3]) {
  if (f.ndim == 3) {
    for (int i = 0; i < 3; ++i) {
      dims[i] = f.shape[i];
      halo[i] = halo_in[i];
    }
  } else if (f.ndim == 2) {
    dims[0] = f.shape[0];
    dims[1] = 1;
    dims[2] = f.shape[1];
    halo[0] = halo_in[0];
    halo[1] = 0;
    halo[2] = halo_in[1];
  } else {
    dims[0] = 1;
    dims[1] = 1;
    dims[2] = f.shape[0];
    halo[0] = 0;
    halo[1] = 0;
    halo[2] = halo_in[0];
  }
}

// Row-pitched layout: unit innermost stride, each outer stride spanning at
// least the dimension inside it (C-contiguous arrays are the tight case).
static bool row_pitched(const csd_field& f) {
  if (f.shape[f.ndim - 1] != 1 && f.strides[f.ndim - 1] != 1) return false;
  for (int i = f.ndim - 2; i >= 0; --i)
    if (f.shape[i] != 1 && f.strides[i] < f.strides[i + 1] * f.shape[i + 1]) return false;
  return true;
}

// Validate one grid's fields and fill its kernel-side descriptor.
// Cut a column of `nz` rows into about `cnt` items of a multiple of `rows`
// rows each; with `shift`, the first and last item are about 4 % shorter
// than the others (zs rows).  Returns the number of items, every one
// non-empty: item tz covers [tz*zc - zs, (tz+1)*zc - zs) clipped to [0, nz).
static long long split_column(long long nz, long long cnt, int rows, bool shift, int* zc,
                              int* zs) {
  if (cnt < 1) cnt = 1;
  long long s = shift && cnt >= 2 ? (nz / cnt) / 24 / rows * rows : 0;
  long long z = ((nz + 2 * s + cnt - 1) / cnt + rows - 1) / rows * rows;
  long long n = (nz + s + z - 1) / z;
  if (s > 0 && (z <= s || n < 2)) {
    s = 0;
    z = ((nz + cnt - 1) / cnt + rows - 1) / rows * rows;
    n = (nz + z - 1) / z;
  }
  *zc = (int)z;
  *zs = (int)s;
  return n;
}

int csd_plan_items(const csd_kernel_desc* D, long long slots, int zchunk_req, csd_grid* g) {
  if (!D || !g) return fail(CSD_EINVAL, "null argument");
  if (D->rows < 1 || g->tiles[0] < 1 || g->tiles[1] < 1 || g->interior[0] < 1)
    return fail(CSD_EINVAL, "empty work split");
  // Work items (column tiles x Z chunks) sized so that they fill the
  // resident CTAs in one wave: items of equal length that start together
  // keep neighbouring columns on the same planes (their halo rows are then
  // shared in L2) and leave no tail.
  const long long nz = g->interior[0];
  const int rows = D->rows;
  const long long columns = (long long)g->tiles[0] * g->tiles[1];
  int zchunk = zchunk_req > 0 ? zchunk_req : D->zchunk;
  const bool one_wave = zchunk_req <= 0 && D->zchunk == 0;
  if (zchunk <= 0) {
    // -W: W items per resident block (issue-bound bodies balance better)
    const long long waves = zchunk < 0 ? -(long long)zchunk : 1;
    const long long cols = columns > 0 ? columns : 1;
    long long nzc = slots * waves / cols;
    if (nzc < 1) nzc = 1;
    if (waves == 1) {
      // One wave only pays when it keeps most resident slots busy; when the
      // columns leave more than a fifth of them idle (or spill into a thin
      // second wave) about seven waves of shorter items balance instead
      // (measured on 512^3: bricked 7-point, 645 columns on 1184 slots,
      // 238 -> 292 GPts/s; the flat sweep, 1024 items on 1184 slots, keeps
      // its single wave, which beats every multi-wave split there)
      const long long n1 = cols * nzc;
      const long long used = ((n1 + slots - 1) / slots) * slots;
      if (n1 * 5 < used * 4) {
        nzc = (7 * slots + cols / 2) / cols;
        if (nzc < 1) nzc = 1;
      }
    }
    if (nzc > nz) nzc = nz;
    zchunk = (int)((nz + nzc - 1) / nzc);
  }
  g->zchunk = ((zchunk + rows - 1) / rows) * rows;
  if (g->zchunk > nz) g->zchunk = (int)(((nz + rows - 1) / rows) * rows);
  g->tiles[2] = (int)((nz + g->zchunk - 1) / g->zchunk);
  g->ecols = 0;
  g->zshift = g->zshift_e = 0;
  g->zchunk_e = g->zchunk;
  long long items = columns * g->tiles[2];
  // A fused boundary fill makes the X-edge columns and every column's first
  // and last item slower than the rest (their chunks are patched); in a
  // one-wave split the kernel lasts as long as its slowest item, so those
  // items are made shorter: the X-edge columns take ~1.25x as many items
  // from the wave's unused slots, and first/last items give up ~4 % of rows.
  if (D->bc_mode != CSD_BC_NONE && one_wave) {
    const long long spare = slots - items;
    int zc, zs;
    const long long n = split_column(nz, g->tiles[2], rows, true, &zc, &zs);
    g->tiles[2] = (int)n;
    g->zchunk = g->zchunk_e = zc;
    g->zshift = g->zshift_e = zs;
    items = columns * n;
    const long long ncol_e = 2ll * g->tiles[1];
    long long ne = n + (n + 3) / 4;
    if ((ne - n) * ncol_e > spare) ne = n + (spare > 0 ? spare / ncol_e : 0);
    if (ne > nz / rows) ne = nz / rows;
    if (g->tiles[0] >= 3 && ne > n) {
      ne = split_column(nz, ne, rows, true, &zc, &zs);
      if (ne > n) {
        g->ecols = 2;
        g->items_main = (int)((long long)(g->tiles[0] - 2) * g->tiles[1] * n);
        g->zchunk_e = zc;
        g->zshift_e = zs;
        items = g->items_main + ncol_e * ne;
      }
    }
  }
  if (items > 0x7fffffff) return fail(CSD_EINVAL, "too many work items");
  g->items = (int)items;
  return CSD_OK;
}

int csd_grid_item_place(const csd_grid* g, int item, int* tx, int* ty, int* z0, int* nrows) {
  if (!g || !tx || !ty || !z0 || !nrows) return fail(CSD_EINVAL, "null argument");
  if (item < 0 || item >= g->items) return fail(CSD_EINVAL, "item %d out of [0, %d)", item, g->items);
  csd_item_place(g, item, tx, ty, z0, nrows);
  return CSD_OK;
}

static int build_grid(csd_kernel* k, const csd_field* in, int n_in, const csd_field* out,
                      int n_out, const csd_launch_opts& o, DeviceState* st, int loader_req,
                      csd_grid* g, int* loader_out) {
  const csd_kernel_desc& D = k->desc;
  if (!in || (!out && n_out > 0)) return fail(CSD_EINVAL, "null field array");
  if (D.reduce_max && !o.red)
    return fail(CSD_EINVAL, "kernel %s max-reduces: opts.red must point to a device double",
                k->name.c_str());
  if (n_in != D.nin || n_out != D.nout)
    return fail(CSD_EINVAL, "kernel %s takes %d inputs and %d outputs, got %d and %d",
                k->name.c_str(), D.nin, D.nout, n_in, n_out);
  if (n_in > CSD_MAX_FIELDS || n_out > CSD_MAX_FIELDS) return fail(CSD_EINVAL, "too many fields");
  const csd_field& f0 = in[0];
  if (f0.ndim != D.ndim) return fail(CSD_EINVAL, "kernel is %d-D, array is %d-D", D.ndim, f0.ndim);
  const int want_dtype = D.dtype_bytes == 8 ? CSD_DTYPE_F64 : CSD_DTYPE_F32;
  for (int i = 0; i < n_in + n_out; ++i) {
    const csd_field& f = i < n_in ? in[i] : out[i - n_in];
    if (f.ndim != f0.ndim) return fail(CSD_EINVAL, "all fields must have the same ndim");
    for (int d = 0; d < f.ndim; ++d)
      if (f.shape[d] != f0.shape[d]) return fail(CSD_EINVAL, "all fields must have the same shape");
    if (f.dtype != want_dtype) return fail(CSD_EINVAL, "field dtype does not match the kernel");
    if (D.brick_shift == 0 && !row_pitched(f))
      return fail(CSD_EINVAL, "fields must be C-contiguous or row-pitched");
    for (int d = 0; d < f.ndim; ++d)
      if (f.shape[d] != 1 && f.strides[d] != f0.strides[d])
        return fail(CSD_EINVAL, "all fields of a grid must have the same strides");
    if (!f.ptr) return fail(CSD_EINVAL, "null field pointer");
    if ((reinterpret_cast<uintptr_t>(f.ptr) % D.dtype_bytes) != 0)
      return fail(CSD_EALIGN, "field pointer not aligned to its element size");
  }
  if (D.ndyn > 0 && !o.dyn) return fail(CSD_EINVAL, "kernel %s reads device scalars: opts.dyn is null",
                                        k->name.c_str());
  memset(g, 0, sizeof(*g));
  int halo[3];
  view3(f0, g->dims, o.halo, halo);
  g->ndim = f0.ndim;
  // per-step radius: chained steps see zero halos beyond the interior, so the
  // array needs only one step's halo
  const int rad[3] = {D.rz / D.temporal, D.ry / D.temporal, D.rx / D.temporal};
  for (int d = 0; d < 3; ++d) {
    g->halo[d] = halo[d];
    g->interior[d] = (int)(g->dims[d] - 2 * halo[d]);
    if (g->interior[d] <= 0 && g->dims[d] > 0)
      return fail(CSD_EINVAL, "array extent %lld leaves no interior with halo %d", g->dims[d], halo[d]);
    if (halo[d] < rad[d])
      return fail(CSD_EINVAL, "array halo %d is smaller than the stencil radius %d", halo[d], rad[d]);
  }
  if (f0.ndim == 3) {
    g->pitch_y = f0.shape[1] == 1 ? f0.shape[2] : f0.strides[1];
    g->pitch_z = f0.shape[0] == 1 ? f0.shape[1] * g->pitch_y : f0.strides[0];
  } else if (f0.ndim == 2) {
    g->pitch_y = f0.shape[0] == 1 ? f0.shape[1] : f0.strides[0];
    g->pitch_z = g->pitch_y;
  } else {
    g->pitch_y = g->dims[2];
    g->pitch_z = g->dims[2];
  }
  for (int i = 0; i < n_in; ++i) g->in[i] = in[i].ptr;
  for (int i = 0; i < n_out; ++i) g->out[i] = out[i].ptr;
  const long long esz = D.dtype_bytes;
  long long B = 1;
  if (D.brick_shift > 0) {
    // bricked fields: the shape is the logical (padded-array) shape; bricks
    // of B^ndim elements cover it rounded up to whole bricks
    B = 1ll << D.brick_shift;
    g->brick_shift = D.brick_shift;
    g->nbx = (int)((g->dims[2] + B - 1) / B);
    g->nby = f0.ndim == 3 ? (int)((g->dims[1] + B - 1) / B) : 1;
    if (o.loader == CSD_LOADER_TMA && !D.brick_tma)
      return fail(CSD_EINVAL, "this bricked kernel stages with the cp.async loader only");
  }
  // Loader: TMA when every input is 16-byte aligned with 16-byte pitches
  // (bricked fields: when the kernel's TMA entry stages bricks).
  bool tma_ok = D.brick_shift == 0 ? ((g->pitch_y * esz) % 16 == 0) && ((g->pitch_z * esz) % 16 == 0)
                                   : D.brick_tma != 0;
  for (int i = 0; i < n_in; ++i) tma_ok = tma_ok && (reinterpret_cast<uintptr_t>(in[i].ptr) % 16 == 0);
  int loader = loader_req;
  if (loader < 0 || loader > 1) loader = tma_ok ? CSD_LOADER_TMA : CSD_LOADER_LDG;
  if (loader == CSD_LOADER_TMA && !tma_ok)
    return fail(CSD_EALIGN, "TMA path needs 16-byte aligned fields and row pitch");
  const bool brick_tma = D.brick_shift > 0 && loader == CSD_LOADER_TMA;
  // Tile origins: X tiles start at the halo rounded down to 16 bytes (bricked
  // TMA staging: to a brick), Y tiles at the halo (bricked TMA staging: the
  // halo rounded down to the tile height, which divides the brick); rows
  // outside the interior are computed but never stored.  (The tile height
  // divides the brick or is a multiple of it, so every brick row a tile
  // covers starts a box.)
  g->xbase = brick_tma ? (int)((g->halo[2] / B) * B) : (g->halo[2] / D.align) * D.align;
  g->ybase = brick_tma ? (g->halo[1] / D.tile_y) * D.tile_y : g->halo[1];
  g->tiles[0] = (g->halo[2] + g->interior[2] - g->xbase + D.tile_x - 1) / D.tile_x;
  g->tiles[1] = (g->halo[1] + g->interior[1] - g->ybase + D.tile_y - 1) / D.tile_y;
  const long long slots = o.grid > 0 ? o.grid : (long long)k->blocks_per_sm[loader] * st->sms;
  int rc = csd_plan_items(&D, slots, o.zchunk, g);
  if (rc) return rc;
  g->bc_value = o.bc_value;
  for (int i = 0; i < CSD_MAX_SCALARS; ++i) g->scalars[i] = o.scalars[i];
  for (int i = 0; i < CSD_MAX_FIELDS; ++i) g->bc_odd[i] = o.bc_odd[i];
  g->dyn = o.dyn;
  g->red = o.red;
  bool vec = true;
  for (int i = 0; i < n_out; ++i) vec = vec && (reinterpret_cast<uintptr_t>(out[i].ptr) % 16 == 0);
  if (D.brick_shift == 0) vec = vec && ((g->pitch_y * esz) % 16 == 0) && ((g->pitch_z * esz) % 16 == 0);
  g->vec_store = vec ? 1 : 0;
  if (brick_tma) {
    // 5-D view of a bricked field: (x in brick, brick x, y in brick, z in
    // brick, brick y + nby * brick z); strides in bytes of dims 1-4.  The
    // tile map's box is the tile height, the row map's box one row; both
    // deliver whole-brick rows (box_w / B bricks) as flat rows.
    Driver& d = drv();
    const long long nbz = (g->dims[0] + B - 1) / B;
    const unsigned long long B3 = (unsigned long long)(B * B * B);
    for (int i = 0; i < n_in; ++i) {
      unsigned long long gdim[5] = {(unsigned long long)B, (unsigned long long)g->nbx,
                                    (unsigned long long)B, (unsigned long long)B,
                                    (unsigned long long)(g->nby * nbz)};
      unsigned long long gstride[4] = {B3 * esz, (unsigned long long)(B * esz),
                                       (unsigned long long)(B * B * esz),
                                       B3 * (unsigned long long)g->nbx * esz};
      unsigned estride[5] = {1, 1, 1, 1, 1};
      const unsigned rows = (unsigned)(D.tile_y < B ? D.tile_y : B);  // one brick row at most
      unsigned box[5] = {(unsigned)B, (unsigned)(D.box_w / B), rows, 1, 1};
      CUresult r = d.cuTensorMapEncodeTiled(&g->tmap[i], esz == 8 ? TMAP_FLOAT64 : TMAP_FLOAT32, 5,
                                            const_cast<void*>(in[i].ptr), gdim, gstride, box, estride,
                                            0, 0, 2, 0);
      if (r) return cu_fail(r, "cuTensorMapEncodeTiled(bricks)");
      box[2] = 1;
      r = d.cuTensorMapEncodeTiled(&g->tmap_wrap[i], esz == 8 ? TMAP_FLOAT64 : TMAP_FLOAT32, 5,
                                   const_cast<void*>(in[i].ptr), gdim, gstride, box, estride, 0, 0, 2,
                                   0);
      if (r) return cu_fail(r, "cuTensorMapEncodeTiled(brick rows)");
    }
  } else if (loader == CSD_LOADER_TMA) {
    Driver& d = drv();
    for (int i = 0; i < n_in; ++i) {
      unsigned long long gdim[3] = {(unsigned long long)g->dims[2], (unsigned long long)g->dims[1],
                                    (unsigned long long)g->dims[0]};
      unsigned long long gstride[2] = {(unsigned long long)(g->pitch_y * esz),
                                       (unsigned long long)(g->pitch_z * esz)};
      unsigned box[3] = {(unsigned)D.box_w, (unsigned)D.box_h, (unsigned)D.rows};
      unsigned estride[3] = {1, 1, 1};
      CUresult r = d.cuTensorMapEncodeTiled(&g->tmap[i], esz == 8 ? TMAP_FLOAT64 : TMAP_FLOAT32, 3,
                                            in[i].ptr, gdim, gstride, box, estride,
                                            0 /*interleave none*/, 0 /*swizzle none*/,
                                            2 /*L2 promotion 128B*/, 0 /*OOB fill zeros*/);
      if (r) return cu_fail(r, "cuTensorMapEncodeTiled");
    }
    const int rx1 = D.temporal > 0 ? D.rx / D.temporal : D.rx;
    if (D.bc_mode == CSD_BC_PERIODIC && rx1 > 0) {
      // narrow boxes for the periodic X wrap (engine.cuh: Cfg::WRAPW)
      const unsigned wrapw = (unsigned)(((rx1 + D.align - 1) / D.align) * D.align + D.align);
      for (int i = 0; i < n_in; ++i) {
        unsigned long long gdim[3] = {(unsigned long long)g->dims[2], (unsigned long long)g->dims[1],
                                      (unsigned long long)g->dims[0]};
        unsigned long long gstride[2] = {(unsigned long long)(g->pitch_y * esz),
                                         (unsigned long long)(g->pitch_z * esz)};
        unsigned box[3] = {wrapw, (unsigned)D.box_h, (unsigned)D.rows};
        unsigned estride[3] = {1, 1, 1};
        CUresult r = d.cuTensorMapEncodeTiled(&g->tmap_wrap[i],
                                              esz == 8 ? TMAP_FLOAT64 : TMAP_FLOAT32, 3, in[i].ptr,
                                              gdim, gstride, box, estride, 0, 0, 2, 0);
        if (r) return cu_fail(r, "cuTensorMapEncodeTiled(wrap)");
      }
    }
  }
  *loader_out = loader;
  return CSD_OK;
}

int csd_launch(csd_kernel* k, const csd_field* in, int n_in, const csd_field* out, int n_out,
               const csd_launch_opts* opts, void* stream) {
  if (!k) return fail(CSD_EINVAL, "null kernel");
  if (k->desc.reduce_max && !(opts && opts->red))
    return fail(CSD_EINVAL, "kernel %s max-reduces: opts.red must point to a device double",
                k->name.c_str());
  csd_launch_opts o;
  memset(&o, 0, sizeof(o));
  o.loader = -1;
  if (opts) o = *opts;
  CUdevice dev;
  int rc = ensure_context(&dev);
  if (rc) return rc;
  DeviceState* st;
  rc = device_state(dev, &st);
  if (rc) return rc;
  csd_params p;
  memset(&p, 0, sizeof(p));
  int loader = 0;
  rc = build_grid(k, in, n_in, out, n_out, o, st, o.loader, &p.g, &loader);
  if (rc) return rc;
  p.err = reinterpret_cast<int*>(st->err);
  p.timeout_ns = o.timeout_ns ? o.timeout_ns : 2000000000ull;
  p.withhold = o.withhold_chunk > 0 ? o.withhold_chunk : 0;
  int grid = o.grid > 0 ? o.grid : k->blocks_per_sm[loader] * st->sms;
  if (grid > p.g.items) grid = p.g.items;
  if (grid < 1) return CSD_OK;  // nothing to do
  void* args[] = {&p};
  CUresult r = drv().cuLaunchKernel(k->fn[loader], (unsigned)grid, 1, 1, (unsigned)k->desc.threads,
                                    1, 1, (unsigned)k->desc.smem_bytes,
                                    reinterpret_cast<CUstream>(stream), args, nullptr);
  if (r) return cu_fail(r, "cuLaunchKernel");
  return CSD_OK;
}

int csd_grid_build(csd_kernel* k, const csd_field* in, int n_in, const csd_field* out, int n_out,
                   const csd_launch_opts* opts, csd_grid* g, int* items, int* loader_used) {
  if (!k || !g) return fail(CSD_EINVAL, "null argument");
  csd_launch_opts o;
  memset(&o, 0, sizeof(o));
  if (opts) o = *opts;
  CUdevice dev;
  int rc = ensure_context(&dev);
  if (rc) return rc;
  DeviceState* st;
  rc = device_state(dev, &st);
  if (rc) return rc;
  int loader = 0;
  rc = build_grid(k, in, n_in, out, n_out, o, st, o.loader, g, &loader);
  if (rc) return rc;
  if (items) *items = g->items;
  if (loader_used) *loader_used = loader;
  return CSD_OK;
}

int csd_launch_batch(csd_kernel* k, const csd_grid* grids, const int* item_start, int ngrids,
                     int total_items, const csd_launch_opts* opts, void* stream) {
  if (!k || !grids || !item_start || ngrids < 1) return fail(CSD_EINVAL, "bad batch arguments");
  if (total_items < 1) return CSD_OK;
  if ((reinterpret_cast<uintptr_t>(grids) % 64) != 0)
    return fail(CSD_EALIGN, "grid descriptors must be 64-byte aligned in device memory");
  CUdevice dev;
  int rc = ensure_context(&dev);
  if (rc) return rc;
  DeviceState* st;
  rc = device_state(dev, &st);
  if (rc) return rc;
  csd_params p;
  memset(&p, 0, sizeof(p));
  p.grids = grids;
  p.item_start = item_start;
  p.grid_index = opts ? opts->grid_index : nullptr;
  p.ngrids = ngrids;
  p.total_items = total_items;
  p.err = reinterpret_cast<int*>(st->err);
  p.timeout_ns = (opts && opts->timeout_ns) ? opts->timeout_ns : 2000000000ull;
  p.withhold = (opts && opts->withhold_chunk > 0) ? opts->withhold_chunk : 0;
  const int loader = (opts && opts->loader == CSD_LOADER_LDG) ? CSD_LOADER_LDG : CSD_LOADER_TMA;
  int grid = (opts && opts->grid > 0) ? opts->grid : k->blocks_per_sm[loader] * st->sms;
  if (grid > total_items) grid = total_items;
  void* args[] = {&p};
  CUresult r = drv().cuLaunchKernel(k->fn[loader], (unsigned)grid, 1, 1,
                                    (unsigned)k->desc.threads, 1, 1, (unsigned)k->desc.smem_bytes,
                                    reinterpret_cast<CUstream>(stream), args, nullptr);
  if (r) return cu_fail(r, "cuLaunchKernel(batch)");
  return CSD_OK;
}

int csd_error_word(int* value, int reset) {
  CUdevice dev;
  int rc = ensure_context(&dev);
  if (rc) return rc;
  DeviceState* st;
  rc = device_state(dev, &st);
  if (rc) return rc;
  Driver& d = drv();
  CUresult r = d.cuCtxSynchronize();
  if (r) return cu_fail(r, "cuCtxSynchronize");
  int v = 0;
  r = d.cuMemcpyDtoH(&v, st->err, sizeof(int));
  if (r) return cu_fail(r, "cuMemcpyDtoH(error word)");
  if (value) *value = v;
  if (reset && v) {
    int zero = 0;
    r = d.cuMemcpyHtoD(st->err, &zero, sizeof(int));
    if (r) return cu_fail(r, "cuMemcpyHtoD(error word)");
  }
  if (v == CSD_ERR_TIMEOUT)
    return fail(CSD_ETIMEOUT, "a kernel gave up waiting for its input (device error word 0x%x)", v);
  if (v) return fail(CSD_ELAUNCH, "device error word 0x%x", v);
  return CSD_OK;
}

}  // extern "C"
