// Fixed (non-generated) kernels of libcsd: the standalone boundary fill.
//
// apply_boundary fills the halo of one array dimension by dimension, in
// order, like the reference's per-dimension slab copies
// (reference/stencil_ref.py:102-201, target_to_python.py:199-297), so corner
// cells end up with the composition of the per-dimension rules.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/csd.h"

extern "C" int csd_internal_fail(int code, const char* msg);
extern "C" unsigned long long csd_internal_ctx_id(void);

namespace {

// Source index along one dimension of a halo cell (the interior cell whose
// value it takes); interior indices map to themselves.
__device__ __forceinline__ long long fill_src(long long i, long long nd, int h, int bc) {
  if (i >= h && i < nd - h) return i;
  const bool high = i >= nd - h;
  const long long k = high ? i - (nd - h) : i;  // layer 0 .. h-1
  if (bc == CSD_BC_NEUMANN) return high ? nd - h - 1 : h;
  if (bc == CSD_BC_PERIODIC) return high ? h + k : nd - 2 * h + k;
  return high ? nd - h - 1 - k : 2 * h - 1 - k;  // reflecting
}

// Fill every halo cell of a (d0, d1, d2) array in one launch.  The halo is
// enumerated as three disjoint boxes (dim-0 halo layers over the whole
// cross-section; dim-1 layers over the dim-0 interior; dim-2 layers over
// the dim-0 and dim-1 interior), and each cell maps every out-of-interior
// dimension to its source independently.  That equals the dimension-by-
// dimension slab copies of the reference fill (corners take the value of
// the mirrored interior corner) for all four conditions.
template <typename T>
__global__ void fill_halo_kernel(T* u, long long d0, long long d1, long long d2, int h0, int h1,
                                 int h2, int bc, T value) {
  const long long i0 = d0 - 2LL * h0, i1 = d1 - 2LL * h1;
  const long long na = 2LL * h0 * d1 * d2;
  const long long nb = i0 * 2LL * h1 * d2;
  const long long nc = i0 * i1 * 2LL * h2;
  const long long total = na + nb + nc;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    long long a, b, c;
    if (e < na) {
      c = e % d2;
      long long t = e / d2;
      b = t % d1;
      const long long l = t / d1;  // 0 .. 2h0-1
      a = l < h0 ? l : d0 - 2LL * h0 + l;
    } else if (e < na + nb) {
      const long long f = e - na;
      c = f % d2;
      long long t = f / d2;
      const long long l = t % (2LL * h1);
      a = h0 + t / (2LL * h1);
      b = l < h1 ? l : d1 - 2LL * h1 + l;
    } else {
      const long long f = e - na - nb;
      const long long l = f % (2LL * h2);
      long long t = f / (2LL * h2);
      b = h1 + t % i1;
      a = h0 + t / i1;
      c = l < h2 ? l : d2 - 2LL * h2 + l;
    }
    const long long dst = (a * d1 + b) * d2 + c;
    if (bc == CSD_BC_DIRICHLET) {
      u[dst] = value;
    } else {
      const long long src =
          (fill_src(a, d0, h0, bc) * d1 + fill_src(b, d1, h1, bc)) * d2 + fill_src(c, d2, h2, bc);
      u[dst] = u[src];
    }
  }
}

template <typename T>
int apply_boundary_t(const csd_field* f, const int* halo, int bc, double value, cudaStream_t s) {
  long long n[3] = {1, 1, 1};
  int h3[3] = {0, 0, 0};
  const int off = 3 - f->ndim;
  for (int i = 0; i < f->ndim; ++i) {
    n[off + i] = f->shape[i];
    h3[off + i] = halo[i];
  }
  long long cells = 0, inner = 1;
  for (int d = 0; d < 3; ++d) {
    if (h3[d] < 0 || n[d] - 2LL * h3[d] < 1)
      return csd_internal_fail(CSD_EINVAL, "halo leaves no interior");
    if (h3[d] > 0 && bc != CSD_BC_DIRICHLET && n[d] - 2 * h3[d] < h3[d])
      return csd_internal_fail(CSD_EINVAL, "boundary fill needs an interior at least as wide as the halo");
    inner *= n[d] - 2LL * h3[d];
  }
  cells = n[0] * n[1] * n[2] - inner;
  if (cells == 0) return CSD_OK;
  long long blocks = (cells + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  fill_halo_kernel<T><<<(int)blocks, 256, 0, s>>>(reinterpret_cast<T*>(f->ptr), n[0], n[1], n[2],
                                                  h3[0], h3[1], h3[2], bc, (T)value);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return csd_internal_fail(CSD_ELAUNCH, cudaGetErrorString(e));
  return CSD_OK;
}

}  // namespace

// The fill and reduction kernels index packed (C-contiguous) arrays.
static bool packed(const csd_field* f) {
  long long expect = 1;
  for (int i = f->ndim - 1; i >= 0; --i) {
    if (f->shape[i] != 1 && f->strides[i] != expect) return false;
    expect *= f->shape[i];
  }
  return true;
}

extern "C" int csd_apply_boundary(const csd_field* f, const int* halo, int bc, double value,
                                  void* stream) {
  if (!f || !halo || !f->ptr) return csd_internal_fail(CSD_EINVAL, "null argument");
  if (f->ndim < 1 || f->ndim > 3) return csd_internal_fail(CSD_EINVAL, "ndim must be 1-3");
  if (!packed(f)) return csd_internal_fail(CSD_EINVAL, "boundary fill needs a C-contiguous field");
  if (bc < CSD_BC_DIRICHLET || bc > CSD_BC_REFLECTING)
    return csd_internal_fail(CSD_EINVAL, "unknown boundary condition");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (f->dtype == CSD_DTYPE_F64) return apply_boundary_t<double>(f, halo, bc, value, s);
  if (f->dtype == CSD_DTYPE_F32) return apply_boundary_t<float>(f, halo, bc, value, s);
  return csd_internal_fail(CSD_EINVAL, "unsupported dtype");
}

// ---------------------------------------------------------------------------
// Bricked layout conversions
//
// A bricked array holds a (n0, n1, n2) array (1-3 dims, leading dims 1) as
// bricks of B^nd elements, bricks in row-major order over the brick grid
// (ceil(n / B) per dim) and each brick row-major inside: the reference's
// to_bricks reshape/transpose (multigpu_emitter.py:370-408), padded cells
// zero.  One thread per element; to_bricks walks the bricked order (writes
// coalesced, reads in runs of B), from_bricks the flat order.
// ---------------------------------------------------------------------------
namespace {

__device__ __forceinline__ long long brick_off(long long z, long long y, long long x, int nd, int s,
                                               long long nby, long long nbx) {
  const long long m = (1ll << s) - 1;
  if (nd == 3)
    return ((((z >> s) * nby + (y >> s)) * nbx + (x >> s)) << (3 * s)) + ((z & m) << (2 * s)) +
           ((y & m) << s) + (x & m);
  if (nd == 2) return ((((y >> s) * nbx + (x >> s)) << (2 * s)) + ((y & m) << s) + (x & m));
  return x;
}

template <typename T>
__global__ void to_bricks_kernel(const T* __restrict__ flat, T* __restrict__ bricked, long long n0,
                                 long long n1, long long n2, int nd, int s, long long nb0,
                                 long long nb1, long long nb2) {
  const long long B = 1ll << s;
  const long long total = nb0 * nb1 * nb2 * (nd == 3 ? B * B * B : nd == 2 ? B * B : B);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    long long z = 0, y = 0, x;
    const long long m = B - 1;
    if (nd == 3) {
      const long long b = e >> (3 * s), r = e & ((1ll << (3 * s)) - 1);
      x = ((b % nb2) << s) + (r & m);
      y = (((b / nb2) % nb1) << s) + ((r >> s) & m);
      z = ((b / (nb2 * nb1)) << s) + (r >> (2 * s));
    } else if (nd == 2) {
      const long long b = e >> (2 * s), r = e & ((1ll << (2 * s)) - 1);
      x = ((b % nb2) << s) + (r & m);
      y = ((b / nb2) << s) + (r >> s);
    } else {
      x = e;
    }
    const bool in = z < n0 && y < n1 && x < n2;
    bricked[e] = in ? flat[(z * n1 + y) * n2 + x] : T(0);
  }
}

template <typename T>
__global__ void from_bricks_kernel(const T* __restrict__ bricked, T* __restrict__ flat, long long n0,
                                   long long n1, long long n2, int nd, int s, long long nb1,
                                   long long nb2) {
  const long long total = n0 * n1 * n2;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long x = e % n2, t = e / n2, y = t % n1, z = t / n1;
    flat[e] = bricked[brick_off(z, y, x, nd, s, nb1, nb2)];
  }
}

// (n0, n1, n2) view, bricked dimensionality and brick-grid extents of a field
int brick_geometry(const csd_field* f, int brick, long long n[3], long long nb[3], int* nd,
                   int* s) {
  if (!f || !f->ptr) return csd_internal_fail(CSD_EINVAL, "null field");
  if (f->ndim < 1 || f->ndim > 3) return csd_internal_fail(CSD_EINVAL, "ndim must be 1-3");
  if (brick < 2 || brick > 1024 || (brick & (brick - 1)))
    return csd_internal_fail(CSD_EINVAL, "brick size must be a power of two in [2, 1024]");
  if (!packed(f)) return csd_internal_fail(CSD_EINVAL, "the flat array must be C-contiguous");
  *nd = f->ndim;
  *s = 0;
  while ((1 << *s) < brick) ++*s;
  const int off = 3 - f->ndim;
  for (int i = 0; i < 3; ++i) n[i] = 1;
  for (int i = 0; i < f->ndim; ++i) n[off + i] = f->shape[i];
  for (int i = 0; i < 3; ++i) nb[i] = (i < off) ? 1 : (n[i] + brick - 1) / brick;
  return CSD_OK;
}

}  // namespace

extern "C" long long csd_bricked_elems(const long long* shape, int ndim, int brick) {
  if (!shape || ndim < 1 || ndim > 3 || brick < 1) return -1;
  long long e = 1;
  for (int i = 0; i < ndim; ++i) e *= ((shape[i] + brick - 1) / brick) * brick;
  return e;
}

extern "C" int csd_to_bricks(const csd_field* flat, int brick, void* bricked, void* stream) {
  long long n[3], nb[3];
  int nd = 0, s = 0;
  int rc = brick_geometry(flat, brick, n, nb, &nd, &s);
  if (rc) return rc;
  if (!bricked) return csd_internal_fail(CSD_EINVAL, "null bricked buffer");
  const long long total = nb[0] * nb[1] * nb[2] * (nd == 3 ? (long long)brick * brick * brick
                                                   : nd == 2 ? (long long)brick * brick : brick);
  long long blocks = (total + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (flat->dtype == CSD_DTYPE_F64)
    to_bricks_kernel<double><<<(int)blocks, 256, 0, st>>>(
        static_cast<const double*>(flat->ptr), static_cast<double*>(bricked), n[0], n[1], n[2], nd,
        s, nb[0], nb[1], nb[2]);
  else if (flat->dtype == CSD_DTYPE_F32)
    to_bricks_kernel<float><<<(int)blocks, 256, 0, st>>>(
        static_cast<const float*>(flat->ptr), static_cast<float*>(bricked), n[0], n[1], n[2], nd,
        s, nb[0], nb[1], nb[2]);
  else
    return csd_internal_fail(CSD_EINVAL, "unsupported dtype");
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CSD_OK : csd_internal_fail(CSD_ELAUNCH, cudaGetErrorString(e));
}

extern "C" int csd_from_bricks(const void* bricked, int brick, const csd_field* flat, void* stream) {
  long long n[3], nb[3];
  int nd = 0, s = 0;
  int rc = brick_geometry(flat, brick, n, nb, &nd, &s);
  if (rc) return rc;
  if (!bricked) return csd_internal_fail(CSD_EINVAL, "null bricked buffer");
  const long long total = n[0] * n[1] * n[2];
  long long blocks = (total + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (flat->dtype == CSD_DTYPE_F64)
    from_bricks_kernel<double><<<(int)blocks, 256, 0, st>>>(
        static_cast<const double*>(bricked), static_cast<double*>(flat->ptr), n[0], n[1], n[2], nd,
        s, nb[1], nb[2]);
  else if (flat->dtype == CSD_DTYPE_F32)
    from_bricks_kernel<float><<<(int)blocks, 256, 0, st>>>(
        static_cast<const float*>(bricked), static_cast<float*>(flat->ptr), n[0], n[1], n[2], nd,
        s, nb[1], nb[2]);
  else
    return csd_internal_fail(CSD_EINVAL, "unsupported dtype");
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CSD_OK : csd_internal_fail(CSD_ELAUNCH, cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// FP64 reductions over the interior of a field (mass, energy, residual, max)
//
// Deterministic: pass 1 gives CTA b the interior rows [b*R/G, (b+1)*R/G) of
// the (Z*Y) x X row grid; each thread accumulates its elements in a fixed
// order in FP64, then a fixed-shape tree reduces the CTA's threads into
// partials[b].  Pass 2 (one CTA) reduces partials[0..G) the same way.  The
// result depends on G, never on scheduling.
// ---------------------------------------------------------------------------
namespace {

constexpr int RED_THREADS = 256;

template <int OP>
__device__ __forceinline__ double red_combine(double a, double b) {
  if (OP == CSD_RED_MAXABS || OP == CSD_RED_DIFF_MAXABS) return (a != a || a > b) ? a : b;
  return a + b;
}

template <int OP>
__device__ __forceinline__ double red_block(double v, double* sh) {
  // fixed-shape tree: warp shuffles, then the warp totals in order
  for (int o = 16; o > 0; o >>= 1) v = red_combine<OP>(v, __shfl_down_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
    t = sh[0];
    for (int w = 1; w < RED_THREADS / 32; ++w) t = red_combine<OP>(t, sh[w]);
  }
  __syncthreads();
  return t;
}

template <typename T, int OP>
__global__ void __launch_bounds__(RED_THREADS) reduce_pass1(const T* a, const T* b, long long d0,
                                                            long long d1, long long d2, int h0,
                                                            int h1, int h2, double* partials) {
  __shared__ double sh[RED_THREADS / 32];
  const long long ny = d1 - 2 * h1, nx = d2 - 2 * h2;
  const long long rows = (d0 - 2 * h0) * ny;
  const long long r0 = rows * blockIdx.x / gridDim.x, r1 = rows * (blockIdx.x + 1) / gridDim.x;
  double acc = 0.0;
  for (long long r = r0; r < r1; ++r) {
    const long long z = r / ny + h0, y = r % ny + h1;
    const long long base = (z * d1 + y) * d2 + h2;
    for (long long x = threadIdx.x; x < nx; x += RED_THREADS) {
      const double va = (double)a[base + x];
      double v;
      if (OP == CSD_RED_SUM) v = va;
      else if (OP == CSD_RED_SUMSQ) v = va * va;
      else if (OP == CSD_RED_MAXABS) v = fabs(va);
      else {
        const double d = va - (double)b[base + x];
        v = (OP == CSD_RED_DIFF_SUMSQ) ? d * d : fabs(d);
      }
      acc = red_combine<OP>(acc, v);
    }
  }
  const double t = red_block<OP>(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

template <int OP>
__global__ void __launch_bounds__(RED_THREADS) reduce_pass2(const double* partials, int n,
                                                            double* result) {
  __shared__ double sh[RED_THREADS / 32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += RED_THREADS) acc = red_combine<OP>(acc, partials[i]);
  const double t = red_block<OP>(acc, sh);
  if (threadIdx.x == 0) *result = t;
}

template <typename T, int OP>
int reduce_t(const csd_field* a, const csd_field* b, const long long d[3], const int h[3],
             double* partials, int nblocks, double* result, cudaStream_t s) {
  const T* pa = reinterpret_cast<const T*>(a->ptr);
  const T* pb = b ? reinterpret_cast<const T*>(b->ptr) : nullptr;
  reduce_pass1<T, OP><<<nblocks, RED_THREADS, 0, s>>>(pa, pb, d[0], d[1], d[2], h[0], h[1], h[2],
                                                      partials);
  reduce_pass2<OP><<<1, RED_THREADS, 0, s>>>(partials, nblocks, result);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CSD_OK : csd_internal_fail(CSD_ELAUNCH, cudaGetErrorString(e));
}

template <typename T>
int reduce_dispatch(int op, const csd_field* a, const csd_field* b, const long long d[3],
                    const int h[3], double* partials, int nblocks, double* result,
                    cudaStream_t s) {
  switch (op) {
    case CSD_RED_SUM: return reduce_t<T, CSD_RED_SUM>(a, b, d, h, partials, nblocks, result, s);
    case CSD_RED_SUMSQ: return reduce_t<T, CSD_RED_SUMSQ>(a, b, d, h, partials, nblocks, result, s);
    case CSD_RED_MAXABS: return reduce_t<T, CSD_RED_MAXABS>(a, b, d, h, partials, nblocks, result, s);
    case CSD_RED_DIFF_SUMSQ:
      return reduce_t<T, CSD_RED_DIFF_SUMSQ>(a, b, d, h, partials, nblocks, result, s);
    case CSD_RED_DIFF_MAXABS:
      return reduce_t<T, CSD_RED_DIFF_MAXABS>(a, b, d, h, partials, nblocks, result, s);
  }
  return csd_internal_fail(CSD_EINVAL, "unknown reduction");
}

}  // namespace

extern "C" int csd_reduce(const csd_field* a, const csd_field* b, const int* halo, int op,
                          double* partials, int nblocks, double* result, void* stream) {
  if (!a || !a->ptr || !halo || !partials || !result || nblocks < 1)
    return csd_internal_fail(CSD_EINVAL, "null argument or nblocks < 1");
  if (a->ndim < 1 || a->ndim > 3) return csd_internal_fail(CSD_EINVAL, "ndim must be 1-3");
  if (!packed(a)) return csd_internal_fail(CSD_EINVAL, "reductions need C-contiguous fields");
  const bool diff = (op == CSD_RED_DIFF_SUMSQ || op == CSD_RED_DIFF_MAXABS);
  if (diff) {
    if (!b || !b->ptr || b->dtype != a->dtype || b->ndim != a->ndim)
      return csd_internal_fail(CSD_EINVAL, "difference reductions need a second field like the first");
    if (!packed(b)) return csd_internal_fail(CSD_EINVAL, "reductions need C-contiguous fields");
    for (int i = 0; i < a->ndim; ++i)
      if (b->shape[i] != a->shape[i]) return csd_internal_fail(CSD_EINVAL, "field shapes differ");
  }
  long long d[3] = {1, 1, 1};
  int h[3] = {0, 0, 0};
  const int off = 3 - a->ndim;
  for (int i = 0; i < a->ndim; ++i) {
    d[off + i] = a->shape[i];
    h[off + i] = halo[i];
    if (d[off + i] - 2 * h[off + i] < 1) return csd_internal_fail(CSD_EINVAL, "empty interior");
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (a->dtype == CSD_DTYPE_F64)
    return reduce_dispatch<double>(op, a, diff ? b : nullptr, d, h, partials, nblocks, result, s);
  if (a->dtype == CSD_DTYPE_F32)
    return reduce_dispatch<float>(op, a, diff ? b : nullptr, d, h, partials, nblocks, result, s);
  return csd_internal_fail(CSD_EINVAL, "unsupported dtype");
}

// ---------------------------------------------------------------------------
// Allocation-free reduction entry point.
//
// For callers that must not allocate device memory themselves: a host
// process whose device memory is entirely owned by another allocator (a
// framework's caching pool, a fixed up-front reservation), or a loop that
// cannot afford cudaMalloc's implicit device synchronisation between steps.
// They cannot provide the `partials` scratch csd_reduce needs, so this
// variant keeps its per-block partials in a file-scope device array of fixed
// size, which every device holds from the moment the library's kernels load
// until the process exits.
// ---------------------------------------------------------------------------
#include <mutex>

namespace {

// One partial per block of pass 1 (8 KB).  Shared by every call: pass 1
// overwrites each of the `nblocks` entries it uses before pass 2 reads them,
// so nothing has to be cleared between calls, but two calls that run at the
// same time on the GPU (different streams) race on these entries.
static __device__ __align__(256) double g_noalloc_partials[CSD_NOALLOC_MAX_BLOCKS];

// Device address of g_noalloc_partials per device ordinal (the host-side
// name is only a stand-in for the symbol, never a device pointer), with the id
// of the context it was looked up in: after cudaDeviceReset the device gets a
// new context, the old address is void, and the next call looks it up again.
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[64] = {nullptr};
unsigned long long g_noalloc_ctx[64] = {0};

int noalloc_scratch(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return csd_internal_fail(CSD_ENODEV, cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return csd_internal_fail(CSD_EINVAL, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  const unsigned long long ctx = csd_internal_ctx_id();
  if (!g_noalloc_ptr[dev] || ctx == 0 || ctx != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess)
      return csd_internal_fail(CSD_ELAUNCH, cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<double*>(p);
    g_noalloc_ctx[dev] = csd_internal_ctx_id();  // the lookup may have created the context
  }
  *out = g_noalloc_ptr[dev];
  return CSD_OK;
}

}  // namespace

extern "C" int csd_reduce_noalloc(const csd_field* a, const csd_field* b, const int* halo, int op,
                                  int nblocks, double* result, void* stream) {
  if (nblocks < 1 || nblocks > CSD_NOALLOC_MAX_BLOCKS)
    return csd_internal_fail(CSD_EINVAL,
                             "csd_reduce_noalloc: nblocks must be 1..1024 (the static scratch "
                             "holds 1024 partials)");
  if (!a || !a->ptr || !halo || !result)
    return csd_internal_fail(CSD_EINVAL, "csd_reduce_noalloc: null argument");
  double* partials = nullptr;
  int rc = noalloc_scratch(&partials);
  if (rc) return rc;
  return csd_reduce(a, b, halo, op, partials, nblocks, result, stream);
}

// ---------------------------------------------------------------------------
// CFL time-step control for batched solvers: dt[i] = cfl * scale[i] / smax[i]
// (smax = the per-grid maximum signal speed from a max-reduction launch),
// then smax[i] = 0 so the next reduction starts afresh.  One thread per grid.
// ---------------------------------------------------------------------------
namespace {
__global__ void cfl_update_kernel(int n, double* smax, const double* scale, double cfl,
                                  double dt_max, double* dt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double s = smax[i];
  double v = (s > 0.0) ? __ddiv_rn(__dmul_rn(cfl, scale[i]), s) : dt_max;
  if (v > dt_max) v = dt_max;
  dt[i] = v;
  smax[i] = 0.0;
}
}  // namespace

extern "C" int csd_cfl_update(int n, double* smax, const double* scale, double cfl, double dt_max,
                              double* dt, void* stream) {
  if (n < 1 || !smax || !scale || !dt) return csd_internal_fail(CSD_EINVAL, "bad cfl arguments");
  cfl_update_kernel<<<(n + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      n, smax, scale, cfl, dt_max, dt);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CSD_OK : csd_internal_fail(CSD_ELAUNCH, cudaGetErrorString(e));
}
