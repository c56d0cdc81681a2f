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

namespace {

template <typename T>
__global__ void fill_dim_kernel(T* u, long long d0, long long d1, long long d2, int dim, int h,
                                int bc, T value) {
  // The array is viewed as (d0, d1, d2); `dim` selects the dimension whose
  // halo is filled.  Each thread owns one halo cell of that dimension.
  const long long n[3] = {d0, d1, d2};
  const long long nd = n[dim];
  long long other = 1;
  for (int i = 0; i < 3; ++i)
    if (i != dim) other *= n[i];
  const long long total = 2LL * h * other;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long k2 = e / other;      // 0 .. 2h-1 : which halo layer
    long long rest = e % other;
    const bool high = k2 >= h;
    const long long k = high ? k2 - h : k2;
    long long idx[3];
    // rest enumerates the other two dims in order
    int j = 2;
    for (int i = 2; i >= 0; --i) {
      if (i == dim) continue;
      idx[i] = rest % n[i];
      rest /= n[i];
      (void)j;
    }
    long long dst_i, src_i;
    if (!high) {
      dst_i = k;
      if (bc == CSD_BC_NEUMANN) src_i = h;
      else if (bc == CSD_BC_PERIODIC) src_i = nd - 2 * h + k;
      else src_i = 2 * h - 1 - k;  // reflecting
    } else {
      dst_i = nd - h + k;
      if (bc == CSD_BC_NEUMANN) src_i = nd - h - 1;
      else if (bc == CSD_BC_PERIODIC) src_i = h + k;
      else src_i = nd - h - 1 - k;
    }
    idx[dim] = dst_i;
    const long long dst = (idx[0] * n[1] + idx[1]) * n[2] + idx[2];
    if (bc == CSD_BC_DIRICHLET) {
      u[dst] = value;
    } else {
      idx[dim] = src_i;
      const long long src = (idx[0] * n[1] + idx[1]) * n[2] + idx[2];
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
  for (int d = 0; d < 3; ++d) {
    if (h3[d] == 0) continue;
    if (bc != CSD_BC_DIRICHLET && n[d] - 2 * h3[d] < h3[d])
      return csd_internal_fail(CSD_EINVAL, "boundary fill needs an interior at least as wide as the halo");
    long long other = 1;
    for (int i = 0; i < 3; ++i)
      if (i != d) other *= n[i];
    const long long total = 2LL * h3[d] * other;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    fill_dim_kernel<T><<<blocks, 256, 0, s>>>(reinterpret_cast<T*>(f->ptr), n[0], n[1], n[2], d,
                                              h3[d], bc, (T)value);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return csd_internal_fail(CSD_ELAUNCH, cudaGetErrorString(e));
  }
  return CSD_OK;
}

}  // namespace

extern "C" int csd_apply_boundary(const csd_field* f, const int* halo, int bc, double value,
                                  void* stream) {
  if (!f || !halo || !f->ptr) return csd_internal_fail(CSD_EINVAL, "null argument");
  if (f->ndim < 1 || f->ndim > 3) return csd_internal_fail(CSD_EINVAL, "ndim must be 1-3");
  if (bc < CSD_BC_DIRICHLET || bc > CSD_BC_REFLECTING)
    return csd_internal_fail(CSD_EINVAL, "unknown boundary condition");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (f->dtype == CSD_DTYPE_F64) return apply_boundary_t<double>(f, halo, bc, value, s);
  if (f->dtype == CSD_DTYPE_F32) return apply_boundary_t<float>(f, halo, bc, value, s);
  return csd_internal_fail(CSD_EINVAL, "unsupported dtype");
}
