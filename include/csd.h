/*
 * csd.h -- C ABI of the B200 stencil backend (libcsd.so).
 *
 * The reference (cutile-stencil-dsl) has no native boundary: its generated
 * module is Python that calls cuTile (`ct.launch`, emitted by
 * cutile/lowering/target_to_python.py:356-399) and CuPy slice copies for
 * boundaries (target_to_python.py:199-297).  This header is the boundary
 * that replaces those calls.  Each entry point cites the reference interface
 * it stands in for, or says that it has none.
 *
 * Conventions: every function returns 0 on success or a CSD_E* code; the
 * message of the last failure on the calling thread is csd_last_error().
 * Arrays are C-contiguous device buffers described by csd_field; strides
 * are in elements.  Launches are asynchronous on the given CUDA stream
 * (NULL = the legacy default stream) and allocate nothing per call.
 */
#ifndef CSD_H
#define CSD_H

#include <stddef.h>
#include <stdint.h>

#include "../cutile-stencil-dsl_b200/csrc/include/csd/params.h"

#ifdef __cplusplus
extern "C" {
#endif

#define CSD_OK 0
#define CSD_EINVAL 1      /* invalid argument (shape, dtype, count) */
#define CSD_EALIGN 2      /* misaligned pointer or pitch for the requested path */
#define CSD_ECOMPILE 3    /* NVRTC compilation failed (log in csd_last_error) */
#define CSD_ELAUNCH 4     /* CUDA driver / launch failure */
#define CSD_ETIMEOUT 5    /* a kernel gave up waiting (device error word set) */
#define CSD_ENODEV 6      /* no CUDA driver or device */
#define CSD_ENOSYM 7      /* kernel or descriptor missing from a module */

#define CSD_DTYPE_F32 1
#define CSD_DTYPE_F64 2

typedef struct csd_module csd_module;
typedef struct csd_kernel csd_kernel;

/* One array argument: C-contiguous, `ndim` dims, sizes in `shape`. */
typedef struct csd_field {
  void* ptr;
  int ndim;
  int dtype;            /* CSD_DTYPE_* */
  int64_t shape[3];
  int64_t strides[3];   /* elements; must describe a C-contiguous layout */
} csd_field;

/* Per-launch (per-grid) options (zero-initialise for defaults). */
typedef struct csd_launch_opts {
  int halo[3];          /* array halo width per array dim (interior = shape - 2*halo) */
  int zchunk;           /* output rows per work item along dim 0 (0 = sized at launch) */
  int grid;             /* persistent CTAs (0 = occupancy x SM count) */
  int loader;           /* -1 auto, CSD_LOADER_TMA, CSD_LOADER_LDG */
  double bc_value;      /* Dirichlet value when the kernel fuses a boundary fill */
  uint64_t timeout_ns;  /* bound on device waits (0 = 2 s) */
  double scalars[CSD_MAX_SCALARS];  /* values of the stencil's scalar parameters */
  const double* dyn;    /* device array of per-grid dynamic scalars (e.g. dt), or NULL */
  double* red;          /* device double receiving a max-reduction, or NULL */
  int bc_odd[CSD_MAX_FIELDS];       /* per field: bit d = sign flip when mirrored in dim d */
  const int* grid_index;  /* csd_launch_batch: device map from batch position to descriptor
                             index in `grids` (NULL = identity), so descriptors can stay
                             resident in a pool while the batch changes */
  int withhold_chunk;   /* failure-test hook (0 = off): the first work item of CTA 0 never
                           requests input chunk withhold_chunk - 1, so its wait runs out after
                           timeout_ns; the CTA drains its other copies and exits, and
                           csd_error_word then reports CSD_ERR_TIMEOUT.  Nothing faults or
                           hangs: every other CTA finishes normally. */
} csd_launch_opts;

/* Library version (major*100 + minor). */
int csd_version(void);

/* sizeof(csd_grid), for callers that allocate descriptor arrays. */
size_t csd_grid_size(void);

/* Message of the last error on this thread ("" if none). */
const char* csd_last_error(void);

/* Compile `src` (CUDA C++ of a generated stencil module) for sm_100a with
 * NVRTC, caching the cubin under `cache_dir` (NULL: no disk cache), and load
 * it into the current device's primary context.  `headers`/`header_names`
 * provide the engine headers the source includes.  Replaces cuTile's JIT of
 * the generated module at first launch (reference: README.md:487-492,
 * runtime/launcher.py:62-74 `load_module`). */
int csd_module_load(const char* src, int n_headers, const char* const* headers,
                    const char* const* header_names, const char* options,
                    const char* cache_dir, csd_module** out);

/* Compile only (no device needed): writes the cubin path into `cubin_path`
 * (buffer of `path_len` bytes) and the NVRTC log (ptxas -v) into `log`. */
int csd_compile(const char* src, int n_headers, const char* const* headers,
                const char* const* header_names, const char* options, const char* cache_dir,
                char* cubin_path, size_t path_len, char* log, size_t log_len);

/* Load a prebuilt sm_100a cubin (`image`, `size` bytes) into the current
 * device's primary context: the ahead-of-time form of csd_module_load, for a
 * generated module compiled by nvcc from the `.cu` that
 * CompileResult.build_aot writes.  Stands in for loading the artefact of the
 * reference's `CompileResult.code` / `emit_to_file` (runtime/launcher.py:57-60)
 * without a JIT at first launch. */
int csd_module_load_image(const void* image, size_t size, csd_module** out);

int csd_module_unload(csd_module* m);

/* Look up stencil kernel `name` (its `<name>_tma`, `<name>_ldg` entry points
 * and `<name>_desc` descriptor).  Stands in for the generated
 * `<name>_kernel` object (target_to_python.py:34-191). */
int csd_kernel_get(csd_module* m, const char* name, csd_kernel** out);

/* Copy the kernel's compile-time descriptor. */
int csd_kernel_describe(const csd_kernel* k, csd_kernel_desc* out);

/* Registers per thread, local (spill) bytes per thread and resident blocks
 * per SM of the TMA variant.  Replaces the reference's cubin probe
 * (runtime/regcheck.py:136-212) with driver attributes. */
int csd_kernel_resources(csd_kernel* k, int* regs, int* local_bytes, int* blocks_per_sm);

/* One stencil pass: read `in[0..n_in)`, write the interior of
 * `out[0..n_out)`.  Equivalent of `launch_<name>(inputs..., outputs...)`
 * (stencil_to_target.py:677-843): `temporal` steps per call for chained
 * kernels, output halos untouched. */
int csd_launch(csd_kernel* k, const csd_field* in, int n_in, const csd_field* out, int n_out,
               const csd_launch_opts* opts, void* stream);

/* Describe one grid of a batched launch: validates the fields like
 * csd_launch and writes the kernel-side descriptor (TMA maps included) into
 * host memory `*g`; `*items` receives its number of work items and
 * `*loader_used` the copy path it qualifies for (opts->loader = -1: TMA when
 * aligned, else cp.async; all grids of one batch must use the same path).
 * The caller copies the descriptors of all grids to device memory for
 * csd_launch_batch.  No reference counterpart (the reference launches one
 * grid per call). */
int csd_grid_build(csd_kernel* k, const csd_field* in, int n_in, const csd_field* out, int n_out,
                   const csd_launch_opts* opts, csd_grid* g, int* items, int* loader_used);

/* Work split of grid `g` (tiles[0], tiles[1] and interior[0] set) for kernel
 * `desc` on `slots` resident CTAs: sets zchunk, tiles[2], items and, for
 * fused-boundary kernels sized for one wave, the uneven split described at
 * csd_grid::ecols.  `zchunk_req` > 0 forces the rows per item.  Host only
 * (csd_launch and csd_grid_build call it).  Replaces the reference's
 * `_fit_tiles` grid sizing (target_to_python.py:305-348). */
int csd_plan_items(const csd_kernel_desc* desc, long long slots, int zchunk_req, csd_grid* g);

/* Host decode of work item `item` of a planned grid: column (tx, ty) and the
 * interior Z rows [z0, z0 + nrows) it writes (the kernels use the same
 * function, csd_item_place).  No reference counterpart. */
int csd_grid_item_place(const csd_grid* g, int item, int* tx, int* ty, int* z0, int* nrows);

/* One persistent launch over many grids of uneven sizes: `grids` (device)
 * holds `ngrids` descriptors from csd_grid_build, `item_start` (device) the
 * prefix sums of their work items (ngrids + 1 ints, last = total).  Work
 * items are spread over the resident CTAs; each grid is advanced exactly as
 * csd_launch would.  `grid` in `opts` overrides the CTA count; `loader` in
 * `opts` selects the copy path the descriptors were built for. */
int csd_launch_batch(csd_kernel* k, const csd_grid* grids, const int* item_start, int ngrids,
                     int total_items, const csd_launch_opts* opts, void* stream);

/* Per-grid CFL step for batched solvers (device arrays of length n):
 * dt[i] = min(cfl * scale[i] / smax[i], dt_max) (dt_max when smax[i] is 0),
 * then smax[i] = 0 for the next max-reduction.  No reference counterpart
 * (the reference's examples use a fixed host-side dt). */
int csd_cfl_update(int n, double* smax, const double* scale, double cfl, double dt_max,
                   double* dt, void* stream);

/* Fill the halo of `f` in place with boundary condition `bc` (CSD_BC_*),
 * dimension by dimension.  Equivalent of `apply_boundary_<name>(u)`
 * (target_to_python.py:199-297) and stencil_ref.apply_boundary
 * (reference/stencil_ref.py:102-201). */
int csd_apply_boundary(const csd_field* f, const int* halo, int bc, double value, void* stream);

#define CSD_RED_SUM 0         /* mass:      sum(a) */
#define CSD_RED_SUMSQ 1       /* energy:    sum(a^2) */
#define CSD_RED_MAXABS 2      /* max |a| (NaN propagates) */
#define CSD_RED_DIFF_SUMSQ 3  /* residual:  sum((a-b)^2) */
#define CSD_RED_DIFF_MAXABS 4 /* max |a-b| */

/* FP64 reduction over the interior of `a` (and `b` for the DIFF ops),
 * deterministic for a given `nblocks`: pass 1 writes one partial per block
 * into the caller's device scratch `partials[nblocks]`, pass 2 writes the
 * total to the device double `*result`.  No reference counterpart: the
 * reference reduces on the host with NumPy (e.g. examples/shallow_water.py
 * energy); the B200 path keeps these global sums on the device in FP64. */
int csd_reduce(const csd_field* a, const csd_field* b, const int* halo, int op,
               double* partials, int nblocks, double* result, void* stream);

/* csd_reduce without caller-provided scratch, for callers that cannot
 * allocate device memory (their device memory belongs to another allocator,
 * or a step loop must not pay cudaMalloc's device synchronisation).  The
 * per-block partials live in a file-scope device array of
 * CSD_NOALLOC_MAX_BLOCKS = 1024 doubles (8 KB) that every device keeps until
 * the process exits; `nblocks` above 1024 is rejected with CSD_EINVAL.  The
 * first call on a device looks up the array's device address (with that
 * device current); make that first call before any stream capture.  After
 * cudaDeviceReset the device has a new context and the next call looks the
 * address up again, so that call too belongs before any capture.  Calls
 * share the array, so calls that overlap on the GPU race; each call
 * overwrites the partials it uses, so no clearing is needed.  Nothing is
 * allocated.  No counterpart in the reference. */
#define CSD_NOALLOC_MAX_BLOCKS 1024
int csd_reduce_noalloc(const csd_field* a, const csd_field* b, const int* halo, int op,
                       int nblocks, double* result, void* stream);

/* Bricked layout (replaces the generated to_bricks / from_bricks helpers,
 * multigpu_emitter.py:370-424).  A bricked array stores a 1-3-D array as
 * bricks of B^ndim elements (B = `brick`, a power of two), bricks row-major
 * over the brick grid ceil(shape / B), each brick row-major inside; cells of
 * the padding are zero.  csd_bricked_elems gives the element count of the
 * bricked buffer.  `flat` must be C-contiguous; both calls are one kernel
 * launch on `stream`.  A kernel compiled with layout="bricked" reads and
 * writes fields in this layout (fields described by their flat shape). */
long long csd_bricked_elems(const long long* shape, int ndim, int brick);
int csd_to_bricks(const csd_field* flat, int brick, void* bricked, void* stream);
int csd_from_bricks(const void* bricked, int brick, const csd_field* flat, void* stream);

/* Read (and with reset != 0, clear) the device error word of the current
 * device; synchronises the device.  `value` receives the word (0, or
 * CSD_ERR_TIMEOUT when a kernel's wait for its input ran out: that CTA
 * drained its copies in flight and stopped, so its outputs are incomplete).
 * Returns CSD_OK for a clear word, CSD_ETIMEOUT for CSD_ERR_TIMEOUT. */
int csd_error_word(int* value, int reset);

#ifdef __cplusplus
}
#endif

#endif /* CSD_H */
