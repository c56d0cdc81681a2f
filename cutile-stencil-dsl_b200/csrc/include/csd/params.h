// Launch parameters and kernel descriptors shared by the host runtime
// (libcsd.so, compiled by nvcc/g++) and the JIT-compiled stencil kernels
// (NVRTC).  Plain C layout, no system headers, identical on both sides.
#ifndef CSD_PARAMS_H
#define CSD_PARAMS_H

#define CSD_MAX_FIELDS 8
#define CSD_MAX_SCALARS 8
#define CSD_DESC_MAGIC 0x43534434u /* "CSD4": bumped with every csd_grid layout change */

#define CSD_LOADER_TMA 0
#define CSD_LOADER_LDG 1

#define CSD_BC_NONE 0
#define CSD_BC_DIRICHLET 1
#define CSD_BC_NEUMANN 2
#define CSD_BC_PERIODIC 3
#define CSD_BC_REFLECTING 4

#define CSD_ERR_TIMEOUT 0x7001

#ifdef __cplusplus
extern "C" {
#endif

// Opaque 128-byte TMA descriptor (same size/alignment as CUtensorMap).
typedef struct __attribute__((aligned(64))) csd_tmap {
  unsigned long long opaque[16];
} csd_tmap;

// One grid (a set of same-shaped fields) as a kernel sees it.  Arrays are
// viewed as 3-D (Z, Y, X) with X innermost; a 2-D array (rows, cols) is
// (rows, 1, cols), a 1-D array (n) is (1, 1, n).
typedef struct __attribute__((aligned(64))) csd_grid {
  csd_tmap tmap[CSD_MAX_FIELDS];      // TMA descriptors of the inputs
  const void* in[CSD_MAX_FIELDS];     // input base pointers
  void* out[CSD_MAX_FIELDS];          // output base pointers
  long long dims[3];                  // full extents (Z, Y, X), halo included
  long long pitch_y;                  // elements between consecutive Y
  long long pitch_z;                  // elements between consecutive Z
  int halo[3];                        // array halo per internal dim (Z, Y, X)
  int interior[3];                    // dims - 2 * halo
  int tiles[3];                       // x tiles, y tiles, z chunks
  int items;                          // tiles[0] * tiles[1] * tiles[2]
  int zchunk;                         // output rows of Z per work item
  int xbase;                          // X origin of tile 0 (halo rounded down to 16 B)
  int vec_store;                      // 1 when 16-byte output stores are aligned
  int ndim;                           // array dimensionality (1-3)
  // Uneven work split of fused-boundary kernels.  Chunks of an X-edge column
  // also take the boundary patch, so with ecols == 2 the two X-edge columns
  // get their own, shorter items (item numbers items_main onward, zchunk_e
  // rows); and the first and last item of a column, which patch the Z
  // boundary, are zshift (zshift_e) rows shorter than the others: item tz of
  // a column covers interior rows [tz*zc - zs, (tz+1)*zc - zs) clipped to
  // [0, nz).  ecols == 0 and zshift == 0 give the uniform split.
  int ecols;
  int items_main;
  int zchunk_e;
  int zshift;
  int zshift_e;
  double scalars[CSD_MAX_SCALARS];    // per-grid constants read by the body (s<k>)
  const double* dyn;                  // per-grid device scalars (d<k>), may be null
  double* red;                        // per-grid max-reduction slot, may be null
  double bc_value;                    // Dirichlet value of a fused boundary fill
  int bc_odd[CSD_MAX_FIELDS];         // bit d: mirrored values of field f flip sign in dim d
  // Bricked fields (kernels compiled for a brick size): the array is stored
  // as bricks of B^ndim elements (B = 1 << brick_shift), brick-major, each
  // brick row-major inside; nbx / nby bricks along X / Y of the padded array.
  int brick_shift;                    // 0: flat (pitched) layout
  int nbx, nby;
  int ybase;                          // Y origin of tile row 0 (the Y halo, or for bricked
                                      // TMA staging the halo rounded down to the tile height)
  // Periodic-X kernels (TMA loader): narrow boxes (wrap width x box height x
  // rows) of the inputs, loaded from the far side of a row for X-edge chunks.
  // Bricked fields staged by TMA: the one-row box of each input (tmap holds
  // the tile-height box).
  csd_tmap tmap_wrap[CSD_MAX_FIELDS];
} csd_grid;

#if defined(__CUDACC__) || defined(__CUDACC_RTC__)
#define CSD_HOST_DEVICE __host__ __device__ __forceinline__
#else
#define CSD_HOST_DEVICE static inline
#endif

// Column (tx, ty) and interior Z rows [z0, z0 + nrows) of work item `item` of
// grid `g` (the split is described at csd_grid::ecols).  The kernels and the
// host (csd_grid_item_place) decode items with this one function.
CSD_HOST_DEVICE void csd_item_place(const csd_grid* g, int item, int* tx, int* ty, int* z0,
                                    int* nrows) {
  const int edge = g->ecols != 0 && item >= g->items_main;
  const int c = edge ? item - g->items_main : item;
  const int w = g->ecols == 0 ? g->tiles[0] : (edge ? 2 : g->tiles[0] - 2);
  const int zc = edge ? g->zchunk_e : g->zchunk;
  const int zs = edge ? g->zshift_e : g->zshift;
  const int cx = c % w;
  const int t1 = c / w;
  const int tz = t1 / g->tiles[1];
  int lo = tz * zc - zs, hi = (tz + 1) * zc - zs;
  if (lo < 0) lo = 0;
  if (hi > g->interior[0]) hi = g->interior[0];
  *ty = t1 % g->tiles[1];
  *tx = edge ? (cx ? g->tiles[0] - 1 : 0) : cx + (g->ecols ? 1 : 0);
  *z0 = lo;
  *nrows = hi - lo;
}

// Kernel parameter: one grid inline, or a device array of grids.
typedef struct __attribute__((aligned(64))) csd_params {
  csd_grid g;                         // the grid of a single-grid launch
  const csd_grid* grids;              // batched launch: device array (null otherwise)
  const int* item_start;              // batched: prefix sums of items, ngrids + 1 entries
  const int* grid_index;              // batched: descriptor of batch position k (null = k)
  int ngrids;
  int total_items;
  int* err;                           // device error word (0 = ok)
  unsigned long long timeout_ns;      // bound on every wait for input
  int withhold;                       // failure-test hook (csd_launch_opts::withhold_chunk)
} csd_params;

// Compile-time configuration of a kernel, exported by each JIT module as
// `extern "C" __device__ const csd_kernel_desc <name>_desc`.
typedef struct csd_kernel_desc {
  unsigned int magic;
  int ndim;          // stencil dimensionality (1-3)
  int nin, nout;     // fields read / written
  int dtype_bytes;   // 4 or 8
  int rz, ry, rx;    // stencil radius per internal dim (whole temporal chain)
  int rows;          // Z rows per streaming step
  int tile_y, tile_x;
  int vec;           // X points per thread
  int threads;
  int stages;        // chunks in flight
  int nslot;         // ring slots
  int halo_chunks;
  int pad_left, box_w, box_h;
  int smem_bytes;
  int zchunk;        // default Z rows per work item (0 = sized at launch for one
                     // item per resident block, -W = W items per resident block)
  int temporal;      // stencil steps per pass
  int bc_mode;       // CSD_BC_* fused into the staging (0 = none)
  int min_blocks;
  int align;         // elements per 16 bytes
  int nscalars;      // static per-grid scalars the body reads
  int ndyn;          // device per-grid scalars the body reads
  int reduce_max;    // 1: the body also max-reduces a value into grid.red
  int brick_shift;   // log2 of the brick size of a bricked-layout kernel (0 = flat)
  int brick_tma;     // 1: the bricked kernel's TMA entry stages bricks with tensor copies
} csd_kernel_desc;

#ifdef __cplusplus
}
#endif

#endif  // CSD_PARAMS_H
