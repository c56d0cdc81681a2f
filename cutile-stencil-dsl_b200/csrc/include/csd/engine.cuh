// Streaming stencil engine for sm_100a.
//
// A work item is a column of TY x TX points (internal dims Y, X) that walks
// ZCHUNK output rows of Z, ROWS rows per step.  Input rows reach shared
// memory as chunks of ROWS x BOXH x BOXW elements (the tile plus the
// stencil halo, X padded to 16-byte boundaries), either as one TMA tile
// copy per field per chunk (cp.async.bulk.tensor, completion counted on an
// mbarrier) or, when the array pitch is not 16-byte aligned, as per-element
// cp.async copies arriving on the same mbarrier.  Chunks live in a ring of
// NSLOT slots: 2*HC+1 are read by the current step, STAGES more are in
// flight.  Work items are handed out round-robin to a persistent grid.
//
// With TEMPORAL = T > 1 one pass chains T stencil steps (time skewing): at
// ring step i, stage s computes chunk i - s*HC of the s-th intermediate field
// into its own shared-memory ring (which is (T-s)*radius wider than the
// tile), and stage T writes the final field.  Intermediate points outside the
// domain interior are zero, which is what T separate launches through
// zero-halo scratch buffers produce.
//
// The stencil body is a functor emitted from the DSL: it reads "strips"
// (a row segment of one field at a Z/Y offset) through the tile view and
// evaluates each point with round-to-nearest intrinsics in DSL term order.
#ifndef CSD_ENGINE_CUH
#define CSD_ENGINE_CUH

#include "csd/params.h"
#include "csd/ptx.cuh"

namespace csd {

// Bound on the drain of an aborted work item (copies still in flight).
constexpr unsigned long long kDrainNs = 2000000000ull;
// Temporal chains: with CSD_CHAIN_SKEW (the default) stage s + 1 reads
// field s only from chunks finished at earlier ring steps (one more ring slot
// per stage, one barrier per ring step); without it stage s + 1 reads the
// chunk stage s wrote in the same step (a barrier after every stage).
#ifndef CSD_CHAIN_SKEW
#define CSD_CHAIN_SKEW 1
#endif
// Unroll also unit counts that do not divide the block (last round predicated).
#ifndef CSD_UNROLL_RAGGED
#define CSD_UNROLL_RAGGED 1
#endif

template <typename T>
struct VecOf;
template <>
struct VecOf<double> {
  typedef double2 type;
  static constexpr int N = 2;
};
template <>
struct VecOf<float> {
  typedef float4 type;
  static constexpr int N = 4;
};

__host__ __device__ constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }
__host__ __device__ constexpr int align_up(int a, int b) { return cdiv(a, b) * b; }
// floor division for possibly negative numerators (b > 0)
__host__ __device__ constexpr int fdiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }
__host__ __device__ constexpr int imax(int a, int b) { return a > b ? a : b; }

// ---------------------------------------------------------------------------
// Compile-time configuration
// ---------------------------------------------------------------------------
template <typename T_, int NIN_, int NOUT_, int RZ_, int RY_, int RX_, int ROWS_, int TY_, int TX_,
          int NT_, int STAGES_, int TEMPORAL_, int LOADER_, int BC_, int REDUCE_ = 0,
          int BRICK_ = 0, int RPY_ = 1, int VEC_ = 0>
struct Cfg {
  typedef T_ T;
  // Bricked layout: BRICK_ = (ndim << 4) | log2(brick size), 0 = flat.
  static constexpr int BRICK_SHIFT = BRICK_ & 15, BRICK_NDIM = BRICK_ >> 4;
  static constexpr int BRICK_B = BRICK_SHIFT ? (1 << BRICK_SHIFT) : 1;
  // Bricked fields staged by TMA: a 5-D tensor map over (x in brick, brick
  // x, y in brick, z in brick, brick y + nby * brick z) turns every box into
  // flat rows of whole bricks in shared memory, so the chunk layout (and the
  // body) are those of the flat path; tiles start on a brick in X and on a
  // tile height that divides the brick in Y.
  static constexpr bool BTMA = BRICK_SHIFT > 0 && LOADER_ == CSD_LOADER_TMA;
  static constexpr int NIN = NIN_, NOUT = NOUT_;
  static constexpr int RZ = RZ_, RY = RY_, RX = RX_;  // radius of ONE step
  static constexpr int ROWS = ROWS_, TY = TY_, TX = TX_;
  static constexpr int NT = NT_, STAGES = STAGES_, TEMPORAL = TEMPORAL_;
  static constexpr int LOADER = LOADER_, BC = BC_;
  static constexpr int REDUCE = REDUCE_;  // 1: max-reduce output 0 into grid.red, store nothing
  // Y rows per thread: a unit is RPY rows x VEC points, so the body can read
  // the strip of row y + 1 at offset dy once for both rows that need it
  static constexpr int RPY = RPY_;
  static constexpr int ALIGN = 16 / (int)sizeof(T);
  // points per unit along X: one 16-byte vector by default; a wider unit
  // (several vectors) reads each staged row group with fewer strips per
  // point, for single-step flat kernels with one row per thread
  static constexpr int VEC = VEC_ > 0 ? VEC_ : ALIGN;
  static_assert(VEC % ALIGN == 0 &&
                    (VEC == ALIGN || (TEMPORAL_ == 1 && BRICK_ == 0 && RPY_ == 1)),
                "units wider than one vector: single-step flat kernels, one row per thread");
  static constexpr int HC = RZ > 0 ? cdiv(RZ, ROWS) : 0;  // halo chunks per side, per step
  // Column layout shared by every buffer: smem column c <-> x = X0 - PADL + c.
  // bricked TMA rows: whole bricks, each row 128-byte aligned (TMA destination)
  static constexpr int BALIGN = imax(BRICK_B, 128 / (int)sizeof(T));
  static constexpr int PADL = BTMA ? align_up(RX, BRICK_B)
                            : TEMPORAL == 1 ? align_up(RX, VEC)
                                            : align_up(TEMPORAL * RX + 2 * ALIGN - 2, ALIGN);
  static constexpr int BOXW = BTMA ? align_up(PADL + TX + RX, BALIGN)
                            : TEMPORAL == 1 ? align_up(PADL + TX + RX, ALIGN)
                                            : align_up(PADL + TX + TEMPORAL * RX + 2 * ALIGN - 2, ALIGN);
  static_assert(BRICK_ == 0 || LOADER_ == CSD_LOADER_LDG ||
                    (BRICK_NDIM == 3 && ROWS_ == 1 && TEMPORAL_ == 1 && BC_ != CSD_BC_PERIODIC &&
                     (BRICK_B % TY_ == 0 || TY_ % BRICK_B == 0) && TX_ % BRICK_B == 0 &&
                     (BRICK_B * (int)sizeof(T_)) % 16 == 0 && BOXW / BRICK_B <= 256),
                "bricked TMA staging: 3-D bricks, one row per chunk, single step, no periodic "
                "wrap, tile height dividing or divided by the brick, tile width a multiple of it");
  // rows of one tile-row box (a box stays inside one brick row)
  static constexpr int BTMA_ROWS = TY_ < BRICK_B ? TY_ : BRICK_B;
  // Height (Y rows) of the buffer holding the field after s steps.
  static __host__ __device__ constexpr int H(int s) { return TY + 2 * (TEMPORAL - s) * RY; }
  static constexpr int BOXH = TY + 2 * TEMPORAL * RY;
  static constexpr int NSLOT = 2 * HC + 1 + STAGES;              // input ring
  // Intermediate rings: stage s + 1 reads field s only from chunks finished
  // in earlier ring steps, so one slot more than the 2*HC+1 it reads is being
  // written meanwhile (one barrier per ring step, not one per stage).
  static constexpr bool SKEW = CSD_CHAIN_SKEW != 0;
  static constexpr int NSLOT_I = 2 * HC + (SKEW ? 2 : 1);
  // Chunk of field s computed at ring step i: i - STAGE_OFF(s).
  static __host__ __device__ constexpr int STAGE_OFF(int s) { return s * HC + (SKEW ? s - 1 : 0); }
  static constexpr int SLOT_ELEMS = align_up(ROWS * BOXH * BOXW, 128 / (int)sizeof(T));
  static constexpr int CHUNK_BYTES = ROWS * BOXH * BOXW * (int)sizeof(T);  // TMA bytes
  static __host__ __device__ constexpr int ISLOT_ELEMS(int s) {
    return align_up(ROWS * H(s) * BOXW, 128 / (int)sizeof(T));
  }
  // Intermediate rings of stages 1..s-1; each stage keeps one ring per field
  // (a chain maps output field f to input field f of the next step).
  static __host__ __device__ constexpr int inter_elems_upto(int s) {
    return s <= 1 ? 0 : inter_elems_upto(s - 1) + NIN * NSLOT_I * ISLOT_ELEMS(s - 1);
  }
  static constexpr int RING_ELEMS = NIN * NSLOT * SLOT_ELEMS;
  static constexpr int INTER_ELEMS = inter_elems_upto(TEMPORAL);
  // Periodic X wrap (TMA loader): for a chunk at an X edge, a narrow TMA box
  // of WRAPW columns from the far side of the same rows lands with the chunk
  // in a per-slot wrap buffer: per field, a left and a right block of
  // ROWS x BOXH x WRAPW, each block 128-byte aligned.
  static constexpr int PLINES = ROWS * BOXH;
  static constexpr int PBUF = (BC == CSD_BC_PERIODIC && LOADER == CSD_LOADER_TMA && RX > 0) ? 1 : 0;
  static constexpr int WRAPW = align_up(RX, ALIGN) + ALIGN;
  static constexpr int WRAP_ELEMS = ROWS * BOXH * WRAPW;
  static constexpr int WRAP_BLOCK = align_up(WRAP_ELEMS, 128 / (int)sizeof(T));
  static constexpr int PBUF_SLOT = PBUF ? NIN * 2 * WRAP_BLOCK : 0;
  static constexpr int PBUF_ELEMS = NSLOT * PBUF_SLOT;
  static constexpr int BAR_OFFSET = (RING_ELEMS + INTER_ELEMS + PBUF_ELEMS) * (int)sizeof(T);
  // +128: the dynamic shared-memory base is aligned up to 128 bytes in the kernel
  static constexpr int SMEM_BYTES = BAR_OFFSET + 8 * NSLOT + 64 + 128;
  static_assert(BOXW <= 256 && BOXH <= 256 && ROWS <= 256, "TMA box limit");
  static_assert(TX % VEC == 0, "tile width must be a multiple of the vector width");
  static_assert(TEMPORAL == 1 || NIN == NOUT,
                "a temporal chain feeds output field f into input field f of the next step");
  static_assert(HC * ROWS >= RZ, "halo chunks");
  static_assert(BC == CSD_BC_NONE || TEMPORAL == 1, "fused boundary fill is single-step");
  static_assert(RPY >= 1 && TY % RPY == 0, "tile height must be a multiple of the rows per thread");
  static_assert(RPY == 1 || TEMPORAL == 1, "temporal chains take one row per thread");
};

// ---------------------------------------------------------------------------
// Strips: VEC consecutive points' worth of one row segment [LO, VEC-1+HI]
// ---------------------------------------------------------------------------
template <typename T, int LO, int HI, int VEC>
struct Strip {
  T v[VEC + HI - LO];
};

template <typename T, int LO, int HI, int VEC, int ALIGN>
__device__ __forceinline__ Strip<T, LO, HI, VEC> load_strip(const T* row, int x) {
  // row: smem row base; x: column of the unit's first point (multiple of ALIGN)
  constexpr int A0 = fdiv(LO, ALIGN) * ALIGN;             // aligned start offset
  constexpr int A1 = align_up(VEC + HI, ALIGN);            // aligned end offset (exclusive)
  constexpr int NV = (A1 - A0) / ALIGN;
  typedef typename VecOf<T>::type V;
  T buf[NV * ALIGN];
  const V* src = reinterpret_cast<const V*>(row + x + A0);
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const V t = src[i];
    *reinterpret_cast<V*>(&buf[i * ALIGN]) = t;
  }
  Strip<T, LO, HI, VEC> s;
#pragma unroll
  for (int i = 0; i < VEC + HI - LO; ++i) s.v[i] = buf[i + (LO - A0)];
  return s;
}

// View of one buffer (ring of chunks) for the body functor.
template <class C>
struct TileView {
  typedef typename C::T T;
  const T* base[C::NIN];  // per-field ring base
  int slot0;              // slot of the step's first source chunk
  int nslot;              // slots in the ring
  int slot_elems;
  int height;             // Y rows per chunk row
  int y_off;              // buffer row of the unit's y (source has extra halo rows)
  const double* scal;     // per-grid constants (csd_grid.scalars)
  const double* dyn;      // per-grid device scalars (csd_grid.dyn)

  __device__ __forceinline__ double scalar(int k) const { return scal[k]; }
  __device__ __forceinline__ double dynamic(int k) const { return dyn[k]; }

  // Row segment of field F at Z offset DZ and Y offset DY for unit (r, y, x).
  template <int F, int DZ, int DY, int LO, int HI>
  __device__ __forceinline__ Strip<T, LO, HI, C::VEC> strip(int r, int y, int x) const {
    const int q = C::HC * C::ROWS + r + DZ;  // >= 0
    const int c = q / C::ROWS;
    const int rr = q - c * C::ROWS;
    int slot = slot0 + c;
    if (slot >= nslot) slot -= nslot;
    const T* row = base[F] + slot * slot_elems + (rr * height + (y + y_off + DY)) * C::BOXW;
    return load_strip<T, LO, HI, C::VEC, C::ALIGN>(row, x);
  }
};

// Output value pack for one unit.
template <typename T, int NOUT, int VEC>
struct OutPack {
  T v[NOUT][VEC];
};

__device__ __forceinline__ void store_vec(double* p, const double* v) {
  *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
}
__device__ __forceinline__ void store_vec(float* p, const float* v) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
// One unit's VEC points as 16-byte vector stores.
template <int VEC, typename T>
__device__ __forceinline__ void store_unit(T* p, const T* v) {
  constexpr int A = 16 / (int)sizeof(T);
#pragma unroll
  for (int i = 0; i < VEC; i += A) store_vec(p + i, v + i);
}

// Fused boundary fill: map an out-of-interior index of one dim to the
// interior index whose value it takes (periodic / Neumann / reflecting), as
// apply_boundary does with its slab copies.  Dirichlet is handled by value.
__device__ __forceinline__ long long bc_map(long long i, int h, int n, int mode) {
  if (i >= h && i < h + n) return i;
  if (mode == CSD_BC_PERIODIC) {
    // one wrap covers every cell within a radius <= n of the interior; the
    // 64-bit remainder (a long software sequence) is only for wider halos
    if (i < h && i + n >= h) return i + n;
    if (i >= h + n && i - n < h + n) return i - n;
    long long k = (i - h) % n;
    if (k < 0) k += n;
    return h + k;
  }
  if (mode == CSD_BC_NEUMANN) return i < h ? h : h + n - 1;
  // reflecting: index h-1-k <- h+k, h+n+k <- h+n-1-k
  if (i < h) return 2 * h - 1 - i;
  return 2 * (h + n) - 1 - i;
}

// ---------------------------------------------------------------------------
// Correctly rounded division and square root for stencil bodies
// ---------------------------------------------------------------------------
// The IEEE-exact __fdiv_rn/__ddiv_rn/__fsqrt_rn/__dsqrt_rn sequences send a
// zero dividend or radicand to their out-of-line fix-up path.  In a field at
// rest (zero momenta, zero flux differences) that is the common case and
// doubles a flux stencil's instruction count, so the zero cases are settled
// here by their IEEE definitions and the intrinsic only sees non-zero
// operands: 0/y is a zero signed sign(x) XOR sign(y) for y != 0 and y not NaN,
// 0/0 and 0/NaN are NaN, sqrt(+-0) is +-0.  Every result equals the
// intrinsic's own.
__device__ __forceinline__ float div_rn(float x, float y) {
  const bool z = (x == 0.0f);
  const float q = __fdiv_rn(z ? 1.0f : x, y);
  const float zq = (y == 0.0f || y != y)
                       ? __int_as_float(0x7fffffff)
                       : __int_as_float((__float_as_int(x) ^ __float_as_int(y)) & 0x80000000);
  return z ? zq : q;
}
__device__ __forceinline__ double div_rn(double x, double y) {
  const bool z = (x == 0.0);
  const double q = __ddiv_rn(z ? 1.0 : x, y);
  const double zq =
      (y == 0.0 || y != y)
          ? __longlong_as_double(0x7fffffffffffffffll)
          : __longlong_as_double((__double_as_longlong(x) ^ __double_as_longlong(y)) &
                                 (long long)0x8000000000000000ull);
  return z ? zq : q;
}
__device__ __forceinline__ float sqrt_rn(float x) {
  const bool z = (x == 0.0f);
  const float r = __fsqrt_rn(z ? 1.0f : x);
  return z ? x : r;
}
__device__ __forceinline__ double sqrt_rn(double x) {
  const bool z = (x == 0.0);
  const double r = __dsqrt_rn(z ? 1.0 : x);
  return z ? x : r;
}

// Element offset of array cell (z, y, x) (internal 3-D view): pitched rows,
// or bricks of B^ndim elements (brick-major, row-major inside a brick).
template <class C>
__device__ __forceinline__ long long elem_off(const csd_grid& g, long long z, long long y,
                                              long long x) {
  if constexpr (C::BRICK_SHIFT == 0) {
    return z * g.pitch_z + y * g.pitch_y + x;
  } else {
    constexpr int S = C::BRICK_SHIFT;
    constexpr long long M = (1ll << S) - 1;
    if constexpr (C::BRICK_NDIM == 3) {
      const long long b = ((z >> S) * g.nby + (y >> S)) * g.nbx + (x >> S);
      return (b << (3 * S)) + ((z & M) << (2 * S)) + ((y & M) << S) + (x & M);
    } else if constexpr (C::BRICK_NDIM == 2) {
      const long long b = (z >> S) * g.nbx + (x >> S);
      return (b << (2 * S)) + ((z & M) << S) + (x & M);
    } else {
      return x;  // 1-D bricks are contiguous runs: the flat layout
    }
  }
}

// ---------------------------------------------------------------------------
// Chunk loaders
// ---------------------------------------------------------------------------
template <class C>
struct Loader {
  typedef typename C::T T;

  // X origins of the wrap boxes of a periodic chunk at (x0): the left halo
  // cells [hx - RX, hx) take columns [hx - RX + nx, hx + nx), the right halo
  // cells [hx + nx, hx + nx + RX) take [hx, hx + RX); each box starts at the
  // 16-byte boundary at or below its first column.
  static __device__ __forceinline__ int wrap_x(const csd_grid& g, int side) {
    const int hx = g.halo[2], nx = g.interior[2];
    const int first = side ? hx : hx - C::RX + nx;
    return (first / C::ALIGN) * C::ALIGN;
  }

  // Issue the copies of one chunk (all fields) of grid `g` into `slot`.
  static __device__ __forceinline__ void issue(const csd_grid& g, T* ring, unsigned bar, int slot,
                                               int x0, int y0, int z0) {
    if constexpr (C::LOADER == CSD_LOADER_TMA && !C::BTMA) {
      if (threadIdx.x == 0) {
        bool left = false, right = false;
        if constexpr (C::PBUF) {
          left = x0 < g.halo[2];
          right = x0 + C::BOXW > g.halo[2] + g.interior[2];
        }
        const unsigned wrap_bytes = (unsigned)(C::WRAP_ELEMS * sizeof(T) * C::NIN);
        ptx::mbar_arrive_expect_tx(bar, (unsigned)(C::CHUNK_BYTES * C::NIN) +
                                            (left ? wrap_bytes : 0u) + (right ? wrap_bytes : 0u));
#pragma unroll
        for (int f = 0; f < C::NIN; ++f) {
          T* dst = ring + (f * C::NSLOT + slot) * C::SLOT_ELEMS;
          ptx::tma_load_3d(ptx::smem_addr(dst), &g.tmap[f], x0, y0, z0, bar);
        }
        if constexpr (C::PBUF) {
          T* pbuf = ring + C::RING_ELEMS + C::INTER_ELEMS + slot * C::PBUF_SLOT;
#pragma unroll
          for (int f = 0; f < C::NIN; ++f) {
            if (left)
              ptx::tma_load_3d(ptx::smem_addr(pbuf + (f * 2 + 0) * C::WRAP_BLOCK),
                               &g.tmap_wrap[f], wrap_x(g, 0), y0, z0, bar);
            if (right)
              ptx::tma_load_3d(ptx::smem_addr(pbuf + (f * 2 + 1) * C::WRAP_BLOCK),
                               &g.tmap_wrap[f], wrap_x(g, 1), y0, z0, bar);
          }
        }
      }
    } else if constexpr (C::BTMA) {
      // Bricked fields, TMA: per field the tile's TY rows in boxes of
      // BTMA_ROWS rows (one per brick row they cover) and one single-row box
      // per halo row.  x0 is a multiple of the brick; y0 + RY = Y0 is a
      // multiple of TY, so every tile-row box lies in one brick row.
      // Coordinates below zero
      // or past the bricked extent read zeros; a row just outside the array
      // in Y may read another brick plane, but such rows only feed points
      // outside the interior, which are never stored.
      if (threadIdx.x == 0) {
        constexpr int S = C::BRICK_SHIFT, BM = C::BRICK_B - 1;
        ptx::mbar_arrive_expect_tx(bar, (unsigned)(C::CHUNK_BYTES * C::NIN));
        const int bx = x0 >> S;
        const int zi = z0 & BM, bz = z0 >> S;
        const int ym = y0 + C::RY;
#pragma unroll
        for (int f = 0; f < C::NIN; ++f) {
          T* dst = ring + (f * C::NSLOT + slot) * C::SLOT_ELEMS;
#pragma unroll
          for (int m = 0; m < C::TY / C::BTMA_ROWS; ++m) {
            const int y = ym + m * C::BTMA_ROWS;
            ptx::tma_load_5d(ptx::smem_addr(dst + (C::RY + m * C::BTMA_ROWS) * C::BOXW), &g.tmap[f],
                             0, bx, y & BM, zi, bz * g.nby + (y >> S), bar);
          }
#pragma unroll
          for (int k = 0; k < 2 * C::RY; ++k) {
            const int yy = k < C::RY ? k : C::TY + k;   // low halo rows, then high
            const int y = y0 + yy;
            ptx::tma_load_5d(ptx::smem_addr(dst + yy * C::BOXW), &g.tmap_wrap[f], 0, bx, y & BM,
                             zi, bz * g.nby + (y >> S), bar);
          }
        }
      }
    } else if constexpr (C::BRICK_SHIFT > 0) {
      // Bricked fields: every 16-byte group of a box row (X aligned to the
      // group, bricks at least one group wide) is contiguous in its brick
      // row, so it moves as one 16-byte copy; groups past the array's X end
      // are zero-filled in part or whole.
      constexpr int G = C::ALIGN;
      constexpr int GW = C::BOXW / G;
      constexpr int NG = C::ROWS * C::BOXH * GW;
      static_assert((1 << C::BRICK_SHIFT) >= G, "bricks narrower than a 16-byte group");
      const long long NZ = g.dims[0], NY = g.dims[1], NX = g.dims[2];
#pragma unroll 1
      for (int e = threadIdx.x; e < NG; e += C::NT) {
        const int xx = (e % GW) * G;
        const int t = e / GW;
        const int yy = t % C::BOXH;
        const int rr = t / C::BOXH;
        const long long gx = (long long)x0 + xx, gy = (long long)y0 + yy, gz = (long long)z0 + rr;
        const bool row_ok = gy >= 0 && gy < NY && gz >= 0 && gz < NZ && gx >= 0;
        long long n = row_ok ? NX - gx : 0;
        n = n < 0 ? 0 : (n > G ? G : n);
        const long long off = n > 0 ? elem_off<C>(g, gz, gy, gx) : 0;
#pragma unroll
        for (int f = 0; f < C::NIN; ++f) {
          T* dst = ring + (f * C::NSLOT + slot) * C::SLOT_ELEMS + e * G;
          const T* src = reinterpret_cast<const T*>(g.in[f]) + off;
          ptx::cp_async_16_partial(ptx::smem_addr(dst), src, (int)(n * (long long)sizeof(T)));
        }
      }
      ptx::cp_async_arrive(bar);
    } else {
      constexpr int N = C::ROWS * C::BOXH * C::BOXW;
      const long long NZ = g.dims[0], NY = g.dims[1], NX = g.dims[2];
#pragma unroll 1
      for (int e = threadIdx.x; e < N; e += C::NT) {
        const int xx = e % C::BOXW;
        const int t = e / C::BOXW;
        const int yy = t % C::BOXH;
        const int rr = t / C::BOXH;
        const long long gx = (long long)x0 + xx, gy = (long long)y0 + yy, gz = (long long)z0 + rr;
        const bool ok = gx >= 0 && gx < NX && gy >= 0 && gy < NY && gz >= 0 && gz < NZ;
        const long long off = ok ? elem_off<C>(g, gz, gy, gx) : 0;
#pragma unroll
        for (int f = 0; f < C::NIN; ++f) {
          T* dst = ring + (f * C::NSLOT + slot) * C::SLOT_ELEMS + e;
          const T* src = reinterpret_cast<const T*>(g.in[f]) + off;
          ptx::cp_async_zfill<sizeof(T)>(ptx::smem_addr(dst), src, ok);
        }
      }
      ptx::cp_async_arrive(bar);
    }
  }
};

// Overwrite the cells of a freshly landed chunk that lie outside the domain
// interior, but within the stencil radius of it, with their boundary-
// condition values (fused boundary fill).  `bc_odd[f]` bit d: a value
// mirrored across a boundary of dim d changes sign (a wall's normal
// momentum); the sign is the product over mirrored dims.  One warp per chunk
// line (Z row, Y row): lines outside the interior in Z or Y take their cells
// from the mirrored line in global memory; the X-halo cells of interior
// lines come from the same line in shared memory (Neumann, reflecting), the
// prefetched wrap buffer (periodic, TMA loader) or global memory (periodic,
// cp.async loader).
template <class C>
__device__ __forceinline__ bool odd_flip(const csd_grid& g, int f, bool out_x, bool out_y,
                                         bool out_z) {
  const int odd = g.bc_odd[f];
  if (g.ndim == 3) return ((odd & 1) && out_z) ^ ((odd & 2) && out_y) ^ ((odd & 4) && out_x);
  if (g.ndim == 2) return ((odd & 1) && out_z) ^ ((odd & 2) && out_x);
  return (odd & 1) && out_x;
}

template <class C>
__device__ __forceinline__ void patch_cell(const csd_grid& g, typename C::T* ring, int slot, int e,
                                           long long gx, long long gy, long long gz, bool out_y,
                                           bool out_z) {
  typedef typename C::T T;
  const int hz = g.halo[0], hy = g.halo[1], hx = g.halo[2];
  const int nz = g.interior[0], ny = g.interior[1], nx = g.interior[2];
  const bool out_x = (gx < hx || gx >= hx + nx) && g.dims[2] > 1;
  // every field's value is loaded before the first store (see patch_line)
  T v[C::NIN];
  if (C::BC == CSD_BC_DIRICHLET) {
#pragma unroll
    for (int f = 0; f < C::NIN; ++f) v[f] = (T)g.bc_value;
  } else {
    const long long mx = out_x ? bc_map(gx, hx, nx, C::BC) : gx;
    const long long my = out_y ? bc_map(gy, hy, ny, C::BC) : gy;
    const long long mz = out_z ? bc_map(gz, hz, nz, C::BC) : gz;
    const long long off = elem_off<C>(g, mz, my, mx);
#pragma unroll
    for (int f = 0; f < C::NIN; ++f) {
      v[f] = __ldg(reinterpret_cast<const T*>(g.in[f]) + off);
      if (C::BC == CSD_BC_REFLECTING && odd_flip<C>(g, f, out_x, out_y, out_z)) v[f] = -v[f];
    }
  }
#pragma unroll
  for (int f = 0; f < C::NIN; ++f) ring[(f * C::NSLOT + slot) * C::SLOT_ELEMS + e] = v[f];
}

// A whole line outside the interior in Z or Y, from global memory.  Per
// field, each lane issues all of its loads before any store: the stores go
// to shared memory through a generic pointer that the compiler cannot tell
// apart from the loads' global memory, so interleaved loads and stores would
// pay the global latency once per cell.
template <class C>
__device__ __forceinline__ void patch_line(const csd_grid& g, typename C::T* ring, int slot,
                                           int line, int x0, int xa, int xb, long long gy,
                                           long long gz, bool out_y, bool out_z, int lane) {
  typedef typename C::T T;
  constexpr int MAXC = (C::BOXW + 31) / 32;
  const int hz = g.halo[0], hy = g.halo[1], hx = g.halo[2];
  const int nz = g.interior[0], ny = g.interior[1], nx = g.interior[2];
  const long long my = out_y ? bc_map(gy, hy, ny, C::BC) : gy;
  const long long mz = out_z ? bc_map(gz, hz, nz, C::BC) : gz;
#pragma unroll
  for (int f = 0; f < C::NIN; ++f) {
    T v[MAXC];
    T* dst = ring + (f * C::NSLOT + slot) * C::SLOT_ELEMS + line * C::BOXW;
#pragma unroll
    for (int c = 0; c < MAXC; ++c) {
      const int xx = xa + lane + 32 * c;
      v[c] = T(0);
      if (xx < xb) {
        const long long gx = (long long)x0 + xx;
        const bool out_x = (gx < hx || gx >= hx + nx) && g.dims[2] > 1;
        if (C::BC == CSD_BC_DIRICHLET) {
          v[c] = (T)g.bc_value;
        } else {
          const long long mx = out_x ? bc_map(gx, hx, nx, C::BC) : gx;
          v[c] = __ldg(reinterpret_cast<const T*>(g.in[f]) + elem_off<C>(g, mz, my, mx));
          if (C::BC == CSD_BC_REFLECTING && odd_flip<C>(g, f, out_x, out_y, out_z)) v[c] = -v[c];
        }
      }
    }
#pragma unroll
    for (int c = 0; c < MAXC; ++c) {
      const int xx = xa + lane + 32 * c;
      if (xx < xb) dst[xx] = v[c];
    }
  }
}

// X-halo cell `xx` (box column) of an interior line: the value from shared
// memory (same line, wrap buffer) where the condition allows.
template <class C>
__device__ __forceinline__ void patch_x_cell(const csd_grid& g, typename C::T* ring, int slot,
                                             int line, int xx, int x0, long long gy,
                                             long long gz, int side) {
  typedef typename C::T T;
  const int hx = g.halo[2], nx = g.interior[2];
  const long long gx = (long long)x0 + xx;
  if (C::BC == CSD_BC_DIRICHLET || (C::BC == CSD_BC_PERIODIC && !C::PBUF)) {
    patch_cell<C>(g, ring, slot, line * C::BOXW + xx, gx, gy, gz, false, false);
    return;
  }
  const T* pbuf = ring + C::RING_ELEMS + C::INTER_ELEMS + slot * C::PBUF_SLOT;
  const long long src = bc_map(gx, hx, nx, C::BC);
  const int sx = (int)(src - x0);  // source box column (same line)
  // periodic: column of the source in its wrap block
  const int wx = C::PBUF ? (int)(src - Loader<C>::wrap_x(g, side)) : 0;
  // sources of all fields first, then the stores (see patch_line)
  T v[C::NIN];
#pragma unroll
  for (int f = 0; f < C::NIN; ++f) {
    const T* slot_base = ring + (f * C::NSLOT + slot) * C::SLOT_ELEMS;
    if (C::BC == CSD_BC_PERIODIC) {
      v[f] = pbuf[(f * 2 + side) * C::WRAP_BLOCK + line * C::WRAPW + wx];
    } else {
      v[f] = slot_base[line * C::BOXW + sx];
      if (C::BC == CSD_BC_REFLECTING && odd_flip<C>(g, f, true, false, false)) v[f] = -v[f];
    }
  }
#pragma unroll
  for (int f = 0; f < C::NIN; ++f)
    ring[(f * C::NSLOT + slot) * C::SLOT_ELEMS + line * C::BOXW + xx] = v[f];
}

template <class C>
__device__ __forceinline__ void patch_boundary(const csd_grid& g, typename C::T* ring, int slot,
                                               int x0, int y0, int z0) {
  const int hz = g.halo[0], hy = g.halo[1], hx = g.halo[2];
  const int nz = g.interior[0], ny = g.interior[1], nx = g.interior[2];
  const bool edge = x0 < hx || x0 + C::BOXW > hx + nx || y0 < hy || y0 + C::BOXH > hy + ny ||
                    z0 < hz || z0 + C::ROWS > hz + nz;
  if (!edge) return;
  constexpr int NW = C::NT / 32;
  const int lane = threadIdx.x & 31;
  // cells an interior point can read: the interior grown by the radius,
  // clipped to the array
  const long long xlo = max((long long)hx - C::RX, 0ll);
  const long long xhi = min((long long)hx + nx + C::RX, g.dims[2]);
  const long long ylo = max((long long)hy - C::RY, 0ll);
  const long long yhi = min((long long)hy + ny + C::RY, g.dims[1]);
  const long long zlo = max((long long)hz - C::RZ, 0ll);
  const long long zhi = min((long long)hz + nz + C::RZ, g.dims[0]);
  const int xa = (int)max(xlo - x0, 0ll);
  const int xb = (int)min(xhi - x0, (long long)C::BOXW);
  // interior lines with X-halo cells read from shared memory must see the
  // landed chunk only (sources are interior cells, never patched)
  for (int line = threadIdx.x >> 5; line < C::PLINES; line += NW) {
    const int yy = line % C::BOXH;
    const int rr = line / C::BOXH;
    const long long gy = (long long)y0 + yy, gz = (long long)z0 + rr;
    if (gy < ylo || gy >= yhi || gz < zlo || gz >= zhi) continue;
    const bool out_y = (gy < hy || gy >= hy + ny) && g.dims[1] > 1;
    const bool out_z = (gz < hz || gz >= hz + nz) && g.dims[0] > 1;
    if (out_y || out_z) {
      patch_line<C>(g, ring, slot, line, x0, xa, xb, gy, gz, out_y, out_z, lane);
    } else {
      // left: [xa, hx - x0), right: [hx + nx - x0, xb)
      const int l1 = min(xb, hx - x0);
      for (int xx = xa + lane; xx < l1; xx += 32)
        patch_x_cell<C>(g, ring, slot, line, xx, x0, gy, gz, 0);
      for (int xx = max(xa, hx + nx - x0) + lane; xx < xb; xx += 32)
        patch_x_cell<C>(g, ring, slot, line, xx, x0, gy, gz, 1);
    }
  }
  // The slot is refilled by TMA (async proxy) only after a block barrier and
  // the issuing thread's proxy fence (the refill path), which orders these
  // generic writes before it.
}

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  // non-negative doubles order like their bit patterns (NaN above +inf)
  atomicMax(reinterpret_cast<unsigned long long*>(addr),
            (unsigned long long)__double_as_longlong(v));
}

// Grid of global work item `item` in a batch: binary search of the items
// prefix; `local` receives the item's index within its grid.
__device__ __forceinline__ int batch_grid_of(const csd_params& p, int item, int& local) {
  int lo = 0, hi = p.ngrids - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (p.item_start[mid] <= item) lo = mid;
    else hi = mid - 1;
  }
  local = item - p.item_start[lo];
  return p.grid_index ? p.grid_index[lo] : lo;
}

// ---------------------------------------------------------------------------
// The engine
// ---------------------------------------------------------------------------
template <class C, class Body, bool BATCHED>
__device__ __forceinline__ void engine_items(const csd_params& p, typename C::T* ring,
                                             typename C::T* inter, unsigned long long* bars,
                                             int& abort_flag, double* red_warp);

// Single-grid launches read the descriptor from the kernel parameters
// (constant bank operands); batched launches from the device work list.
template <class C, class Body>
__device__ __forceinline__ void stream_engine(const csd_params& p) {
  typedef typename C::T T;
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  // TMA destinations must be 128-byte aligned: align the base explicitly
  unsigned char* smem_raw = smem_dyn + ((128u - (ptx::smem_addr(smem_dyn) & 127u)) & 127u);
  T* ring = reinterpret_cast<T*>(smem_raw);
  T* inter = ring + C::RING_ELEMS;
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem_raw + C::BAR_OFFSET);
  __shared__ int abort_flag;
  __shared__ double red_warp[32];

  if (threadIdx.x == 0) {
    abort_flag = 0;
#pragma unroll 1
    for (int s = 0; s < C::NSLOT; ++s)
      ptx::mbar_init(ptx::smem_addr(&bars[s]),
                     C::LOADER == CSD_LOADER_TMA ? 1u : (unsigned)C::NT);
    ptx::fence_mbar_init();
  }
  // Zero the intermediate rings once: rows/columns a stage never writes are
  // read only by points whose results are discarded, but must not hold NaN
  // garbage that could be mistaken for data by a debugging reader.
  for (int e = threadIdx.x; e < C::INTER_ELEMS; e += C::NT) inter[e] = T(0);
  __syncthreads();
  if (p.grids == nullptr)
    engine_items<C, Body, false>(p, ring, inter, bars, abort_flag, red_warp);
  else
    engine_items<C, Body, true>(p, ring, inter, bars, abort_flag, red_warp);
}

template <class C, class Body, bool BATCHED>
__device__ __forceinline__ void engine_items(const csd_params& p, typename C::T* ring,
                                             typename C::T* inter, unsigned long long* bars,
                                             int& abort_flag, double* red_warp) {
  typedef typename C::T T;
  constexpr int T_ = C::TEMPORAL;
  constexpr int HCT = C::HC * T_;  // input halo chunks per side for the whole chain
  // units per thread up to which a stage unrolls its unit loop (the body's
  // choice: small bodies gain, wide ones would keep several units' strips live)
#ifdef CSD_UNROLL_UNITS
  constexpr int UNR = CSD_UNROLL_UNITS;
#else
  constexpr int UNR = Body::UNROLL;
#endif
  unsigned seq = 0;                // chunks consumed by this CTA so far
  const int total = BATCHED ? p.total_items : p.g.items;

  for (int gitem = blockIdx.x; gitem < total; gitem += gridDim.x) {
    int item = gitem;
    const csd_grid& g = BATCHED ? p.grids[batch_grid_of(p, gitem, item)] : p.g;
    const int hz = g.halo[0], hy = g.halo[1], hx = g.halo[2];
    const int nz = g.interior[0], ny = g.interior[1], nx = g.interior[2];
    int tx, ty, z0, nrows;
    csd_item_place(&g, item, &tx, &ty, &z0, &nrows);
    const int X0 = g.xbase + tx * C::TX;  // array column of the tile's first point
    const int Y0 = g.ybase + ty * C::TY;
    const int nsteps = cdiv(nrows, C::ROWS);
    const int nchunks = nsteps + 2 * HCT;
    // array coordinates of input chunk 0
    const int cx = X0 - C::PADL;
    const int cy = Y0 - T_ * C::RY;
    const int cz = hz + z0 - HCT * C::ROWS;
    double red_acc = 0.0;
    // output addressing, read once per item (a batch's descriptor is in
    // global memory and would be re-read after every store otherwise)
    const long long pitch_y = g.pitch_y, pitch_z = g.pitch_z;
    const bool vec_store = g.vec_store != 0;
    T* outp[C::NOUT];
#pragma unroll
    for (int f = 0; f < C::NOUT; ++f) outp[f] = reinterpret_cast<T*>(g.out[f]);

    // failure-test hook: the first item of CTA 0 never requests input chunk
    // `hold`, so the wait for it runs out (csd_launch_opts::withhold_chunk)
    const int hold = (p.withhold > 0 && blockIdx.x == 0 && gitem == (int)blockIdx.x) ? p.withhold - 1 : -1;

    // prologue: fill the ring
    const int pre = min(nchunks, C::NSLOT);
    int issued = pre;   // chunks [0, issued) have been issued
    int waited = 0;     // chunks [0, waited) have landed
    for (int k = 0; k < pre; ++k) {
      const unsigned gq = seq + k;
      const int slot = gq % C::NSLOT;
      if (k != hold)
        Loader<C>::issue(g, ring, ptx::smem_addr(&bars[slot]), slot, cx, cy, cz + k * C::ROWS);
    }

    // ring steps: one per input chunk, then T-1 more that drain the chain
    for (int i = 0; i < nchunks + (C::SKEW ? T_ - 1 : 0); ++i) {
      // wait for input chunk i
      if (i < nchunks) {
        const unsigned gq = seq + i;
        const int slot = gq % C::NSLOT;
        const unsigned parity = (gq / C::NSLOT) & 1u;
        if (!ptx::mbar_wait(ptx::smem_addr(&bars[slot]), parity, p.timeout_ns)) {
          abort_flag = 1;
          if (p.err) atomicExch(p.err, CSD_ERR_TIMEOUT);
        }
        waited = i;
        if constexpr (C::BC != CSD_BC_NONE) {
          // Every thread has seen the chunk land (its own wait), the slot's
          // previous readers finished before the refill was issued, and the
          // patch reads only landed interior cells: no barrier is needed
          // before it.  After a timed-out wait the patch still touches only
          // in-bounds memory and the block leaves at the barrier below.
          patch_boundary<C>(g, ring, slot, cx, cy, cz + i * C::ROWS);
        }
      }
      // Each thread has waited for chunk i itself, so a barrier is needed
      // here only when the boundary patch wrote into the chunk (other threads
      // read those cells): refills are ordered by the barrier that ends every
      // step, and chained stages read only what earlier steps (or, without
      // the skewed schedule, the barrier between stages) completed.  Without
      // it a failed wait is acted on at the end-of-step barrier (the step's
      // results are discarded with the launch's).
      // Measured on 512^3: chains gain without it (FP64 T=2 351 -> 356, 8 x
      // 128 tiles 359 -> 366 GPts/s); single-step kernels keep it (box27 266
      // with it, 262 without; the 7-point sweeps equal).
      constexpr bool kTopBarrier = C::BC != CSD_BC_NONE || T_ == 1;
      if constexpr (kTopBarrier) {
        __syncthreads();
        if (abort_flag) break;
      }

      // stages 1..T: stage s computes chunk k_s = i - STAGE_OFF(s) of its
      // field; stage 1 reads input chunks up to i (landed above), stage
      // s > 1 reads field s-1 up to chunk k_s + HC = i - STAGE_OFF(s-1) - 1,
      // finished at an earlier step, so the stages need no barrier between
      // them
#pragma unroll
      for (int s = 1; s <= T_; ++s) {
        const int k = i - C::STAGE_OFF(s);   // chunk index in the common chunk grid
        const int klo = s * C::HC;     // first chunk of field s that is needed
        const int khi = nsteps + (2 * T_ - s) * C::HC;  // one past the last
        if (k < klo || k >= khi) continue;
        // source: field s-1, chunks k-HC .. k+HC
        TileView<C> src;
        const int c0 = k - C::HC;  // first source chunk
        if (s == 1) {
#pragma unroll
          for (int f = 0; f < C::NIN; ++f) src.base[f] = ring + f * C::NSLOT * C::SLOT_ELEMS;
          src.slot0 = (int)((seq + (unsigned)c0) % C::NSLOT);
          src.nslot = C::NSLOT;
          src.slot_elems = C::SLOT_ELEMS;
        } else {
#pragma unroll
          for (int f = 0; f < C::NIN; ++f)
            src.base[f] = inter + C::inter_elems_upto(s - 1) + f * C::NSLOT_I * C::ISLOT_ELEMS(s - 1);
          src.slot0 = c0 % C::NSLOT_I;
          src.nslot = C::NSLOT_I;
          src.slot_elems = C::ISLOT_ELEMS(s - 1);
        }
        src.height = C::H(s - 1);
        src.y_off = C::RY;  // source buffer has RY more rows on each side
        src.scal = g.scalars;
        src.dyn = g.dyn;
        const int hs = C::H(s);
        // destination geometry
        const bool last = (s == T_);
        int xv_lo, xv_hi;
        if (last) {
          xv_lo = C::PADL / C::VEC;
          xv_hi = (C::PADL + C::TX) / C::VEC;
        } else {
          xv_lo = fdiv(C::PADL - (T_ - s) * C::RX, C::VEC);
          xv_hi = cdiv(C::PADL + C::TX + (T_ - s) * C::RX, C::VEC);
        }
        const int nxv = xv_hi - xv_lo;
        const int hsu = hs / C::RPY;  // units per chunk row along Y
        const int units = C::ROWS * hsu * nxv;
        // Z row (interior index) of this chunk's first row for field s
        const int zrow0 = z0 + (k - HCT) * C::ROWS;
        const int ybuf0 = Y0 - (T_ - s) * C::RY;  // array row of dst buffer row 0
        T* dst = last ? nullptr
                      : inter + C::inter_elems_upto(s) + (k % C::NSLOT_I) * C::ISLOT_ELEMS(s);
        auto unit = [&](const int u) {
          const int xv = xv_lo + u % nxv;
          const int t2 = u / nxv;
          const int y = (t2 % hsu) * C::RPY;
          const int r = t2 / hsu;
          OutPack<T, C::NOUT, C::VEC * C::RPY> o;
          Body::template compute<C>(src, r, y, xv * C::VEC, o);
          const int gz = hz + zrow0 + r;                 // array coordinates
          const int gx0 = X0 - C::PADL + xv * C::VEC;
          const bool zin = zrow0 + r >= 0 && zrow0 + r < nz;
#pragma unroll
          for (int j = 0; j < C::RPY; ++j) {
            const int gy = ybuf0 + y + j;
            const bool yin = gy >= hy && gy < hy + ny;
            const T* ov[C::NOUT];
#pragma unroll
            for (int f = 0; f < C::NOUT; ++f) ov[f] = o.v[f] + j * C::VEC;
            if (last) {
              if (!(zin && yin && (zrow0 + r) < z0 + nrows)) continue;
              if constexpr (C::REDUCE) {
#pragma unroll
                for (int e = 0; e < C::VEC; ++e) {
                  const int gx = gx0 + e;
                  if (gx >= hx && gx < hx + nx) {
                    const double v = (double)ov[0][e];
                    red_acc = (v != v || v > red_acc) ? v : red_acc;
                  }
                }
                continue;
              }
              const bool full = gx0 >= hx && gx0 + C::VEC <= hx + nx;
              if constexpr (C::BRICK_SHIFT == 0) {
                const long long rowoff = (long long)gz * pitch_z + (long long)gy * pitch_y;
#pragma unroll
                for (int f = 0; f < C::NOUT; ++f) {
                  T* out = outp[f] + rowoff;
                  if (full && vec_store) {
                    store_unit<C::VEC>(out + gx0, ov[f]);
                  } else {
#pragma unroll
                    for (int e = 0; e < C::VEC; ++e) {
                      const int gx = gx0 + e;
                      if (gx >= hx && gx < hx + nx) out[gx] = ov[f][e];
                    }
                  }
                }
              } else {
                // a VEC-aligned run of VEC points stays inside one brick row
                const long long off0 = elem_off<C>(g, gz, gy, gx0);
#pragma unroll
                for (int f = 0; f < C::NOUT; ++f) {
                  if (full && vec_store) {
                    store_unit<C::VEC>(outp[f] + off0, ov[f]);
                  } else {
#pragma unroll
                    for (int e = 0; e < C::VEC; ++e) {
                      const int gx = gx0 + e;
                      if (gx >= hx && gx < hx + nx) outp[f][off0 + e] = ov[f][e];
                    }
                  }
                }
              }
            } else {
              // intermediate field(s): zero outside the domain interior, as
              // the zero-halo scratch buffers of T separate launches hold;
              // a unit wholly inside stores one 16-byte vector per field
              const bool whole = zin && yin && gx0 >= hx && gx0 + C::VEC <= hx + nx;
#pragma unroll
              for (int f = 0; f < C::NOUT; ++f) {
                T* d = dst + f * C::NSLOT_I * C::ISLOT_ELEMS(s) + (r * hs + y + j) * C::BOXW +
                       xv * C::VEC;
                if (whole) {
                  store_unit<C::VEC>(d, ov[f]);
                } else {
#pragma unroll
                  for (int e = 0; e < C::VEC; ++e) {
                    const int gx = gx0 + e;
                    const bool in = zin && yin && gx >= hx && gx < hx + nx;
                    d[e] = in ? ov[f][e] : T(0);
                  }
                }
              }
            }
          }  // rows of the unit
        };
        // A short count of units per thread is unrolled, so that the units'
        // coordinates fold into per-thread constants and their loads overlap;
        // longer counts loop.
        if ((units % C::NT == 0 || CSD_UNROLL_RAGGED) && cdiv(units, C::NT) <= UNR) {
          // a ragged last round is predicated off for the threads past the end
#pragma unroll
          for (int q = 0; q < (UNR > 0 ? UNR : 1); ++q) {
            const int u = threadIdx.x + q * C::NT;
            if (q < cdiv(units, C::NT) && (units % C::NT == 0 || u < units)) unit(u);
          }
        } else {
#pragma unroll 1
          for (int u = threadIdx.x; u < units; u += C::NT) unit(u);
        }
        if constexpr (!C::SKEW) {
          if (s < T_) __syncthreads();   // stage s + 1 reads what stage s just wrote
        }
      }
      // every stage's reads of this step are done before the refill below
      // and before the next step overwrites a ring slot
      __syncthreads();
      if constexpr (!kTopBarrier) {
        if (abort_flag) break;
      }

      // refill: input chunk i - 2*HC is dead, its slot takes chunk i - 2*HC + NSLOT
      {
        const int dead = i - 2 * C::HC;
        if (dead >= 0 && dead + C::NSLOT < nchunks) {
          const int nk = dead + C::NSLOT;
          const unsigned gq = seq + nk;
          const int slot = gq % C::NSLOT;
          if (C::LOADER == CSD_LOADER_TMA && threadIdx.x == 0) ptx::fence_proxy_async_smem();
          if (nk != hold)
            Loader<C>::issue(g, ring, ptx::smem_addr(&bars[slot]), slot, cx, cy, cz + nk * C::ROWS);
          issued = nk + 1;
        }
      }
    }
    if (abort_flag) {
      // drain: every copy this CTA requested must land before it exits (the
      // copies write its shared memory).  The bound is fixed and generous,
      // independent of the caller's timeout_ns, so a short caller limit ends
      // the waits for input but never the drain; the chunk withheld by the
      // failure-test hook was never requested and is skipped.
      if (threadIdx.x == 0) {
        for (int k = waited; k < issued; ++k) {
          if (k == hold) continue;
          const unsigned gq = seq + k;
          ptx::mbar_wait(ptx::smem_addr(&bars[gq % C::NSLOT]), (gq / C::NSLOT) & 1u, kDrainNs);
        }
      }
      __syncthreads();
      return;
    }
    if constexpr (C::REDUCE) {
      // block max of the item, one atomic per block and item
      for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_down_sync(0xffffffffu, red_acc, o);
        red_acc = (w != w || w > red_acc) ? w : red_acc;
      }
      if ((threadIdx.x & 31) == 0) red_warp[threadIdx.x >> 5] = red_acc;
      __syncthreads();
      if (threadIdx.x == 0) {
        double m = red_warp[0];
        for (int w = 1; w < C::NT / 32; ++w) m = (red_warp[w] != red_warp[w] || red_warp[w] > m) ? red_warp[w] : m;
        if (g.red) atomic_max_nonneg(g.red, m);
      }
      __syncthreads();
    }
    seq += nchunks;
  }
}

}  // namespace csd

#endif  // CSD_ENGINE_CUH
