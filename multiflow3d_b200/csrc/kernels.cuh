// Device kernels of libmf3d (sm_100a): the multigrid V-cycle.
//
// Storage of a multigrid level of one block (the reference keeps it in
// `cof`, mgsolver.for:20-38): the correction phi and the right-hand side,
// each with a one-cell ghost shell, split by red/black colour.  Cell (i,j,k)
// (0-based, ghost-inclusive, 0..n+1) has colour c = (i+j+k+1)&1 - colour 0
// is the reference's even MOD(i+j+k,2) on its 1-based indices, updated first
// (mgsolver.for:552) - and lives at element
//     c*cstr + (k*(ny+2) + j)*hp + (i>>1)
// of the block's level array, hp = (nx+3)/2 rounded up to 16 bytes (the row
// pitch of a TMA tensor map).  A red-black half-sweep streams exactly one
// colour in and the other out: 12 B/cell/half-sweep in FP64.
//
// Every block owns its arrays (a resident hierarchy); a launch covers any
// set of blocks through a table of per-block descriptors, so independent
// domains of different sizes share one launch per phase.  Each descriptor
// names its domain; a domain that has converged is skipped (`act`).
//
// The 7-point coefficients are not stored per cell (the reference streams 7
// arrays, ~80 B/cell/sweep): per level and block, six 1-D arrays (aw, ae
// along x; as, an along y; ab, at along z) with the Neumann faces zeroed
// (mgsolver.for:184-203); ap = -(aw+ae+as+an+ab+at) is re-formed per cell
// in the reference's order (mgsolver.for:205-208), bit-identical to `cof`.
//
// Every FP64 expression keeps the reference's evaluation order; the file is
// built with -fmad=false so no multiply-add is contracted.
#pragma once

#include <cstdint>
#include <cuda.h>  // CUtensorMap (type only: the library does not link the driver)
#include <cuda_runtime.h>

namespace mf3d {

constexpr int kTile = 256;  // threads per CTA of the 1-D item kernels

// Per-block, per-level descriptor (device side).
struct BlkLev {
  void *phi;          // colour 0 of phi; colour 1 at +cstr elements
  void *rhs;          // colour 0 of rhs
  const void *coef;   // aw[nx+2] ae[nx+2] as[ny+2] an[ny+2] ab[nz+2] at[nz+2]
  const void *geo;    // restriction ratios rx[nx+2] ry[ny+2] rz[nz+2]
  long long cstr;     // elements per colour array (padded)
  int nx, ny, nz, hp; // interior cells (0 = block absent at this level)
  int nmask;          // Neumann faces: bit f set for f = W,E,S,N,B,T
  int dom;            // domain of the block
  const CUtensorMap *tm;  // TMA maps: phi colour 0, phi colour 1 (RB_RJ+2 rows), rhs colour 0, 1 (RB_RJ rows)
  const void *cc;     // variable density (L_LSM): per-cell aw, ae, as, an, ab, at, six arrays of
                      // the level's colour-split layout, array m at element m*2*cstr; else null
  void *tdf;          // line relaxation: the TDMA factors a, apr of each direction (k_tdma_factor); else null
};

// compact row pitch: (nx+3)/2 entries rounded up to a multiple of 16 bytes
__host__ __device__ inline int hp_of(int nx, int elem) {
  const int per = 16 / elem;
  return ((nx + 3) / 2 + per - 1) / per * per;
}
__device__ inline int colour_of(int i, int j, int k) { return (i + j + k + 1) & 1; }
__device__ inline long long cell_off(const BlkLev &B, int i, int j, int k) {
  return colour_of(i, j, k) * B.cstr + ((long long)k * (B.ny + 2) + j) * B.hp + (i >> 1);
}
template <typename T>
__device__ inline T *phi_of(const BlkLev &B) { return (T *)B.phi; }
template <typename T>
__device__ inline T *rhs_of(const BlkLev &B) { return (T *)B.rhs; }
// coefficient arrays
template <typename T>
struct Coef {
  const T *aw, *ae, *as, *an, *ab, *at;
  __device__ Coef(const BlkLev &B) {
    aw = (const T *)B.coef;
    ae = aw + (B.nx + 2);
    as = ae + (B.nx + 2);
    an = as + (B.ny + 2);
    ab = an + (B.ny + 2);
    at = ab + (B.nz + 2);
  }
};

// The six coefficients of cell (i,j,k): per cell under L_LSM (the
// reference's `cof`, mgsolver.for:120-203), else from the 1-D arrays.
template <typename T>
__device__ __forceinline__ void cell_coefs(const BlkLev &B, const Coef<T> &cf, int i, int j, int k, T &aw, T &ae,
                                           T &as, T &an, T &ab, T &at) {
  if (B.cc) {
    const T *c = (const T *)B.cc;
    const long long o = cell_off(B, i, j, k), m = 2 * B.cstr;
    aw = c[o]; ae = c[o + m]; as = c[o + 2 * m]; an = c[o + 3 * m]; ab = c[o + 4 * m]; at = c[o + 5 * m];
  } else {
    aw = cf.aw[i]; ae = cf.ae[i]; as = cf.as[j]; an = cf.an[j]; ab = cf.ab[k]; at = cf.at[k];
  }
}

// Programmatic dependent launch.  The host launches the kernels of a solve
// with programmatic stream serialisation, so a kernel's CTAs may be resident
// before the kernel it depends on has finished: they are placed as that
// kernel's CTAs retire, instead of after a full drain and a launch gap.
// Every kernel therefore begins with this wait, which returns once all
// prerequisite grids have completed and their memory operations are
// visible; nothing is read or written before it.  Without a programmatic
// predecessor it returns at once.  No kernel signals its dependents early
// (griddepcontrol.launch_dependents): the next grid launches as this one's
// CTAs exit.  Signalling right after the wait measured slower (11.0 against
// 11.4 solves/s), the waiting CTAs taking issue slots from the last wave.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// A CTA's work: block position and the origin of its tile.  2-D tiles:
// threadIdx.x runs along i (or the compact index h), threadIdx.y along j;
// k0 is the plane (or the first plane of a z-marching chunk).
struct Tile {
  int blk;
  int k0;
  int j0;
  int i0;
};

// Tile shapes (threads per CTA = TX * RJ).
// red-black z-march: 32 x RB_TY threads, RB_CR rows per thread (RB_RJ rows
// per CTA); planes per CTA chosen per level
constexpr int RB_TX = 32, RB_TY = 4, RB_CR = 4, RB_RJ = RB_TY * RB_CR;
constexpr int RW_TX = 32, RW_RJ = 8, RW_KCH = 8;    // row tiles, RW_KCH planes per CTA
constexpr int OZ_TX = 32, OZ_RJ = 8, OZ_KCH = 16;   // outer calvel/calmas z-march

// ---------------------------------------------------------------------------
// TMA and mbarrier primitives (inline PTX, sm_90+ forms; built for sm_100a).
// Every wait is bounded: a copy that has not landed after kMaxWaitNs records
// an error code for the host and the CTA returns.
// ---------------------------------------------------------------------------
constexpr unsigned long long kMaxWaitNs = 2000000000ull;  // 2 s
// ERR_WALL_LAW: a smooth-wall law did not converge; ERR_MID_BARRIER: a grid
// barrier of the middle-level launch gave up waiting
enum : int { ERR_TMA_WAIT = 1, ERR_WALL_LAW = 2, ERR_MID_BARRIER = 3 };

// Testing aid (mf3d_test_stall_copy): when nonzero, the first red-black
// half-sweep CTA that sees it takes it (atomically, so exactly one CTA) and
// declares that many more bytes on its first plane's barrier than its
// copies deliver.  That barrier's phase then never completes: the bounded
// wait gives up after kMaxWaitNs, records ERR_TMA_WAIT and the CTA leaves,
// its copies long since landed.  Zero (no effect) unless a test sets it.
__device__ int g_test_extra_tx = 0;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Raise the current phase's expected transaction bytes without arriving.
__device__ __forceinline__ void mbar_add_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for phase `parity` of `bar`; false (and *err set) after kMaxWaitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int *err) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > kMaxWaitNs) {
      atomicExch(err, ERR_TMA_WAIT);
      return false;
    }
  }
}
// 3-D tiled TMA load of one box into shared memory, completing on `bar`.
// x (innermost) must be a multiple of 16 bytes / element size.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// L2 eviction priorities (createpolicy): a line loaded or stored with
// evict_last outlives evict_normal and evict_first lines in L2.
__device__ __forceinline__ uint64_t l2_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// tma_load_3d with an L2 eviction priority for the loaded lines
__device__ __forceinline__ void tma_load_3d_hint(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z,
                                                 uint64_t pol) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint [%0], "
      "[%1, {%3, %4, %5}], [%2], %6;" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z), "l"(pol)
      : "memory");
}
// a store with an L2 eviction priority
__device__ __forceinline__ void st_hint(double *p, double v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(__cvta_generic_to_global(p)), "d"(v), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void st_hint(float *p, float v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(__cvta_generic_to_global(p)), "f"(v), "l"(pol)
               : "memory");
}

// ---------------------------------------------------------------------------
// Red-black Gauss-Seidel half-sweep (mgsolver.for:547-601) of one colour over
// a set of blocks: phi = (rhs - (aw*w + ae*e + as*s + an*n + ab*b + at*t)) /
// ap, neighbours of the other colour.  Ghost cells are read as they are: the
// reference refreshes them only after the whole sweep.
// FROM_ZERO: the level was just zeroed (pp = 0 at the start of a V-cycle,
// coarse phi = 0 after mgrestr), so the other colour is read as 0 without a
// load; the result is bit-identical.
//
// Lanes run over q, the rank of a cell of this colour within its row: cell
// i = 2q + 2 - s with s = i & 1 = (colour + j + k + 1) & 1, so a row of nx
// cells keeps ceil(nx/2) lanes busy whatever its parity.  Its west and east
// neighbours (other colour) sit at compact h = q and q+1, the others and the
// rhs at h = q + 1 - s.  A column is q0..q0+31 of rows j0..j0+RB_RJ-1 of one
// block (each thread RB_CR rows RB_TY apart, which share s); a segment is a
// run of planes k0..k1 of one column.  The planes of all columns of the
// launch are laid end to end and split evenly over the CTAs the device holds
// at once, so every CTA marches the same number of planes - a CTA whose
// share crosses a column boundary runs two segments, each with its own ring
// fill - and the launch is one wave with no tail.
// Per plane one thread issues two TMA box loads - the other colour over
// compact columns q0..q0+W-1 and rows j0-1..j0+RB_RJ, the rhs over the same
// columns and rows j0..j0+RB_RJ-1 - into a ring of RB_NS stages, RB_PD
// planes ahead of the plane being computed.  Loads are numbered across the
// CTA's segments, which fixes each one's stage and mbarrier phase.  Boxes
// that reach past the array read zeros (never used).
// ---------------------------------------------------------------------------
constexpr int RB_PD = 2;          // prefetch distance in planes
constexpr int RB_KMAX = 64;       // planes per segment at most
constexpr int RB_NS = RB_PD + 2;  // stages: planes k-1 .. k+RB_PD (a power of two)
static_assert((RB_NS & (RB_NS - 1)) == 0, "RB_NS must be a power of two");

// A run of planes k0..k1 of one sweep column (block blk, compact columns
// q0.., rows j0..).
struct RbSeg {
  int blk, k0, k1, j0, q0, pad0, pad1, pad2;
};

template <typename T>
struct RbShape {
  static constexpr int W = (33 * (int)sizeof(T) + 15) / 16 * 16 / (int)sizeof(T);  // box width: 33 used
  static constexpr int OE = (RB_RJ + 2) * W, RE = RB_RJ * W;                        // elements per box
  static constexpr int OB = (OE * (int)sizeof(T) + 127) / 128 * 128;                // bytes per stage slot
  static constexpr int RBY = (RE * (int)sizeof(T) + 127) / 128 * 128;
};

// CTA c runs segments first[c] .. first[c+1]-1 of `segs`.
template <typename T, bool FROM_ZERO>
__global__ void __launch_bounds__(RB_TX *RB_TY) k_rbgs(const BlkLev *__restrict__ bl, const RbSeg *__restrict__ segs,
                                                       const int *__restrict__ first, const int *__restrict__ act,
                                                       int colour, int *__restrict__ err) {
  pdl_wait();
  using S = RbShape<T>;
  constexpr int W = S::W;
  constexpr int OB = FROM_ZERO ? 0 : S::OB;
  __shared__ __align__(128) unsigned char sbuf[RB_NS * (OB + S::RBY)];
  __shared__ __align__(8) uint64_t bar[RB_NS];
  __shared__ int abort_s;  // set when a wait gave up: every thread leaves after the next barrier
  __shared__ T sab[RB_KMAX], sat[RB_KMAX];  // z coefficients of the segment's planes
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * RB_TX + tx;
  auto slot_o = [&](int st) { return (T *)(sbuf + st * OB); };
  auto slot_r = [&](int st) { return (T *)(sbuf + RB_NS * OB + st * S::RBY); };
  // L2: the rhs is read once per half-sweep (evict first); the colour
  // written here is what the next half-sweep reads (evict last)
  const uint64_t pol_first = l2_evict_first(), pol_last = l2_evict_last();
  if (tid == 0) {
    for (int st = 0; st < RB_NS; ++st) mbar_init(&bar[st], 1);
    mbar_fence_init();
    abort_s = 0;
  }
  // loads the CTA issued in earlier segments: load n goes to stage n % RB_NS
  // and completes phase (n / RB_NS) & 1 of that stage's mbarrier
  int base = 0;
  bool hook = tid == 0;  // testing aid, looked at once per CTA
  const int s_end = first[blockIdx.x + 1];
  for (int si = first[blockIdx.x]; si < s_end; ++si) {
    const RbSeg t = segs[si];
    const BlkLev B = bl[t.blk];
    if (!act[B.dom]) continue;
    const int q0 = t.q0, q = q0 + tx;
    const int nx = B.nx, ny = B.ny, hp = B.hp;
    const long long rs = (long long)(ny + 2) * hp;  // plane stride
    T *__restrict__ M = phi_of<T>(B) + colour * B.cstr + q0;
    const CUtensorMap *mo = B.tm + (1 - colour), *mr = B.tm + 2 + colour;
    const Coef<T> cf(B);
    const int k0 = t.k0, k1 = t.k1;
    // coefficients of this lane's two cells (s = 0: i = 2q+2; s = 1: i = 2q+1)
    const int ia = min(2 * q + 2, nx + 1), ib = min(2 * q + 1, nx + 1);
    const T aw0 = cf.aw[ia], ae0 = cf.ae[ia], aw1 = cf.aw[ib], ae1 = cf.ae[ib];
    // per row: as, an and ap's first four terms (summed left to right)
    T as[RB_CR], an[RB_CR], pa0[RB_CR], pa1[RB_CR];
    int rowoff[RB_CR];  // j*hp of each row
#pragma unroll
    for (int m = 0; m < RB_CR; ++m) {
      const int j = t.j0 + ty + RB_TY * m;
      const bool jin = j <= ny;
      as[m] = jin ? cf.as[j] : (T)0;
      an[m] = jin ? cf.an[j] : (T)0;
      pa0[m] = ((aw0 + ae0) + as[m]) + an[m];
      pa1[m] = ((aw1 + ae1) + as[m]) + an[m];
      rowoff[m] = j * hp;
    }
    const int nrow = t.j0 + ty > ny ? 0 : min(RB_CR, (ny - t.j0 - ty) / RB_TY + 1);  // rows inside the block
    auto loads = [&](int kk) { return FROM_ZERO ? (kk >= k0 && kk <= k1) : (kk >= k0 - 1 && kk <= k1 + 1); };
    // the loaded planes are consecutive (k0-1 is loaded unless FROM_ZERO)
    constexpr int lead = FROM_ZERO ? 0 : 1;
    auto stage = [&](int kk) { return (base + kk - k0 + lead) & (RB_NS - 1); };
    auto parity = [&](int kk) { return (unsigned)(((base + kk - k0 + lead) / RB_NS) & 1); };
    auto issue = [&](int kk) {
      const int st = stage(kk);
      const bool wr = kk >= k0 && kk <= k1;
      const unsigned bytes =
          (FROM_ZERO ? 0u : (unsigned)(S::OE * sizeof(T))) + (wr ? (unsigned)(S::RE * sizeof(T)) : 0u);
      mbar_expect_tx(&bar[st], bytes);
      if (!FROM_ZERO) tma_load_3d(slot_o(st), mo, &bar[st], q0, t.j0 - 1, kk);
      if (wr) tma_load_3d_hint(slot_r(st), mr, &bar[st], q0, t.j0, kk, pol_first);
    };
    for (int z = tid; z <= k1 - k0; z += RB_TX * RB_TY) {
      sab[z] = cf.ab[k0 + z];
      sat[z] = cf.at[k0 + z];
    }
    __syncthreads();  // the barriers' init; the previous segment's readers of sab/sat and of the ring are done
    if (tid == 0) {
      if (hook && *(volatile int *)&g_test_extra_tx) {
        const unsigned extra = (unsigned)atomicExch(&g_test_extra_tx, 0);
        if (extra) mbar_add_tx(&bar[stage(FROM_ZERO ? k0 : k0 - 1)], extra);
      }
      hook = false;
      for (int kk = k0 - 1; kk < k0 + RB_PD; ++kk)
        if (loads(kk)) issue(kk);
    }
    bool ok = true;
    if (loads(k0 - 1)) ok = mbar_wait(&bar[stage(k0 - 1)], parity(k0 - 1), err);
    if (ok) ok = mbar_wait(&bar[stage(k0)], parity(k0), err);
    for (int k = k0; k <= k1; ++k) {
      if (tid == 0 && ok && loads(k + RB_PD)) issue(k + RB_PD);  // refills the slot of plane k-2
      if (ok && !FROM_ZERO) ok = mbar_wait(&bar[stage(k + 1)], parity(k + 1), err);
      if (ok && FROM_ZERO && k > k0) ok = mbar_wait(&bar[stage(k)], parity(k), err);
      const int s = (colour + t.j0 + ty + k + 1) & 1;  // the same for all rows of the thread
      const int i = 2 * q + 2 - s;
      if (ok && i <= nx) {
        const int st = stage(k), hc = tx + 1 - s;
        const T ab = sab[k - k0], at = sat[k - k0];
        const T aw = s ? aw1 : aw0, ae = s ? ae1 : ae0;
        const T *o = slot_o(st), *ob = slot_o(stage(k - 1)), *ot = slot_o(stage(k + 1));
        const T *r = slot_r(st);
        T *Mk = M + (long long)k * rs + hc;
#pragma unroll
        for (int m = 0; m < RB_CR; ++m) {
          if (m < nrow) {
            const int rr = ty + RB_TY * m;  // row within the tile
            T w = (T)0, e = (T)0, so_ = (T)0, no = (T)0, bo = (T)0, to = (T)0;
            if (!FROM_ZERO) {
              w = o[(rr + 1) * W + tx];
              e = o[(rr + 1) * W + tx + 1];
              so_ = o[rr * W + hc];
              no = o[(rr + 2) * W + hc];
              bo = ob[(rr + 1) * W + hc];
              to = ot[(rr + 1) * W + hc];
            }
            const T ap = (T)-1.0 * (((s ? pa1[m] : pa0[m]) + ab) + at);
            st_hint(Mk + rowoff[m],
                    ((r[rr * W + hc] - (aw * w + ae * e + as[m] * so_ + an[m] * no + ab * bo + at * to)) / ap),
                    pol_last);
          }
        }
      }
      if (!ok) abort_s = 1;
      __syncthreads();  // plane k-1's slot is refilled next iteration
      if (abort_s) return;
    }
    base += (k1 - k0 + 1) + (FROM_ZERO ? 0 : 2);
  }
}

// ---------------------------------------------------------------------------
// The same half-sweep for small levels (their arrays sit in L2): one thread
// per item (q, j, k) of a flat list over the blocks, operands loaded
// directly - no staging pipeline whose fill would dominate a launch of a few
// thousand cells.  Arithmetic and order as in k_rbgs.  pre[b] = first item
// of block b (ceil(nx/2)*ny*nz items per block).
// ---------------------------------------------------------------------------
template <typename T, bool FROM_ZERO>
__global__ void __launch_bounds__(kTile) k_rbgs_small(const BlkLev *__restrict__ bl, const int *__restrict__ pre,
                                                      const int *__restrict__ blocks, int nb,
                                                      const int *__restrict__ act, int colour) {
  pdl_wait();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= pre[nb]) return;
  int lo = 0, hi = nb - 1;  // last list entry whose first item <= t
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  const BlkLev &B = bl[blocks[lo]];
  if (!act[B.dom]) return;
  const int Q = (B.nx + 1) / 2;
  int r = t - pre[lo];
  const int q = r % Q;
  r /= Q;
  const int j = r % B.ny + 1, k = r / B.ny + 1;
  const int s = (colour + j + k + 1) & 1;
  const int i = 2 * q + 2 - s;
  if (i > B.nx) return;
  const Coef<T> cf(B);
  const long long rs = (long long)(B.ny + 2) * B.hp, base = (long long)k * rs + (long long)j * B.hp;
  const int h = q + 1 - s;
  const T *O = phi_of<T>(B) + (1 - colour) * B.cstr;
  T *M = phi_of<T>(B) + colour * B.cstr;
  const T *R = rhs_of<T>(B) + colour * B.cstr;
  T w = (T)0, e = (T)0, so = (T)0, no = (T)0, bo = (T)0, to = (T)0;
  if (!FROM_ZERO) {
    w = O[base + q];
    e = O[base + q + 1];
    so = O[base - B.hp + h];
    no = O[base + B.hp + h];
    bo = O[base - rs + h];
    to = O[base + rs + h];
  }
  T aw, ae, as, an, ab, at;
  cell_coefs(B, cf, i, j, k, aw, ae, as, an, ab, at);
  const T ap = (T)-1.0 * (aw + ae + as + an + ab + at);
  M[base + h] = ((R[base + h] - (aw * w + ae * e + as * so + an * no + ab * bo + at * to)) / ap);
}

// All of a cluster's CTAs (one hardware barrier; release/acquire at cluster
// scope, so global stores before it are seen by the cluster after it).
// Every warp reaches it converged: a __syncthreads() comes first.
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// ---------------------------------------------------------------------------
// Lexicographic Gauss-Seidel (mgsolver.for:403-428), loop order k, i, j:
// cell (i,j,k) reads new values at i-1, j-1, k-1 and old ones at i+1, j+1,
// k+1, so every hyperplane i+j+k = const is independent and the planes run
// in order.  Each block is a cluster of `cl` CTAs (cl = 1: a plain CTA),
// CTA r owning a slice of k; per plane its threads take the slice's (j, k)
// with i = plane - j - k inside the block, and a cluster barrier closes the
// plane.  The neighbours are read through L2 (ld.global.cg): the k-1 layer
// of a slice's first plane was written by the previous CTA of the cluster.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(1024) k_lexgs(const BlkLev *__restrict__ bl, const int *__restrict__ blocks,
                                                const int *__restrict__ act, int cl) {
  pdl_wait();
  const BlkLev B = bl[blocks[blockIdx.x / cl]];
  if (!act[B.dom]) return;  // every CTA of the cluster holds the same block
  const int rank = blockIdx.x % cl;
  T *P = phi_of<T>(B);
  const T *R = rhs_of<T>(B);
  const Coef<T> cf(B);
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  const int per = (nz + cl - 1) / cl, klo = rank * per + 1, khi = min(nz, klo + per - 1);
  for (int sum = 3; sum <= nx + ny + nz; ++sum) {
    const int kb = max(klo, sum - nx - ny), ke = min(khi, sum - 2);
    for (int idx = threadIdx.x; idx < (ke - kb + 1) * ny; idx += blockDim.x) {
      const int j = idx % ny + 1, k = kb + idx / ny;
      const int i = sum - j - k;
      if (i < 1 || i > nx) continue;
      T aw, ae, as, an, ab, at;
      cell_coefs(B, cf, i, j, k, aw, ae, as, an, ab, at);
      const T ap = (T)-1.0 * (aw + ae + as + an + ab + at);
      const T w = __ldcg(P + cell_off(B, i - 1, j, k)), e = __ldcg(P + cell_off(B, i + 1, j, k));
      const T so = __ldcg(P + cell_off(B, i, j - 1, k)), no = __ldcg(P + cell_off(B, i, j + 1, k));
      const T bo = __ldcg(P + cell_off(B, i, j, k - 1)), to = __ldcg(P + cell_off(B, i, j, k + 1));
      const T r = R[cell_off(B, i, j, k)];
      P[cell_off(B, i, j, k)] = ((r - (aw * w + ae * e + as * so + an * no + ab * bo + at * to)) / ap);
    }
    __syncthreads();
    if (cl > 1) cluster_sync_all();
  }
}

// ---------------------------------------------------------------------------
// Line TDMA relaxation (mgsolver.for:430-545): Thomas solves along j-lines
// (line order k, i), then i-lines (k, j), then k-lines (i, j), each pass a
// Gauss-Seidel over lines.  A line (u, v) reads the new values of lines
// (u-1, v) and (u, v-1) and the old ones of (u+1, v) and (u, v+1), so the
// lines of one diagonal u + v = s are independent and the diagonals run in
// order.  Directions: 0 j-lines at (i=u, k=v); 1 i-lines at (j=u, k=v);
// 2 k-lines at (i=u, j=v); m runs along the line.
//
// The forward recurrence splits in two.  apr(m) = 1/(ap - lo*a(m-1)) and
// a(m) = up*apr(m) (a(0) = 0; lo/up = as/an, aw/ae, ab/at) read coefficients
// only, so k_tdma_factor forms them once per set of coefficients.  The sweep
// then runs c(m) = (rhs'(m) - lo*c(m-1))*apr(m), c(0) = the first ghost, with
// rhs' = su - (the four transverse terms in the reference's order), and
// phi(m) = c(m) - a(m)*phi(m+1) from the far ghost down - the reference's
// expressions, evaluated in its order, so the result is bit for bit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tdma_dims(const BlkLev &B, int dir, int &nu, int &nv, int &n) {
  nu = dir == 1 ? B.ny : B.nx;
  nv = dir == 2 ? B.ny : B.nz;
  n = dir == 0 ? B.ny : dir == 1 ? B.nx : B.nz;
}
__device__ __forceinline__ void tdma_cell(int dir, int u, int v, int m, int &i, int &j, int &k) {
  if (dir == 0) { i = u; j = m; k = v; }
  else if (dir == 1) { i = m; j = u; k = v; }
  else { i = u; j = v; k = m; }
}
// element of a(m) (w = 0) or apr(m) (w = 1) of line (u, v): six arrays of
// nx*ny*nz values, each line's m contiguous
__device__ __forceinline__ long long tdma_fidx(const BlkLev &B, int dir, int u, int v, int m, int w) {
  int nu, nv, n;
  tdma_dims(B, dir, nu, nv, n);
  return (2 * dir + w) * ((long long)B.nx * B.ny * B.nz) + ((long long)(v - 1) * nu + (u - 1)) * n + (m - 1);
}

// One thread per line of direction `dir`, blockIdx.y = listed block.
template <typename T>
__global__ void k_tdma_factor(const BlkLev *__restrict__ bl, const int *__restrict__ blocks, int dir) {
  pdl_wait();
  const BlkLev B = bl[blocks[blockIdx.y]];
  int nu, nv, n;
  tdma_dims(B, dir, nu, nv, n);
  const long long line = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (line >= (long long)nu * nv) return;
  const int u = (int)(line % nu) + 1, v = (int)(line / nu) + 1;
  T *A = (T *)B.tdf + tdma_fidx(B, dir, u, v, 1, 0);
  T *R = (T *)B.tdf + tdma_fidx(B, dir, u, v, 1, 1);
  const Coef<T> cf(B);
  T am = (T)0;
  for (int m = 1; m <= n; ++m) {
    int i, j, k;
    tdma_cell(dir, u, v, m, i, j, k);
    T aw, ae, as, an, ab, at;
    cell_coefs(B, cf, i, j, k, aw, ae, as, an, ab, at);
    const T ap = (T)-1.0 * (aw + ae + as + an + ab + at);
    const T lo = dir == 0 ? as : dir == 1 ? aw : ab, up = dir == 0 ? an : dir == 1 ? ae : at;
    const T apr = (T)1.0 / (ap - lo * am);
    am = up * apr;
    A[m - 1] = am;
    R[m - 1] = apr;
  }
}

constexpr int TD_THREADS = 512, TD_CH = 8;
// Asynchronous copy of one element into shared memory (cp.async, cached at L1).
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(sizeof(T)) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// One relaxation (the three passes) of every listed block.  Each block is a
// cluster of `cl` CTAs (cl = 1: a plain CTA); CTA r owns the lines with u in
// its slice of 1..nu.  Per diagonal, `gmax` of the CTA's lines at a time:
// (1) every thread issues asynchronous copies of su, the four transverse
// neighbours, a and apr of its cells (and the line ends' ghosts) into
// shared memory, all in flight at once; (2) every thread forms rhs' and lo
// of its cells there; (3) one thread per line runs the two recurrences,
// leaving the new values in shared memory; (4) every thread stores them.  A
// cluster barrier closes the diagonal.  A line reads only lines of the
// neighbouring diagonals, so the lines of one diagonal may run in any order.
// Shared memory: seven arrays of gmax lines at stride nmax+1 (odd, so the
// lanes of the recurrence hit distinct banks), then the two ghost arrays.
template <typename T>
__global__ void __launch_bounds__(TD_THREADS) k_tdma_lines(const BlkLev *__restrict__ bl, const int *__restrict__ blocks,
                                                          const int *__restrict__ act, int cl, int gmax, int nmax) {
  pdl_wait();
  extern __shared__ __align__(16) unsigned char td_smem[];
  const BlkLev B = bl[blocks[blockIdx.x / cl]];
  if (!act[B.dom]) return;  // every CTA of the cluster holds the same block
  const int rank = blockIdx.x % cl;
  const long long ld = nmax + 1, sl = (long long)gmax * ld;
  T *rs = (T *)td_smem;  // su, then rhs', then c
  T *lw = rs + sl;       // neighbour 1, then lo
  T *rp = lw + sl;       // apr
  T *aa = rp + sl;       // a
  T *x2 = aa + sl;       // neighbours 2, 3, 4
  T *x3 = x2 + sl;
  T *x4 = x3 + sl;
  T *g0 = x4 + sl;       // ghost before m = 1
  T *g1 = g0 + gmax;     // ghost after m = n
  T *P = phi_of<T>(B);
  const T *R = rhs_of<T>(B);
  const T *TF = (const T *)B.tdf;
  const long long fn = (long long)B.nx * B.ny * B.nz;
  const Coef<T> cf(B);
  for (int dir = 0; dir < 3; ++dir) {
    int nu, nv, n;
    tdma_dims(B, dir, nu, nv, n);
    const int per = (nu + cl - 1) / cl, ulo = rank * per + 1, uhi = min(nu, ulo + per - 1);
    for (int s = 2; s <= nu + nv; ++s) {
      const int u0 = max(ulo, s - nv), u1 = min(uhi, s - 1);
      for (int ga = u0; ga <= u1; ga += gmax) {
        const int gl = min(gmax, u1 - ga + 1);
        // (1) copies in flight
        for (int e = threadIdx.x; e < gl * n; e += TD_THREADS) {
          const int g = e / n, m = e - g * n + 1;
          const int u = ga + g, v = s - u;
          int i, j, k;
          tdma_cell(dir, u, v, m, i, j, k);
          const long long o = g * ld + m - 1;
          cp_async_elem(rs + o, R + cell_off(B, i, j, k));
          if (dir == 0) {  // e, w, t, b
            cp_async_elem(lw + o, P + cell_off(B, i + 1, j, k));
            cp_async_elem(x2 + o, P + cell_off(B, i - 1, j, k));
            cp_async_elem(x3 + o, P + cell_off(B, i, j, k + 1));
            cp_async_elem(x4 + o, P + cell_off(B, i, j, k - 1));
          } else if (dir == 1) {  // n, s, t, b
            cp_async_elem(lw + o, P + cell_off(B, i, j + 1, k));
            cp_async_elem(x2 + o, P + cell_off(B, i, j - 1, k));
            cp_async_elem(x3 + o, P + cell_off(B, i, j, k + 1));
            cp_async_elem(x4 + o, P + cell_off(B, i, j, k - 1));
          } else {  // n, s, e, w
            cp_async_elem(lw + o, P + cell_off(B, i, j + 1, k));
            cp_async_elem(x2 + o, P + cell_off(B, i, j - 1, k));
            cp_async_elem(x3 + o, P + cell_off(B, i + 1, j, k));
            cp_async_elem(x4 + o, P + cell_off(B, i - 1, j, k));
          }
          const long long fo = tdma_fidx(B, dir, u, v, m, 0);
          cp_async_elem(aa + o, TF + fo);
          cp_async_elem(rp + o, TF + fo + fn);
          if (m == 1) {
            int i0, j0, k0;
            tdma_cell(dir, u, v, 0, i0, j0, k0);
            cp_async_elem(g0 + g, P + cell_off(B, i0, j0, k0));
          }
          if (m == n) {
            tdma_cell(dir, u, v, n + 1, i, j, k);
            cp_async_elem(g1 + g, P + cell_off(B, i, j, k));
          }
        }
        cp_async_wait_all();
        __syncthreads();
        // (2) rhs' = (((su - c1*n1) - c2*n2) - c3*n3) - c4*n4, and lo
        for (int e = threadIdx.x; e < gl * n; e += TD_THREADS) {
          const int g = e / n, m = e - g * n + 1;
          const int u = ga + g, v = s - u;
          int i, j, k;
          tdma_cell(dir, u, v, m, i, j, k);
          T aw, ae, as, an, ab, at;
          cell_coefs(B, cf, i, j, k, aw, ae, as, an, ab, at);
          const long long o = g * ld + m - 1;
          T c1, c2, c3, c4, lo;
          if (dir == 0) { c1 = ae; c2 = aw; c3 = at; c4 = ab; lo = as; }
          else if (dir == 1) { c1 = an; c2 = as; c3 = at; c4 = ab; lo = aw; }
          else { c1 = an; c2 = as; c3 = ae; c4 = aw; lo = ab; }
          rs[o] = (((rs[o] - c1 * lw[o]) - c2 * x2[o]) - c3 * x3[o]) - c4 * x4[o];
          lw[o] = lo;
        }
        __syncthreads();
        // (3) the recurrences, TD_CH values at a time in registers so that
        // the shared-memory latency stays off the chain
        if (threadIdx.x < gl) {
          const int g = threadIdx.x, u = ga + g, v = s - u;
          T *cr = rs + g * ld;
          const T *lo = lw + g * ld, *ar = rp + g * ld, *av = aa + g * ld;
          T c = g0[g];
          for (int m0 = 0; m0 < n; m0 += TD_CH) {
            T x[TD_CH], y[TD_CH], z[TD_CH];
#pragma unroll
            for (int q = 0; q < TD_CH; ++q)
              if (m0 + q < n) { x[q] = cr[m0 + q]; y[q] = lo[m0 + q]; z[q] = ar[m0 + q]; }
#pragma unroll
            for (int q = 0; q < TD_CH; ++q)
              if (m0 + q < n) {
                c = (x[q] - y[q] * c) * z[q];
                x[q] = c;
              }
#pragma unroll
            for (int q = 0; q < TD_CH; ++q)
              if (m0 + q < n) cr[m0 + q] = x[q];
          }
          T pv = g1[g];
          for (int m1 = n; m1 > 0; m1 -= TD_CH) {  // cells m1-1 down to m1-TD_CH
            T x[TD_CH], y[TD_CH];
#pragma unroll
            for (int q = 0; q < TD_CH; ++q)
              if (m1 - 1 - q >= 0) { x[q] = cr[m1 - 1 - q]; y[q] = av[m1 - 1 - q]; }
#pragma unroll
            for (int q = 0; q < TD_CH; ++q)
              if (m1 - 1 - q >= 0) {
                pv = (x[q] - y[q] * pv);
                x[q] = pv;
              }
#pragma unroll
            for (int q = 0; q < TD_CH; ++q)
              if (m1 - 1 - q >= 0) cr[m1 - 1 - q] = x[q];
          }
        }
        __syncthreads();
        // (4) every thread stores the group's new values: the line threads
        // keep only the recurrences
        for (int e = threadIdx.x; e < gl * n; e += TD_THREADS) {
          const int g = e / n, m = e - g * n + 1;
          const int u = ga + g, v = s - u;
          int i, j, k;
          tdma_cell(dir, u, v, m, i, j, k);
          P[cell_off(B, i, j, k)] = rs[g * ld + m - 1];
        }
        __syncthreads();  // the staging arrays are reused by the next group
      }
      if (cl > 1) cluster_sync_all();
      else __syncthreads();
    }
  }
}

// The first half-sweep of a red-black relaxation from zero (mgrelax
// scheme 3 right after mgrestr, mgsolver.for:547-601): every neighbour is
// zero, so a red cell becomes rhs / ap - the from-zero sweep's expression
// (rhs - (aw*0 + ... + at*0)) / ap, bit for bit, since subtracting +0 leaves
// rhs unchanged.  The restriction writes it as it forms the coarse rhs,
// which spares the coarse level its red launch.
template <typename TC>
__device__ __forceinline__ void red_from_zero(const BlkLev &Cb, int I, int J, int K, TC rhs) {
  const Coef<TC> cf(Cb);
  TC aw, ae, as, an, ab, at;
  cell_coefs(Cb, cf, I, J, K, aw, ae, as, an, ab, at);
  const TC ap = (TC)-1.0 * (aw + ae + as + an + ab + at);
  phi_of<TC>(Cb)[cell_off(Cb, I, J, K)] = (rhs / ap);
}

// ---------------------------------------------------------------------------
// Residual + restriction (mgrestr, mgsolver.for:619-761): coarse phi := 0
// everywhere (:650-657); interior coarse rhs := 0.125 * sum over the 8
// children of s * (rhs - (aw*w + ae*e + as*s + an*n + ab*b + at*t + ap*p))
// in the reference's child order (:743-747).  s = 8*rx*ry*rz is the volume
// weight of the non-uniform-grid extension and is exactly 1.0 on a uniform
// grid.  One thread per coarse column (I, J) of the ghost-inclusive plane -
// lanes run over I, so the children (fine i = 2I-1, 2I at compact I-1, I)
// of neighbouring lanes are neighbouring elements of both colour arrays -
// marching up `kch` coarse planes.  x and y coefficients are held per thread.
// ---------------------------------------------------------------------------
template <typename TF, typename TC>
__global__ void __launch_bounds__(kTile, 2) k_restrict(const BlkLev *__restrict__ fl, const BlkLev *__restrict__ cl,
                                                      const Tile *__restrict__ tiles, const int *__restrict__ act,
                                                      int kch, int red) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const BlkLev Cb = cl[t.blk];
  if (!act[Cb.dom]) return;
  const int GX = Cb.nx + 2, GY = Cb.ny + 2;
  const int g = t.i0 + threadIdx.x;
  if (g >= GX * GY) return;
  const int J = g / GX, I = g - J * GX;
  const BlkLev Fb = fl[t.blk];
  TC *__restrict__ PC = phi_of<TC>(Cb);
  TC *__restrict__ RC = rhs_of<TC>(Cb);
  const TF *__restrict__ P = phi_of<TF>(Fb);
  const TF *__restrict__ R = rhs_of<TF>(Fb);
  const Coef<TF> cf(Fb);
  const TF *rx = (const TF *)Fb.geo, *ry = rx + (Fb.nx + 2), *rz = ry + (Fb.ny + 2);
  const bool inij = I >= 1 && I <= Cb.nx && J >= 1 && J <= Cb.ny;
  const int Ic = inij ? I : 1, Jc = inij ? J : 1;  // in-bounds indices for the per-thread loads
  TF aw[2], ae[2], sx[2], as[2], an[2], sy[2];
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    const int fi = 2 * Ic - 1 + d, fj = 2 * Jc - 1 + d;
    aw[d] = cf.aw[fi]; ae[d] = cf.ae[fi]; sx[d] = rx[fi];
    as[d] = cf.as[fj]; an[d] = cf.an[fj]; sy[d] = ry[fj];
  }
  const long long cs = Fb.cstr, rowf = Fb.hp, plf = (long long)(Fb.ny + 2) * Fb.hp;
  // fine element of (i, j, k): colour (i+j+k+1)&1, compact i>>1
  auto fo = [&](int i, int j, int k) -> long long {
    return ((i + j + k + 1) & 1) * cs + k * plf + j * rowf + (i >> 1);
  };
  const int K1 = min(t.k0 + kch - 1, Cb.nz + 1);
  for (int K = t.k0; K <= K1; ++K) {
    PC[cell_off(Cb, I, J, K)] = (TC)0;
    if (!inij || K < 1 || K > Cb.nz) continue;
    TF sum = (TF)0;  // acc0 + acc1 + ... + acc7, folded left to right as it is formed
#pragma unroll
    for (int dk = 0; dk < 2; ++dk) {
      const int fk = 2 * K - 1 + dk;
      const TF ab = cf.ab[fk], at = cf.at[fk], sz = rz[fk];
#pragma unroll
      for (int dj = 0; dj < 2; ++dj)
#pragma unroll
        for (int di = 0; di < 2; ++di) {
          const int fi = 2 * I - 1 + di, fj = 2 * J - 1 + dj;
          TF cw = aw[di], ce = ae[di], cs_ = as[dj], cn = an[dj], cb = ab, ct = at;
          if (Fb.cc) cell_coefs(Fb, cf, fi, fj, fk, cw, ce, cs_, cn, cb, ct);
          const TF ap = (TF)-1.0 * (cw + ce + cs_ + cn + cb + ct);
          const TF pw = P[fo(fi - 1, fj, fk)], pe = P[fo(fi + 1, fj, fk)];
          const TF ps = P[fo(fi, fj - 1, fk)], pn = P[fo(fi, fj + 1, fk)];
          const TF pb = P[fo(fi, fj, fk - 1)], pt = P[fo(fi, fj, fk + 1)];
          const TF pp = P[fo(fi, fj, fk)];
          const TF r = R[fo(fi, fj, fk)];
          const TF res = r - (cw * pw + ce * pe + cs_ * ps + cn * pn + cb * pb + ct * pt + ap * pp);
          const TF s = (TF)8.0 * sx[di] * sy[dj] * sz;
          const TF a = res * s;
          sum = (dk | dj | di) ? sum + a : a;
        }
    }
    const TF v = (TF)0.125 * sum;
    RC[cell_off(Cb, I, J, K)] = (TC)v;
    if (red && colour_of(I, J, K) == 0) red_from_zero(Cb, I, J, K, (TC)v);
  }
}

// ---------------------------------------------------------------------------
// The restriction with its fine operands staged by TMA (red-black smoothing
// only: the coarse level's first half-sweep starts from zero and reads no
// coarse phi, so only the coarse ghost shell has to be zeroed; the threads of
// the boundary cells zero their neighbouring ghost cells).  A CTA owns coarse cells I0..I0+31 x J0..J0+7 and marches
// up kch coarse planes.  Fine plane fp is loaded once, into a ring of
// RS_NS slots: both colours of phi over compact columns I0-1..I0-1+W and
// fine rows 2J0-2..2J0+15 (the sweep's phi boxes), and both colours of rhs
// over rows 2J0-1..2J0+14 (the sweep's rhs boxes) when fp holds children.
// Coarse plane K reads fine planes 2K-2..2K+1; the next two are in flight.
// Per coarse cell the arithmetic is k_restrict's, in its order.
// ---------------------------------------------------------------------------
constexpr int RS_NS = 6;  // fine-plane slots: 2K-2 .. 2K+3
template <typename T>
struct RsShape {
  static constexpr int W = RbShape<T>::W;
  static constexpr int PR = RB_RJ + 2, RR = RB_RJ;  // phi and rhs box rows (fine)
  static constexpr int PB = (PR * W * (int)sizeof(T) + 127) / 128 * 128;
  static constexpr int RBY = (RR * W * (int)sizeof(T) + 127) / 128 * 128;
  static constexpr int SLOT = 2 * PB + 2 * RBY;  // phi c0, phi c1, rhs c0, rhs c1
  static constexpr int SMEM = RS_NS * SLOT;
};

template <typename TF, typename TC>
__global__ void __launch_bounds__(kTile) k_restrict_tma(const BlkLev *__restrict__ fl, const BlkLev *__restrict__ cl,
                                                        const Tile *__restrict__ tiles, const int *__restrict__ act,
                                                        int kch, int *__restrict__ err, int red) {
  pdl_wait();
  using S = RsShape<TF>;
  constexpr int W = S::W;
  extern __shared__ __align__(128) unsigned char rs_smem[];
  __shared__ __align__(8) uint64_t bar[RS_NS];
  __shared__ int abort_s;
  const Tile t = tiles[blockIdx.x];
  const BlkLev Cb = cl[t.blk];
  if (!act[Cb.dom]) return;
  const BlkLev Fb = fl[t.blk];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5, tid = threadIdx.x;
  const int I0 = t.i0, J0 = t.j0, K0 = t.k0, K1 = min(t.k0 + kch - 1, Cb.nz);
  const int I = I0 + tx, J = J0 + ty;
  const bool in = I <= Cb.nx && J <= Cb.ny;
  const int Ic = in ? I : 1, Jc = in ? J : 1;
  const Coef<TF> cf(Fb);
  const TF *rx = (const TF *)Fb.geo, *ry = rx + (Fb.nx + 2), *rz = ry + (Fb.ny + 2);
  TF aw[2], ae[2], sx[2], as[2], an[2], sy[2];
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    const int fi = 2 * Ic - 1 + d, fj = 2 * Jc - 1 + d;
    aw[d] = cf.aw[fi]; ae[d] = cf.ae[fi]; sx[d] = rx[fi];
    as[d] = cf.as[fj]; an[d] = cf.an[fj]; sy[d] = ry[fj];
  }
  const int fp0 = 2 * K0 - 2, fp1 = 2 * K1 + 1;  // fine planes of the chunk
  auto slot = [&](int fp) { return rs_smem + ((fp - fp0) % RS_NS) * S::SLOT; };
  auto sidx = [&](int fp) { return (fp - fp0) % RS_NS; };
  auto parity = [&](int fp) { return (unsigned)(((fp - fp0) / RS_NS) & 1); };
  auto issue = [&](int fp) {
    const int st = sidx(fp);
    unsigned char *b = slot(fp);
    const bool kids = fp > fp0 && fp < fp1;
    const unsigned bytes = 2u * S::PR * W * sizeof(TF) + (kids ? 2u * S::RR * W * sizeof(TF) : 0u);
    mbar_expect_tx(&bar[st], bytes);
    tma_load_3d(b, Fb.tm + 0, &bar[st], I0 - 1, 2 * J0 - 2, fp);
    tma_load_3d(b + S::PB, Fb.tm + 1, &bar[st], I0 - 1, 2 * J0 - 2, fp);
    if (kids) {
      tma_load_3d(b + 2 * S::PB, Fb.tm + 2, &bar[st], I0 - 1, 2 * J0 - 1, fp);
      tma_load_3d(b + 2 * S::PB + S::RBY, Fb.tm + 3, &bar[st], I0 - 1, 2 * J0 - 1, fp);
    }
  };
  if (tid == 0) {
    for (int q = 0; q < RS_NS; ++q) mbar_init(&bar[q], 1);
    mbar_fence_init();
    abort_s = 0;
  }
  __syncthreads();
  if (tid == 0)
    for (int fp = fp0; fp < fp0 + RS_NS && fp <= fp1; ++fp) issue(fp);
  bool ok = true;
  for (int K = K0; K <= K1; ++K) {
    // planes 2K-2 .. 2K+1 (the first two were waited for at K-1, except at K0)
    for (int fp = (K == K0 ? 2 * K - 2 : 2 * K); fp <= 2 * K + 1 && ok; ++fp)
      ok = mbar_wait(&bar[sidx(fp)], parity(fp), err);
    if (ok && in) {
      TF sum = (TF)0;
#pragma unroll
      for (int dk = 0; dk < 2; ++dk) {
        const int fk = 2 * K - 1 + dk;
        const TF ab = cf.ab[fk], at = cf.at[fk], sz = rz[fk];
        const unsigned char *pc = slot(fk), *pb = slot(fk - 1), *pt = slot(fk + 1);
#pragma unroll
        for (int dj = 0; dj < 2; ++dj)
#pragma unroll
          for (int di = 0; di < 2; ++di) {
            const int fi = 2 * I - 1 + di, fj = 2 * J - 1 + dj;
            const int c = (fi + fj + fk + 1) & 1;        // colour of the child
            const int col = (fi >> 1) - (I0 - 1);
            const int row = fj - (2 * J0 - 2);            // phi box row
            const TF *Pc = (const TF *)(pc + c * S::PB);  // same colour as the child
            const TF *Po = (const TF *)(pc + (1 - c) * S::PB);
            const TF *Pb = (const TF *)(pb + (1 - c) * S::PB), *Pt = (const TF *)(pt + (1 - c) * S::PB);
            const TF *Rc = (const TF *)(pc + 2 * S::PB + c * S::RBY);
            const TF ap = (TF)-1.0 * (aw[di] + ae[di] + as[dj] + an[dj] + ab + at);
            const TF pw = Po[row * W + ((fi - 1) >> 1) - (I0 - 1)], pe = Po[row * W + ((fi + 1) >> 1) - (I0 - 1)];
            const TF ps = Po[(row - 1) * W + col], pn = Po[(row + 1) * W + col];
            const TF pbv = Pb[row * W + col], ptv = Pt[row * W + col];
            const TF pp = Pc[row * W + col];
            const TF r = Rc[(row - 1) * W + col];
            const TF res = r - (aw[di] * pw + ae[di] * pe + as[dj] * ps + an[dj] * pn + ab * pbv + at * ptv + ap * pp);
            const TF sw = (TF)8.0 * sx[di] * sy[dj] * sz;
            const TF a = res * sw;
            sum = (dk | dj | di) ? sum + a : a;
          }
      }
      const TC rv = (TC)((TF)0.125 * sum);
      rhs_of<TC>(Cb)[cell_off(Cb, I, J, K)] = rv;
      if (red && colour_of(I, J, K) == 0) red_from_zero(Cb, I, J, K, rv);
      // the coarse ghost cells next to this cell (faces, edges, corners) := 0
      const int alo = I == 1 ? -1 : 0, ahi = I == Cb.nx ? 1 : 0;
      const int blo = J == 1 ? -1 : 0, bhi = J == Cb.ny ? 1 : 0;
      const int clo = K == 1 ? -1 : 0, chi = K == Cb.nz ? 1 : 0;
      if (alo | ahi | blo | bhi | clo | chi)
        for (int c = clo; c <= chi; ++c)
          for (int b = blo; b <= bhi; ++b)
            for (int a = alo; a <= ahi; ++a)
              if (a | b | c) phi_of<TC>(Cb)[cell_off(Cb, I + a, J + b, K + c)] = (TC)0;
    }
    if (!ok) abort_s = 1;
    __syncthreads();  // planes 2K-2 and 2K-1 are free
    if (abort_s) return;
    if (tid == 0) {
      if (2 * K + 4 <= fp1) issue(2 * K + 4);
      if (2 * K + 5 <= fp1) issue(2 * K + 5);
    }
  }
}

// ---------------------------------------------------------------------------
// Prolongation + correction + Neumann ghosts (mgcorr, mgsolver.for:763-905,
// then mgbound :902).  Every fine cell, ghosts included, adds the trilinear
// (27,9,3,1)/64 interpolant of the coarse correction, summed in the
// reference's term order (:833-887); a Neumann ghost then takes the value
// of the interior cell mgbound copies into it (W,E,S,N,B,T in order
// composes to a clamp of the index).
// One thread per fine group (2I..2I+1) x (2J..2J+1) x (2K..2K+1): the group
// shares its 8 coarse cells (I..I+1, J..J+1, K..K+1), its 8 fine cells sit
// at compact index I of both colour arrays (consecutive across lanes), and
// a Neumann ghost's mirror cell is in the same group.  Threads march up
// `kch` coarse planes carrying the upper coarse plane.
// ---------------------------------------------------------------------------
template <typename TF, typename TC>
__global__ void __launch_bounds__(kTile) k_prolong(const BlkLev *__restrict__ fl, const BlkLev *__restrict__ cl,
                                                   const Tile *__restrict__ tiles, const int *__restrict__ act,
                                                   int kch) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const BlkLev Fb = fl[t.blk];
  if (!act[Fb.dom]) return;
  const BlkLev Cb = cl[t.blk];
  const int GX = Cb.nx + 1, GY = Cb.ny + 1;
  const int g = t.i0 + threadIdx.x;
  if (g >= GX * GY) return;
  const int J = g / GX, I = g - J * GX;
  const int m = Fb.nmask;
  // the member of the pair that is a Neumann ghost copies its partner
  const bool xw = I == 0 && (m & 1), xe = I == Cb.nx && (m & 2);
  const bool ys = J == 0 && (m & 4), yn = J == Cb.ny && (m & 8);
  const TC *__restrict__ PC = phi_of<TC>(Cb);
  TF *__restrict__ PF = phi_of<TF>(Fb);
  const long long csf = Fb.cstr, rowf = Fb.hp, plf = (long long)(Fb.ny + 2) * Fb.hp;
  auto coarse = [&](int a, int b, int c) -> TF { return (TF)PC[cell_off(Cb, I + a, J + b, c)]; };
  const int K1 = min(t.k0 + kch - 1, Cb.nz);
  // the group's 8 fine cells of coarse plane K (colour-split offsets)
  auto fine = [&](int K, int di, int dj, int dk) -> long long {
    return ((di + dj + dk + 1) & 1) * csf + (2 * K + dk) * plf + (2 * J + dj) * rowf + I;
  };
  TF lo[2][2], hi[2][2], f[2][2][2];  // coarse planes K, K+1; the fine cells of plane K
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      lo[a][b] = coarse(a, b, t.k0);
      hi[a][b] = coarse(a, b, t.k0 + 1);
    }
#pragma unroll
  for (int dk = 0; dk < 2; ++dk)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int di = 0; di < 2; ++di) f[dk][dj][di] = PF[fine(t.k0, di, dj, dk)];
  for (int K = t.k0; K <= K1; ++K) {
    const bool zb = K == 0 && (m & 16), zt = K == Cb.nz && (m & 32);
    TF v[2][2][2];  // [dk][dj][di]
#pragma unroll
    for (int dk = 0; dk < 2; ++dk)
#pragma unroll
      for (int dj = 0; dj < 2; ++dj)
#pragma unroll
        for (int di = 0; di < 2; ++di) {
          // weight of coarse (a,b,c): 3 along an axis where the child sits in that cell, else 1
          auto w = [&](int a, int b, int c) -> TF {
            return (TF)((a == di ? 3 : 1) * (b == dj ? 3 : 1) * (c == dk ? 3 : 1));
          };
          const TF corr = (w(0, 0, 0) * lo[0][0] + w(0, 1, 0) * lo[0][1] + w(0, 0, 1) * hi[0][0] +
                           w(0, 1, 1) * hi[0][1] + w(1, 0, 0) * lo[1][0] + w(1, 1, 0) * lo[1][1] +
                           w(1, 0, 1) * hi[1][0] + w(1, 1, 1) * hi[1][1]) *
                          (TF)0.015625;  // x/64 == x*2^-6 exactly in IEEE arithmetic
          v[dk][dj][di] = f[dk][dj][di] + corr;
        }
    // the next plane's operands load before this plane's stores (other
    // cells: plane K+1's fine cells are 2K+2, 2K+3)
    TF hn[2][2] = {{hi[0][0], hi[0][1]}, {hi[1][0], hi[1][1]}};
    if (K < K1) {
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) hn[a][b] = coarse(a, b, K + 2);
#pragma unroll
      for (int dk = 0; dk < 2; ++dk)
#pragma unroll
        for (int dj = 0; dj < 2; ++dj)
#pragma unroll
          for (int di = 0; di < 2; ++di) f[dk][dj][di] = PF[fine(K + 1, di, dj, dk)];
    }
#pragma unroll
    for (int dk = 0; dk < 2; ++dk)
#pragma unroll
      for (int dj = 0; dj < 2; ++dj)
#pragma unroll
        for (int di = 0; di < 2; ++di) {
          const int si = (di == 0 && xw) ? 1 : (di == 1 && xe) ? 0 : di;
          const int sj = (dj == 0 && ys) ? 1 : (dj == 1 && yn) ? 0 : dj;
          const int sk = (dk == 0 && zb) ? 1 : (dk == 1 && zt) ? 0 : dk;
          const long long o = ((di + dj + dk + 1) & 1) * csf + (2 * K + dk) * plf + (2 * J + dj) * rowf + I;
          // v[sk][sj][si] by selects (constant register indices)
          const TF a0 = si ? v[0][0][1] : v[0][0][0], a1 = si ? v[0][1][1] : v[0][1][0];
          const TF a2 = si ? v[1][0][1] : v[1][0][0], a3 = si ? v[1][1][1] : v[1][1][0];
          const TF b0 = sj ? a1 : a0, b1 = sj ? a3 : a2;
          PF[o] = sk ? b1 : b0;
        }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        lo[a][b] = hi[a][b];
        hi[a][b] = hn[a][b];
      }
  }
}

// ---------------------------------------------------------------------------
// Halo copies of one level: the composition of mgbound + exchangepp +
// mgbound + exchbc_mgpp as element pairs (dst block, dst offset, src block,
// src offset) against the state before the refresh.  Each domain keeps its
// pairs resident on the device (block indices local to the domain, pairs
// whose source is itself overwritten first); a view lists one segment per
// domain.  k_halo_stage reads the staged sources of every segment,
// k_halo_apply then writes every pair.  A thread finds its segment by binary
// search over the segments' first indices.
// ---------------------------------------------------------------------------
struct HaloCopy {
  int dblk, doff, sblk, soff;
};
struct HaloSeg {
  const HaloCopy *pairs;  // the domain's pairs at this level
  long long start;        // first thread index of the segment (apply)
  long long sstart;       // first thread index / stage slot of its staged pairs
  int n, nstaged;         // pairs, staged pairs
  int blk_base;           // view index of the domain's first block
  int dom;                // view domain
};
// Last segment whose key(seg) <= t (segments in increasing key order).
template <bool STAGED>
__device__ __forceinline__ int halo_segment(const HaloSeg *__restrict__ seg, int nseg, long long t) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if ((STAGED ? seg[mid].sstart : seg[mid].start) <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
template <typename T>
__global__ void k_halo_stage(const BlkLev *__restrict__ bl, const HaloSeg *__restrict__ seg, int nseg,
                             long long nstaged, const int *__restrict__ act, T *__restrict__ buf) {
  pdl_wait();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nstaged) return;
  const HaloSeg &S = seg[halo_segment<true>(seg, nseg, t)];
  if (!act[S.dom]) return;
  const HaloCopy c = S.pairs[t - S.sstart];
  buf[t] = phi_of<T>(bl[S.blk_base + c.sblk])[c.soff];
}
template <typename T>
__global__ void k_halo_apply(const BlkLev *__restrict__ bl, const HaloSeg *__restrict__ seg, int nseg, long long n,
                             const int *__restrict__ act, const T *__restrict__ buf) {
  pdl_wait();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const HaloSeg &S = seg[halo_segment<false>(seg, nseg, t)];
  if (!act[S.dom]) return;
  const long long u = t - S.start;
  const HaloCopy c = S.pairs[u];
  const T v = u < S.nstaged ? buf[S.sstart + u] : phi_of<T>(bl[S.blk_base + c.sblk])[c.soff];
  phi_of<T>(bl[S.blk_base + c.dblk])[c.doff] = v;
}

// Zero the ghost shell of a set of blocks (pp = 0 before a V-cycle): one
// thread per ghost cell, enumerated face by face (edges twice - zeros).
template <typename T>
__global__ void k_zero_ghosts(const BlkLev *__restrict__ bl, const int *__restrict__ blocks, int nblk) {
  pdl_wait();
  const int b = blockIdx.y;
  if (b >= nblk) return;
  const BlkLev B = bl[blocks[b]];
  T *P = phi_of<T>(B);
  const int W = B.nx + 2, H = B.ny + 2, D = B.nz + 2;
  const int nyz = H * D, nxz = W * D, nxy = W * H;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 2 * (nyz + nxz + nxy); q += gridDim.x * blockDim.x) {
    int i, j, k, r = q;
    if (r < 2 * nyz) { const int f = r / nyz; r -= f * nyz; i = f ? W - 1 : 0; j = r % H; k = r / H; }
    else if ((r -= 2 * nyz) < 2 * nxz) { const int f = r / nxz; r -= f * nxz; j = f ? H - 1 : 0; i = r % W; k = r / W; }
    else { r -= 2 * nxz; const int f = r / nxy; r -= f * nxy; k = f ? D - 1 : 0; i = r % W; j = r / W; }
    P[cell_off(B, i, j, k)] = (T)0;
  }
}

// ---------------------------------------------------------------------------
// Variable density (L_LSM): the coefficients `coeff` forms at the start of
// every solve (newsolv_mg.for:12-14, mgsolver.for:69-203).  FP64 only.
// ---------------------------------------------------------------------------
// Cell densities of one level of one block: interior cell (i,j,k), 1-based,
// at element off + i + sy*j + sz*k (the ttc field on level 1, an interior
// array i fastest below it).
struct DensView {
  const double *p;
  long long off, sy, sz;
  __device__ double at(int i, int j, int k) const { return p[off + i + sy * j + sz * k]; }
};

// Level g > 1 densities, interior cells i fastest: 0.125 times the sum of
// the 8 children of level g-1 in the reference's order - (j), (j+1), (i+1),
// (i+1, j+1), then the same one plane up - summed left to right
// (mgsolver.for:84-113).  One thread per coarse cell.
__global__ void k_lsm_coarsen(DensView fine, double *__restrict__ coarse, int nx, int ny, int nz) {
  pdl_wait();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nx * ny * nz) return;
  const int i = (int)(t % nx) + 1, j = (int)((t / nx) % ny) + 1, k = (int)(t / ((long long)nx * ny)) + 1;
  const int fi = 2 * i - 1, fj = 2 * j - 1, fk = 2 * k - 1;
  const double sum = fine.at(fi, fj, fk) + fine.at(fi, fj + 1, fk) + fine.at(fi + 1, fj, fk) +
                     fine.at(fi + 1, fj + 1, fk) + fine.at(fi, fj, fk + 1) + fine.at(fi, fj + 1, fk + 1) +
                     fine.at(fi + 1, fj, fk + 1) + fine.at(fi + 1, fj + 1, fk + 1);
  coarse[t] = 0.125 * sum;
}

// Per-cell coefficients of one level of one block (mgsolver.for:120-203):
// face densities from the block's own cells (a boundary cell uses its own
// density), aw = ((dy*dz)/dx)/densim12 and so on with the block's fine
// spacings on every level (cx, cy, cz formed on the host in that order),
// Neumann faces zeroed.  Written to B.cc; one thread per interior cell.
__global__ void k_lsm_coef(BlkLev B, DensView d, double cx, double cy, double cz) {
  pdl_wait();
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nx * ny * nz) return;
  const int i = (int)(t % nx) + 1, j = (int)((t / nx) % ny) + 1, k = (int)(t / ((long long)nx * ny)) + 1;
  const double dc = d.at(i, j, k);
  const double densim12 = i == 1 ? dc : 0.5 * (dc + d.at(i - 1, j, k));
  const double densip12 = i == nx ? dc : 0.5 * (dc + d.at(i + 1, j, k));
  const double densjm12 = j == 1 ? dc : 0.5 * (dc + d.at(i, j - 1, k));
  const double densjp12 = j == ny ? dc : 0.5 * (dc + d.at(i, j + 1, k));
  const double denskm12 = k == 1 ? dc : 0.5 * (dc + d.at(i, j, k - 1));
  const double denskp12 = k == nz ? dc : 0.5 * (dc + d.at(i, j, k + 1));
  double c[6] = {cx / densim12, cx / densip12, cy / densjm12, cy / densjp12, cz / denskm12, cz / denskp12};
  if ((B.nmask & 1) && i == 1) c[0] = 0.0;
  if ((B.nmask & 2) && i == nx) c[1] = 0.0;
  if ((B.nmask & 4) && j == 1) c[2] = 0.0;
  if ((B.nmask & 8) && j == ny) c[3] = 0.0;
  if ((B.nmask & 16) && k == 1) c[4] = 0.0;
  if ((B.nmask & 32) && k == nz) c[5] = 0.0;
  double *out = (double *)B.cc;
  const long long o = cell_off(B, i, j, k), m = 2 * B.cstr;
  for (int q = 0; q < 6; ++q) out[o + q * m] = c[q];
}

}  // namespace mf3d
