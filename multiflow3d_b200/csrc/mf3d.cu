// libmf3d: B200 (sm_100a) pressure-Poisson multigrid for MultiFlow3D's
// projection step.  Host engine (C++) + C ABI of include/mf3d.h.
//
// Resident storage: every block owns its multigrid hierarchy (colour-split
// phi and rhs per level, 1-D coefficient and restriction-weight arrays) and
// its face planes.  Blocks belong to domains; a domain is one projection
// problem (the reference's set of blocks) and converges on its own.  A view
// is a launchable set of blocks: per level it holds the block descriptor
// table, the tile lists and the halo-copy lists of the subsets a lock-step
// V-cycle over domains of different depths needs, the per-domain solve
// state and the CUDA graph of one outer iteration.  One view serves one
// multi-block solve (one domain), a batch (many domains) or the server's
// current mix of resident requests.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <type_traits>
#include <map>
#include <memory>
#include <atomic>
#include <mutex>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include <cudaTypedefs.h>

#include "kernels.cuh"
#include "coarse.cuh"
#include "midcycle.cuh"
#include "lmr.cuh"
#include "mf3d_internal.h"
#include "outer.cuh"

namespace mf3d {

static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }

#define CK(call)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) {                                                                       \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                               \
      return e_ == cudaErrorMemoryAllocation ? MF3D_E_OOM : MF3D_E_CUDA;                          \
    }                                                                                              \
  } while (0)

// Device memory of the library comes from a stream-ordered pool per device
// that keeps up to kPoolKeepBytes of freed memory for reuse.  Allocations
// and frees are ordered on the stream of the context making them (an
// AllocScope names it), so they neither wait for other streams' kernels -
// cudaMalloc/cudaFree may synchronise the whole device - nor go back to the
// driver for every rebuilt table.  Outside a scope, plain cudaMalloc/cudaFree.
constexpr unsigned long long kPoolKeepBytes = 8ull << 30;
static thread_local cudaStream_t g_alloc_stream = nullptr;
struct AllocScope {
  cudaStream_t prev;
  explicit AllocScope(cudaStream_t s) : prev(g_alloc_stream) { g_alloc_stream = s; }
  ~AllocScope() { g_alloc_stream = prev; }
};
static cudaMemPool_t device_pool() {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static cudaMemPool_t pools[kMaxDevices] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof props);
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
    unsigned long long keep = kPoolKeepBytes;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = pool;
  }
  return pools[dev];
}

// MF3D_POISON_ALLOC=1 fills every new device allocation with 0xFF bytes
// (a NaN in every FP64/FP32 element): a kernel that reads library memory
// nothing wrote - which a reused pool block would otherwise hand over with
// an earlier context's data - then ends in a non-finite residual instead of
// a silently different result.  A testing aid; off by default.
static bool poison_allocations() {
  const char *e = std::getenv("MF3D_POISON_ALLOC");
  return e && e[0] && e[0] != '0';
}

// Testing aid (mf3d_test_fail_alloc): the allocation that brings this
// countdown from 0 to -1 fails as if the device were out of memory; -1 = off.
static std::atomic<long long> g_fail_alloc_countdown{-1};
static bool injected_alloc_failure() {
  long long c = g_fail_alloc_countdown.load();
  while (c >= 0 && !g_fail_alloc_countdown.compare_exchange_weak(c, c - 1)) {
  }
  return c == 0;
}

// A device array.  alloc() keeps the current allocation when it is large
// enough (rebuilt launch tables reuse their buffers).
template <typename T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  size_t cap = 0;
  cudaStream_t s_alloc = nullptr;  // stream the allocation is ordered on (null: cudaMalloc)
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n), cap(o.cap), s_alloc(o.s_alloc) {
    o.p = nullptr; o.n = 0; o.cap = 0;
  }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) {
      release();
      p = o.p; n = o.n; cap = o.cap; s_alloc = o.s_alloc;
      o.p = nullptr; o.n = 0; o.cap = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (!p) return;
    if (s_alloc) cudaFreeAsync(p, s_alloc);
    else cudaFree(p);
    p = nullptr;
    n = cap = 0;
  }
  int alloc(size_t count) {
    if (p && count <= cap) {
      n = count;
      return MF3D_OK;
    }
    release();
    if (count == 0) return MF3D_OK;
    if (injected_alloc_failure()) {
      set_error("device allocation: out of memory (injected by mf3d_test_fail_alloc)");
      return MF3D_E_OOM;
    }
    cudaError_t e;
    cudaMemPool_t pool = g_alloc_stream ? device_pool() : nullptr;
    if (pool) {
      e = cudaMallocFromPoolAsync((void **)&p, count * sizeof(T), pool, g_alloc_stream);
      s_alloc = g_alloc_stream;
    } else {
      e = cudaMalloc(&p, count * sizeof(T));
      s_alloc = nullptr;
    }
    if (e != cudaSuccess) {
      p = nullptr;
      set_error(std::string("device allocation: ") + cudaGetErrorString(e));
      return e == cudaErrorMemoryAllocation ? MF3D_E_OOM : MF3D_E_CUDA;
    }
    n = cap = count;
    if (poison_allocations()) {
      e = s_alloc ? cudaMemsetAsync(p, 0xFF, count * sizeof(T), s_alloc) : cudaMemset(p, 0xFF, count * sizeof(T));
      if (e != cudaSuccess) {
        set_error(std::string("poisoning an allocation: ") + cudaGetErrorString(e));
        return MF3D_E_CUDA;
      }
    }
    return MF3D_OK;
  }
  int upload(const std::vector<T> &h, cudaStream_t s) {
    int st = alloc(h.size());
    if (st) return st;
    if (!h.empty()) CK(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
    return MF3D_OK;
  }
};

static inline int grid_of(long long n, int tpb) { return (int)((n + tpb - 1) / tpb); }

// Every kernel of a solve is launched with programmatic stream
// serialisation: its CTAs may be placed while the previous kernel on the
// stream drains, and each kernel's first statement (pdl_wait) holds them
// until that kernel has completed.  This removes the launch gap between the
// dependent kernels of an iteration - most of the cost of the small coarse
// levels.  The edges survive stream capture, so the solve graphs keep them.
// MF3D_PDL=0 (read once) launches without the attribute, for comparison.
static bool pdl_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("MF3D_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}
template <typename... KArgs, typename... Args>
static cudaError_t launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                          Args &&...args) {
  cudaLaunchAttribute at;
  at.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at.val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = &at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// launch() with the grid in clusters of `cl` CTAs along x (cl = 1: none).
template <typename... KArgs, typename... Args>
static cudaError_t launch_cl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, int cl,
                             Args &&...args) {
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
  at[1].id = cudaLaunchAttributeClusterDimension;
  at[1].val.clusterDim.x = (unsigned)cl;
  at[1].val.clusterDim.y = 1;
  at[1].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = at;
  cfg.numAttrs = cl > 1 ? 2 : 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// A cooperative launch (every CTA resident at once, for a kernel with grid
// barriers), in plain stream order: no programmatic overlap with the kernels
// around it, so no other grid holds the SMs its CTAs need.
template <typename... KArgs, typename... Args>
static cudaError_t launch_coop(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                               Args &&...args) {
  cudaLaunchAttribute at;
  at.id = cudaLaunchAttributeCooperative;
  at.val.cooperative = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = &at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// 1-D item tiles: for each block, ceil(items_b / kTile) CTAs (i0 = first item).
static std::vector<Tile> make_tiles(const std::vector<long long> &items) {
  std::vector<Tile> t;
  for (size_t b = 0; b < items.size(); ++b)
    for (long long s = 0; s < items[b]; s += kTile) t.push_back(Tile{(int)b, 0, 0, (int)s});
  return t;
}
// A per-block index box [i0,i1] x [j0,j1] x [k0,k1] (inclusive).
struct Box {
  int i0, i1, j0, j1, k0, k1;
};
static void add_tiles_2d(std::vector<Tile> &t, int blk, const Box &x, int TX, int RJ, int kch) {
  if (x.i1 < x.i0 || x.j1 < x.j0 || x.k1 < x.k0) return;
  for (int k = x.k0; k <= x.k1; k += kch)
    for (int j = x.j0; j <= x.j1; j += RJ)
      for (int i = x.i0; i <= x.i1; i += TX) t.push_back(Tile{blk, k, j, i});
}

// 1/h when h is a (normal) power of two - then x*(1/h) == x/h exactly - else 0.
static double pow2_inverse(double h) {
  if (!(h > 0.0) || !std::isfinite(h)) return 0.0;
  int e;
  const double m = std::frexp(h, &e);
  if (m != 0.5) return 0.0;
  const double inv = 1.0 / h;
  return (std::isfinite(inv) && inv * h == 1.0) ? inv : 0.0;
}

// RN(1/b) for div_rcp when 2^-100 <= b <= 2^100, else 0 (the kernel divides).
static double div_reciprocal(double b) {
  if (!(b >= 0x1p-100 && b <= 0x1p+100)) return 0.0;
  return 1.0 / b;
}

// ---------------------------------------------------------------------------
// Resident storage of one block.
// ---------------------------------------------------------------------------
struct LevelStore {
  int elem = 8;  // bytes per value of this level
  std::vector<std::vector<char>> host;  // host images of the uploaded small arrays
  DevBuf<char> phi, rhs, coef, geo;
  DevBuf<CUtensorMap> tmaps;  // phi c0, phi c1, rhs c0, rhs c1
  DevBuf<double> cc;          // L_LSM: per-cell coefficients (six colour-split arrays)
  DevBuf<double> dens;        // L_LSM, levels > 1: cell densities, interior, i fastest
  BlkLev desc;  // host copy with device pointers
};

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library does not link libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return (PFN_cuTensorMapEncodeTiled_v12000)p;
  }();
  return fn;
}

// A 3-D map over one FP64 field in the reference's layout [tk][tj][ti] with
// a (CV_W x rows x 1) box.
static int field_map(CUtensorMap *m, const double *base, int ti, int tj, int tk, int rows) {
  auto enc = tensor_map_encoder();
  if (!enc) { set_error("cuTensorMapEncodeTiled unavailable"); return MF3D_E_CUDA; }
  const cuuint64_t dims[3] = {(cuuint64_t)ti, (cuuint64_t)tj, (cuuint64_t)tk};
  const cuuint64_t strides[2] = {(cuuint64_t)ti * 8, (cuuint64_t)ti * tj * 8};
  const cuuint32_t box[3] = {(cuuint32_t)CV_W, (cuuint32_t)rows, 1u};
  const cuuint32_t es[3] = {1u, 1u, 1u};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)base, dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) { set_error("cuTensorMapEncodeTiled failed: " + std::to_string((int)r)); return MF3D_E_CUDA; }
  return MF3D_OK;
}

// A 3-D map over one colour array [nz+2][ny+2][hp] with a (W x rows x 1) box.
static int colour_map(CUtensorMap *m, void *base, int elem, const BlkLev &B, int W, int rows) {
  auto enc = tensor_map_encoder();
  if (!enc) { set_error("cuTensorMapEncodeTiled unavailable"); return MF3D_E_CUDA; }
  const cuuint64_t dims[3] = {(cuuint64_t)B.hp, (cuuint64_t)(B.ny + 2), (cuuint64_t)(B.nz + 2)};
  const cuuint64_t strides[2] = {(cuuint64_t)B.hp * elem, (cuuint64_t)B.hp * (B.ny + 2) * elem};
  const cuuint32_t box[3] = {(cuuint32_t)W, (cuuint32_t)rows, 1u};
  const cuuint32_t es[3] = {1u, 1u, 1u};
  const CUresult r = enc(m, elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base,
                         dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) { set_error("cuTensorMapEncodeTiled failed: " + std::to_string((int)r)); return MF3D_E_CUDA; }
  return MF3D_OK;
}

struct BlockStore {
  mf3d_block_desc d;     // neighbour ids refer to blocks of the same domain
  int ngrid = 1;
  int own = 1;           // levels of the block's own size (LMR: below them it keeps the last size)
  int elem = 8;          // bytes per multigrid value (8 FP64, 4 FP32)
  std::vector<LevelStore> lv;  // [1..ngrid]
  DevBuf<double> geo1;   // level-1 widths h[3] (n+2) and face distances df[3] (n+1)
  DevBuf<double> planes; // face planes lo/hi of u, v, w (and the L_LSM face densities)
  DevBuf<double> bcst;   // bounds mode: exchange_bc receive planes of u, v, w
  bool lsm = false;      // variable-density coefficients, formed per solve
  BlkFld fld;            // host template (field pointers bound per call)
  DevBuf<double> inlet;  // west inlet plane of the codes 7, 8, 12, 13 (BlkFld::inl)
  DevBuf<double> wall;   // wall functions: tau, tau2 planes of the six faces (BlkFld::wtau)
  size_t bytes = 0;      // device bytes owned
};

// Build one block's hierarchy: replaces `coeff` (mgsolver.for:2-222) and the
// `cof` sizing of localparameters.for:208-237.
static int build_block(BlockStore &S, const mf3d_block_desc &d, int ngrid, int elem_fine, int elem_coarsest, int pl,
                       bool lsm, bool bounds, cudaStream_t s, int own = 0) {
  const int elem = elem_fine;
  S.d = d;
  S.lsm = lsm;
  S.ngrid = ngrid;
  S.own = own > 0 ? std::min(own, ngrid) : ngrid;
  S.elem = elem;
  S.lv.clear();
  S.lv.resize(ngrid + 1);
  S.bytes = 0;
  const double *ext[3] = {d.hx, d.hy, d.hz};
  const double hh[3] = {d.dx, d.dy, d.dz};
  const int nfine[3] = {d.nx, d.ny, d.nz};
  int nmask = 0;
  const int nbr[6] = {d.iprev, d.inext, d.jprev, d.jnext, d.kprev, d.knext};
  const int bc[6] = {d.bc_west, d.bc_east, d.bc_south, d.bc_north, d.bc_bottom, d.bc_top};
  for (int f = 0; f < 6; ++f)
    if (nbr[f] < 0 && bc[f] != MF3D_BC_PERIODIC) nmask |= 1 << f;
  int st;
  for (int g = 1; g <= ngrid; ++g) {
    LevelStore &L = S.lv[g];
    BlkLev &B = L.desc;
    std::memset(&B, 0, sizeof B);
    const int elem = (g == ngrid && ngrid > 1) ? elem_coarsest : elem_fine;
    L.elem = elem;
    const int gl = std::min(g, S.own);  // LMR: past its own levels a block keeps its last size
    B.nx = d.nx >> (gl - 1);
    B.ny = d.ny >> (gl - 1);
    B.nz = d.nz >> (gl - 1);
    B.hp = hp_of(B.nx, elem);
    B.cstr = (long long)(B.nz + 2) * (B.ny + 2) * B.hp;
    B.cstr = (B.cstr + 31) / 32 * 32;  // 256-byte aligned colour arrays
    B.nmask = nmask;
    const size_t nbytes = (size_t)(2 * B.cstr) * elem;
    if ((st = L.phi.alloc(nbytes))) return st;
    if ((st = L.rhs.alloc(nbytes))) return st;
    CK(cudaMemsetAsync(L.phi.p, 0, nbytes, s));
    CK(cudaMemsetAsync(L.rhs.p, 0, nbytes, s));
    S.bytes += 2 * nbytes;
    // coefficients aw, ae (x), as, an (y), ab, at (z); Neumann faces zeroed
    std::vector<double> coef, geo;
    const int nn[3] = {B.nx, B.ny, B.nz};
    for (int a = 0; a < 3; ++a) {
      std::vector<double> w = level_widths(ext[a], nfine[a], hh[a], ngrid, gl);
      const int n = nn[a];
      const double hl = hh[a] * (double)(1 << (gl - 1));
      const double dd = hl * hl;
      for (int side = 0; side < 2; ++side)
        for (int c = 0; c < n + 2; ++c) {
          double v = 0.0;
          if (c >= 1 && c <= n) {
            if (!ext[a]) v = 1.0 / dd;  // mgsolver.for:184-189
            else v = 1.0 / (w[c] * (0.5 * (w[c] + w[side ? c + 1 : c - 1])));
            const int f = 2 * a + side;
            if ((nmask >> f & 1) && c == (side ? n : 1)) v = 0.0;  // mgsolver.for:192-203
          }
          coef.push_back(v);
        }
    }
    // restriction ratios hf/Hc of this (fine) level: 0.5 exactly on uniform axes
    for (int a = 0; a < 3; ++a) {
      const int n = nn[a];
      if (g < S.own) {
        std::vector<double> wf = level_widths(ext[a], nfine[a], hh[a], ngrid, g);
        std::vector<double> wc = level_widths(ext[a], nfine[a], hh[a], ngrid, g + 1);
        for (int c = 0; c < n + 2; ++c) geo.push_back((c >= 1 && c <= n) ? wf[c] / wc[(c + 1) >> 1] : 0.0);
      } else {
        for (int c = 0; c < n + 2; ++c) geo.push_back(0.0);
      }
    }
    // host images of the small per-level arrays stay with the level until
    // the copies have run (one synchronisation at the end of the domain build)
    auto put = [&](DevBuf<char> &buf, const std::vector<double> &v) -> int {
      int r = buf.alloc(v.size() * elem);
      if (r) return r;
      L.host.emplace_back(v.size() * elem);
      char *h = L.host.back().data();
      if (elem == 8) std::memcpy(h, v.data(), v.size() * 8);
      else for (size_t q = 0; q < v.size(); ++q) ((float *)h)[q] = (float)v[q];
      CK(cudaMemcpyAsync(buf.p, h, v.size() * elem, cudaMemcpyHostToDevice, s));
      return MF3D_OK;
    };
    if ((st = put(L.coef, coef))) return st;
    if ((st = put(L.geo, geo))) return st;
    B.phi = L.phi.p;
    B.rhs = L.rhs.p;
    B.coef = L.coef.p;
    B.geo = L.geo.p;
    // TMA maps of the sweep (colour arrays start 256-byte aligned, rows 16-byte multiples)
    CUtensorMap tm[4];
    const int W = elem == 8 ? RbShape<double>::W : RbShape<float>::W;
    for (int c = 0; c < 2; ++c) {
      if ((st = colour_map(&tm[c], L.phi.p + (size_t)c * B.cstr * elem, elem, B, W, RB_RJ + 2))) return st;
      if ((st = colour_map(&tm[2 + c], L.rhs.p + (size_t)c * B.cstr * elem, elem, B, W, RB_RJ))) return st;
    }
    if ((st = L.tmaps.alloc(4))) return st;
    L.host.emplace_back(sizeof tm);
    std::memcpy(L.host.back().data(), tm, sizeof tm);
    CK(cudaMemcpyAsync(L.tmaps.p, L.host.back().data(), sizeof tm, cudaMemcpyHostToDevice, s));
    B.tm = L.tmaps.p;
    if (lsm) {  // FP64 only: formed by k_lsm_coef at every solve
      if ((st = L.cc.alloc((size_t)12 * B.cstr))) return st;
      CK(cudaMemsetAsync(L.cc.p, 0, L.cc.n * sizeof(double), s));
      B.cc = L.cc.p;
      S.bytes += L.cc.n * sizeof(double);
      if (g > 1) {
        if ((st = L.dens.alloc((size_t)B.nx * B.ny * B.nz))) return st;
        S.bytes += L.dens.n * sizeof(double);
      }
    }
  }
  // level-1 field geometry: widths, face distances (bit-exact dx on a uniform axis)
  std::vector<double> g1;
  size_t off_h[3], off_df[3], off_rh[3], off_rdf[3];
  for (int a = 0; a < 3; ++a) {
    std::vector<double> w = level_widths(ext[a], nfine[a], hh[a], ngrid, 1);
    off_h[a] = g1.size();
    for (int c = 0; c < nfine[a] + 2; ++c) g1.push_back(ext[a] ? w[c] : hh[a]);
    off_df[a] = g1.size();
    for (int c = 0; c <= nfine[a]; ++c) g1.push_back(ext[a] ? 0.5 * (w[c] + w[c + 1]) : hh[a]);
    off_rh[a] = g1.size();
    for (int c = 0; c < nfine[a] + 2; ++c) g1.push_back(div_reciprocal(g1[off_h[a] + c]));
    off_rdf[a] = g1.size();
    for (int c = 0; c <= nfine[a]; ++c) g1.push_back(div_reciprocal(g1[off_df[a] + c]));
  }
  if ((st = S.geo1.upload(g1, s))) return st;
  const size_t pyz = (size_t)d.ny * d.nz, pxz = (size_t)d.nx * d.nz, pxy = (size_t)d.nx * d.ny;
  if ((st = S.planes.alloc(3 * (pyz + pxz + pxy)))) return st;
  CK(cudaMemsetAsync(S.planes.p, 0, S.planes.n * sizeof(double), s));
  CK(cudaStreamSynchronize(s));  // g1 is a local
  S.bytes += (S.geo1.n + S.planes.n) * sizeof(double);
  BlkFld &F = S.fld;
  std::memset(&F, 0, sizeof F);
  F.nx = d.nx; F.ny = d.ny; F.nz = d.nz; F.pl = pl;
  F.ti = d.nx + 2 * pl; F.tj = d.ny + 2 * pl;
  for (int a = 0; a < 3; ++a) {
    F.h[a] = S.geo1.p + off_h[a];
    F.df[a] = S.geo1.p + off_df[a];
    F.rh[a] = S.geo1.p + off_rh[a];
    F.rdf[a] = S.geo1.p + off_rdf[a];
  }
  double *pp = S.planes.p;
  F.lo[0] = pp; F.hi[0] = pp + pyz; pp += 2 * pyz;
  F.lo[1] = pp; F.hi[1] = pp + pxz; pp += 2 * pxz;
  F.lo[2] = pp; F.hi[2] = pp + pxy; pp += 2 * pxy;
  F.dlo[0] = pp; F.dlo[1] = pp + pyz; F.dlo[2] = pp + pyz + pxz;
  F.L1 = S.lv[1].desc;
  const int bcs[6] = {d.bc_west, d.bc_east, d.bc_south, d.bc_north, d.bc_bottom, d.bc_top};
  const int nbrs[6] = {d.iprev, d.inext, d.jprev, d.jnext, d.kprev, d.knext};
  for (int f = 0; f < 6; ++f) {
    F.bcode[f] = bcs[f];
    F.pface[f] = (bcs[f] == MF3D_BC_PERIODIC && nbrs[f] < 0) ? (nbrs[f ^ 1] < 0 ? 1 : 2) : 0;
  }
  if (bounds) {
    const long long ti = d.nx + 2 * pl, tj = d.ny + 2 * pl, tk = d.nz + 2 * pl;
    F.bcplane = std::max(tj * tk, std::max(ti * tk, ti * tj));
    if ((st = S.bcst.alloc((size_t)18 * F.bcplane))) return st;
    F.bcst = S.bcst.p;
    S.bytes += S.bcst.n * sizeof(double);
  }
  for (int a = 0; a < 3; ++a) F.pinv[a] = ext[a] ? 0.0 : pow2_inverse(hh[a]);
  return MF3D_OK;
}

// A halo copy between blocks of one domain (domain-local block indices).
struct HaloLocal {
  int dblk, doff, sblk, soff;
};

// One domain: its blocks, halo copy lists per level, face rules.
struct DomainStore {
  int ngrid = 1;
  std::vector<std::unique_ptr<BlockStore>> blocks;
  std::vector<std::vector<HaloLocal>> halo;  // per level, staged pairs first
  std::vector<int> nstaged;                  // per level
  std::vector<DevBuf<HaloCopy>> dhalo;       // per level, the same pairs on the device
  std::vector<FaceRule> rules;               // 6 per block, domain-local sources
  // exchange(1..3) and exchange(4) + pbound of the fields as copy maps
  // (mf3d_create contexts, build_field_maps): u, v, w pairs and p pairs,
  // staged pairs first; the evolution lists of the chained u, v, w ghosts
  DevBuf<FxCopy> fx_uvw, fx_p, fxe_sub, fxe_chain;
  DevBuf<FxCell> fxe_cells;
  long long nfx_uvw = 0, nsfx_uvw = 0, nfx_p = 0, nsfx_p = 0;
  long long nfxe_sub = 0, nsfxe_sub = 0, nfxe_chain = 0, nfxe_cells = 0;
  bool fx_per_iteration = false;
  // LMR: per level, the halo refresh as a program (build_halo_lmr) where
  // refinements meet on the level; empty elsewhere
  struct LmrLevel {
    DevBuf<LmrTerm> terms;
    DevBuf<LmrNode> nodes;
    DevBuf<LmrWrite> writes;
    std::vector<int> depth_start;
    int n_writes = 0;
  };
  std::vector<LmrLevel> lmr;
  size_t bytes = 0;
};

// The field exchange maps of a domain (FxCopy lists, pairs whose source is
// itself written first: they are staged).
//   p:  exchange(4) + pbound, applied whole after every p += pp.
//   u, v, w, `per_iteration` (the 4th-order calmas path, which writes u, v, w
//       in every outer iteration): exchange(1..3) whole, applied at every
//       calvel point.
//   u, v, w otherwise (the fused path writes u, v, w once, after the loop):
//       the final exchange, whose chained sources - ghost cells of the state
//       before it that an earlier exchange wrote - read the `prev` slots
//       that k_fx_evolve fills; and the evolution lists of those chains (see
//       k_fx_evolve).
static int build_field_maps(DomainStore &D, const std::vector<mf3d_block_desc> &descs, int pl, int pl_ex,
                            bool per_iteration, cudaStream_t s) {
  const int nb = (int)descs.size();
  std::vector<long long> base(nb);
  long long acc = 0;
  for (int b = 0; b < nb; ++b) {
    base[b] = acc;
    acc += (long long)(descs[b].nx + 2 * pl) * (descs[b].ny + 2 * pl) * (descs[b].nz + 2 * pl);
  }
  if (nb > 65535) { set_error("field exchange map: more than 65535 blocks"); return MF3D_E_UNSUPPORTED; }
  auto blk_of = [&](long long id) { return (int)(std::upper_bound(base.begin(), base.end(), id) - base.begin()) - 1; };
  auto loc = [&](long long id, unsigned short &blk, unsigned &off) {
    const int b = blk_of(id);
    blk = (unsigned short)b;
    off = (unsigned)(id - base[b]);
  };
  // 1-based field indices of a cell and whether it is a ghost cell
  auto ijk = [&](long long id, int &b, int &i, int &j, int &k) {
    b = blk_of(id);
    long long r = id - base[b];
    const long long ti = descs[b].nx + 2 * pl, tj = descs[b].ny + 2 * pl;
    i = (int)(r % ti) + 1;
    r /= ti;
    j = (int)(r % tj) + 1;
    k = (int)(r / tj) + 1;
  };
  auto ghost = [&](long long id) {
    int b, i, j, k;
    ijk(id, b, i, j, k);
    return i <= pl || j <= pl || k <= pl || i > descs[b].nx + pl || j > descs[b].ny + pl || k > descs[b].nz + pl;
  };
  int st;
  // p: whole
  {
    std::vector<HaloPair> pr = build_field_map(descs, base, pl, 4, 0, true);
    std::vector<FxCopy> staged, plain;
    auto written = [&](long long id) {
      auto it = std::lower_bound(pr.begin(), pr.end(), id, [](const HaloPair &x, long long v) { return x.dst < v; });
      return it != pr.end() && it->dst == id;
    };
    for (const auto &x : pr) {
      FxCopy c;
      loc(x.dst, c.dblk, c.doff);
      loc(x.src, c.sblk, c.soff);
      c.comp = 3;
      (written(x.src) ? staged : plain).push_back(c);
    }
    D.nsfx_p = (long long)staged.size();
    staged.insert(staged.end(), plain.begin(), plain.end());
    D.nfx_p = (long long)staged.size();
    if ((st = D.fx_p.upload(staged, s))) return st;
    D.bytes += staged.size() * sizeof(FxCopy);
  }
  // u, v, w
  std::vector<FxCopy> fin_staged, fin_plain, sub_staged, sub_plain, chain;
  std::vector<FxCell> cells;
  for (int op = 1; op <= 3; ++op) {
    std::vector<HaloPair> pr = build_field_map(descs, base, pl, op, pl_ex, false);
    auto find = [&](long long id) {
      auto it = std::lower_bound(pr.begin(), pr.end(), id, [](const HaloPair &x, long long v) { return x.dst < v; });
      return (it != pr.end() && it->dst == id) ? (long long)(it - pr.begin()) : -1LL;
    };
    if (per_iteration) {
      for (const auto &x : pr) {
        FxCopy c;
        loc(x.dst, c.dblk, c.doff);
        loc(x.src, c.sblk, c.soff);
        c.comp = op - 1;
        (find(x.src) >= 0 ? fin_staged : fin_plain).push_back(c);
      }
      continue;
    }
    // C: the ghost cells whose values chains carry across exchanges - chained
    // sources that some exchange writes, closed over the ghost sources of
    // the pairs writing them
    std::vector<char> inC(pr.size(), 0);  // by pair index (the pair writing the cell)
    std::vector<long long> work;
    for (const auto &x : pr)
      if (ghost(x.src)) {
        const long long q = find(x.src);
        if (q >= 0 && !inC[q]) { inC[q] = 1; work.push_back(q); }
      }
    while (!work.empty()) {
      const long long q = work.back();
      work.pop_back();
      if (!ghost(pr[q].src)) continue;
      const long long r = find(pr[q].src);
      if (r >= 0 && !inC[r]) { inC[r] = 1; work.push_back(r); }
    }
    // prev slots: one per chained source in C
    std::unordered_map<long long, unsigned> slot;
    for (const auto &x : pr)
      if (ghost(x.src) && find(x.src) >= 0 && !slot.count(x.src)) {
        const unsigned sl = (unsigned)chain.size();
        slot[x.src] = sl;
        FxCopy c;
        loc(x.src, c.sblk, c.doff);
        c.dblk = c.sblk;
        c.soff = sl;
        c.comp = op - 1;
        chain.push_back(c);
      }
    std::unordered_set<long long> seen_cell;
    for (size_t q = 0; q < pr.size(); ++q) {
      const auto &x = pr[q];
      // the final exchange
      FxCopy f;
      loc(x.dst, f.dblk, f.doff);
      loc(x.src, f.sblk, f.soff);
      f.comp = op - 1;
      auto it = slot.find(x.src);
      if (it != slot.end()) {
        f.comp |= 8;
        f.soff = it->second;
        fin_plain.push_back(f);  // prev is not written by the apply: no staging
      } else {
        (find(x.src) >= 0 ? fin_staged : fin_plain).push_back(f);
      }
      if (!inC[q]) continue;
      // the evolution sub-map: pairs writing C, staged when their source is
      // written by the sub-map; interior sources formed by calvel first
      FxCopy c;
      loc(x.dst, c.dblk, c.doff);
      loc(x.src, c.sblk, c.soff);
      c.comp = op - 1;
      const long long r = find(x.src);
      (r >= 0 && inC[r] ? sub_staged : sub_plain).push_back(c);
      if (!ghost(x.src) && seen_cell.insert(x.src).second) {
        FxCell e;
        int b, i, j, k;
        ijk(x.src, b, i, j, k);
        e.blk = b; e.comp = op - 1; e.i = i - pl; e.j = j - pl; e.k = k - pl;  // level-1 indices
        cells.push_back(e);
      }
    }
  }
  D.nsfx_uvw = (long long)fin_staged.size();
  fin_staged.insert(fin_staged.end(), fin_plain.begin(), fin_plain.end());
  D.nfx_uvw = (long long)fin_staged.size();
  D.nsfxe_sub = (long long)sub_staged.size();
  sub_staged.insert(sub_staged.end(), sub_plain.begin(), sub_plain.end());
  D.nfxe_sub = (long long)sub_staged.size();
  D.nfxe_chain = (long long)chain.size();
  D.nfxe_cells = (long long)cells.size();
  D.fx_per_iteration = per_iteration;
  if ((st = D.fx_uvw.upload(fin_staged, s))) return st;
  if ((st = D.fxe_sub.upload(sub_staged, s))) return st;
  if ((st = D.fxe_chain.upload(chain, s))) return st;
  if ((st = D.fxe_cells.upload(cells, s))) return st;
  D.bytes += (fin_staged.size() + sub_staged.size() + chain.size()) * sizeof(FxCopy) + cells.size() * sizeof(FxCell);
  CK(cudaStreamSynchronize(s));  // the host vectors are locals
  return MF3D_OK;
}

static long long level_off(const BlkLev &B, int i, int j, int k) {
  const int c = (i + j + k + 1) & 1;
  return c * B.cstr + ((long long)k * (B.ny + 2) + j) * B.hp + (i >> 1);
}

// `own` (LMR, else null): each block's levels of its own size; `rdv`:
// rdv(block, g) per block, indexed [b][g].
static int build_domain(DomainStore &D, const mf3d_block_desc *blocks, int nb, int ngrid, int elem, int elem_coarsest,
                        int pl, cudaStream_t s, bool lsm = false, bool bounds = false, int field_maps_pl_ex = -1,
                        bool fx_per_iteration = false, const std::vector<int> *own = nullptr,
                        const std::vector<std::vector<int>> *rdv = nullptr) {
  D.ngrid = ngrid;
  D.blocks.clear();
  std::vector<mf3d_block_desc> descs(blocks, blocks + nb);
  int st = face_rules(descs, D.rules);
  if (st) return st;
  D.bytes = 0;
  for (int b = 0; b < nb; ++b) {
    D.blocks.emplace_back(new BlockStore());
    if ((st = build_block(*D.blocks.back(), descs[b], ngrid, elem, elem_coarsest, pl, lsm, bounds, s,
                          own ? (*own)[b] : 0)))
      return st;
    D.bytes += D.blocks.back()->bytes;
  }
  D.halo.assign(ngrid + 1, {});
  D.nstaged.assign(ngrid + 1, 0);
  D.lmr.clear();
  D.lmr.resize(ngrid + 1);
  for (int g = 1; g <= ngrid; ++g) {
    if (rdv) {
      bool mixed = false;
      for (int b = 1; b < nb; ++b) mixed |= (*rdv)[b][g] != (*rdv)[0][g];
      if (mixed) {
        std::vector<LevelGeom> geom(nb);
        std::vector<long long> base(nb);
        std::vector<int> rg(nb);
        long long acc = 0;
        for (int b = 0; b < nb; ++b) {
          const BlkLev &B = D.blocks[b]->lv[g].desc;
          geom[b] = LevelGeom{B.nx, B.ny, B.nz};
          base[b] = acc;
          acc += geom[b].cells();
          rg[b] = (*rdv)[b][g];
        }
        const LmrProgram P = build_halo_lmr(descs, geom, base, rg);
        auto loc = [&](long long id, int &blk, int &off) {
          const int b = (int)(std::upper_bound(base.begin(), base.end(), id) - base.begin()) - 1;
          long long lin = id - base[b];
          const LevelGeom &G = geom[b];
          const int i = (int)(lin % (G.nx + 2));
          lin /= (G.nx + 2);
          const int j = (int)(lin % (G.ny + 2));
          const int k = (int)(lin / (G.ny + 2));
          blk = b;
          off = (int)level_off(D.blocks[b]->lv[g].desc, i, j, k);
        };
        std::vector<LmrTerm> terms(P.terms.size());
        for (size_t q = 0; q < terms.size(); ++q) {
          const auto &t = P.terms[q];
          terms[q].w = t.w;
          if (t.ref >= 0) loc(t.ref, terms[q].blk, terms[q].off);
          else if (t.ref == kLmrZero) { terms[q].blk = -2; terms[q].off = 0; }
          else { terms[q].blk = -1; terms[q].off = (int)(-2 - t.ref); }
        }
        std::vector<LmrNode> nodes(P.nodes.size());
        for (size_t q = 0; q < nodes.size(); ++q) {
          nodes[q] = LmrNode{P.nodes[q].t0, P.nodes[q].nt, P.nodes[q].scale};
          if (nodes[q].nt < 1 || nodes[q].nt > LMR_MAX_TERMS) {
            set_error("LMR halo program: a node of " + std::to_string(nodes[q].nt) + " terms");
            return MF3D_E_INVALID;
          }
        }
        std::vector<LmrWrite> writes(P.writes.size() + P.copies.size());
        for (size_t q = 0; q < P.writes.size(); ++q) {
          loc(P.writes[q].first, writes[q].blk, writes[q].off);
          writes[q].node = P.writes[q].second;
          writes[q].sblk = writes[q].soff = 0;
        }
        for (size_t q = 0; q < P.copies.size(); ++q) {
          LmrWrite &W = writes[P.writes.size() + q];
          loc(P.copies[q].first, W.blk, W.off);
          loc(P.copies[q].second, W.sblk, W.soff);
          W.node = -1;
        }
        DomainStore::LmrLevel &M = D.lmr[g];
        if ((st = M.terms.upload(terms, s))) return st;
        if ((st = M.nodes.upload(nodes, s))) return st;
        if ((st = M.writes.upload(writes, s))) return st;
        CK(cudaStreamSynchronize(s));  // the host vectors are locals
        M.depth_start = P.depth_start;
        M.n_writes = (int)writes.size();
        D.bytes += terms.size() * sizeof(LmrTerm) + nodes.size() * sizeof(LmrNode) + writes.size() * sizeof(LmrWrite);
        continue;  // no copy map on this level
      }
    }
    std::vector<LevelGeom> geom(nb);
    std::vector<long long> base(nb);
    long long acc = 0;
    for (int b = 0; b < nb; ++b) {
      const BlkLev &B = D.blocks[b]->lv[g].desc;
      geom[b] = LevelGeom{B.nx, B.ny, B.nz};
      base[b] = acc;
      acc += geom[b].cells();
    }
    std::vector<HaloPair> pairs = build_halo_map(descs, geom, base);
    std::vector<bool> is_dst(acc, false);  // cells written by the refresh
    for (auto &p : pairs) is_dst[p.dst] = true;
    auto loc = [&](long long id, int &blk, int &off) {
      int b = (int)(std::upper_bound(base.begin(), base.end(), id) - base.begin()) - 1;
      long long lin = id - base[b];
      const LevelGeom &G = geom[b];
      int i = (int)(lin % (G.nx + 2));
      long long r = lin / (G.nx + 2);
      int j = (int)(r % (G.ny + 2));
      int k = (int)(r / (G.ny + 2));
      blk = b;
      off = (int)level_off(D.blocks[b]->lv[g].desc, i, j, k);
    };
    for (int pass = 0; pass < 2; ++pass)
      for (auto &p : pairs) {
        const bool staged = is_dst[p.src];
        if ((pass == 0) != staged) continue;
        HaloLocal h;
        loc(p.dst, h.dblk, h.doff);
        loc(p.src, h.sblk, h.soff);
        D.halo[g].push_back(h);
        if (staged) D.nstaged[g]++;
      }
  }
  // resident device copies (domain-local block indices)
  D.dhalo.clear();
  D.dhalo.resize(ngrid + 1);
  for (int g = 1; g <= ngrid; ++g) {
    std::vector<HaloCopy> h(D.halo[g].size());
    for (size_t q = 0; q < h.size(); ++q)
      h[q] = HaloCopy{D.halo[g][q].dblk, D.halo[g][q].doff, D.halo[g][q].sblk, D.halo[g][q].soff};
    if ((st = D.dhalo[g].upload(h, s))) return st;
    D.bytes += h.size() * sizeof(HaloCopy);
  }
  CK(cudaStreamSynchronize(s));  // the host vectors are locals
  if (field_maps_pl_ex >= 0 && (st = build_field_maps(D, descs, pl, field_maps_pl_ex, fx_per_iteration, s))) return st;
  return MF3D_OK;
}

// ---------------------------------------------------------------------------
// A view: launch tables over a set of domains.
// ---------------------------------------------------------------------------
enum Subset { SUB_A = 0, SUB_C = 1, SUB_D = 2 };  // all present / coarsest here / continuing down

// the red-black sweep schedule a level starts with (sweep_segments): the
// fastest on whole solves of 128^3 blocks
constexpr int kDefaultSweepSchedule = 2;

struct ViewLevel {
  DevBuf<BlkLev> tab;                 // one entry per view block (absent: nx = 0)
  std::vector<BlkLev> htab;           // host copy of tab (the autotuner rebuilds tables from it)
  std::vector<int> hblk[3];           // view blocks of each subset
  int sched = kDefaultSweepSchedule;  // red-black sweep schedule (sweep_segments)
  DevBuf<RbSeg> sweep[3];             // red-black sweep segments (k_rbgs), per subset
  DevBuf<int> sfirst[3];              // first segment of each sweep CTA (+ total)
  DevBuf<Tile> cells[3];
  int n_sweep[3] = {0, 0, 0}, n_cells[3] = {0, 0, 0};  // sweep CTAs; cell tiles
  DevBuf<int> spre[3];                // small levels: first sweep item of each listed block (+ total)
  long long small_items[3] = {0, 0, 0};
  int small = 0;                      // 1: the level's sweeps use k_rbgs_small
  DevBuf<Tile> rtile, ptile;          // restriction into this level (SUB_A); prolongation from the next (SUB_D)
  int n_rtile = 0, n_ptile = 0, rkch = 1, pkch = 1;
  DevBuf<Tile> rtma;                  // TMA restriction into this level: coarse interior tiles (SUB_A)
  int n_rtma = 0, rtma_kch = 1;
  DevBuf<int> list[3];
  int n_list[3] = {0, 0, 0};
  DevBuf<HaloSeg> hseg[3];            // one segment per domain of the subset
  int n_hseg[3] = {0, 0, 0};
  long long n_halo[3] = {0, 0, 0}, n_staged[3] = {0, 0, 0};
  DevBuf<char> stage[3];              // staged halo values
  long long cells_sub[3] = {0, 0, 0}; // interior cells of each subset
  // line relaxation (mg_itrsch 2): TDMA factors of every listed block, and the
  // k_tdma_lines shape: cluster size, lines staged at a time, longest line
  DevBuf<char> tdf;
  int td_cl = 1, td_gmax = 1, td_nmax = 1, td_numax = 1, td_lines[3] = {0, 0, 0};
  int lx_cl = 1;                      // lexicographic relaxation (mg_itrsch 1): CTAs per block
  size_t td_smem = 0;
  bool td_fp64 = true;                // the level relaxes in FP64
  // LMR (single-domain views): the level's halo program where refinements
  // meet on it (DomainStore::LmrLevel), and the blocks past their own last
  // level - restricted into this level by injection, corrected from the next
  // one by addition - as item lists over their ghost-inclusive cells
  const LmrTerm *lmr_terms = nullptr;
  const LmrNode *lmr_nodes = nullptr;
  const LmrWrite *lmr_writes = nullptr;
  std::vector<int> lmr_depth;
  int lmr_nwrites = 0;
  DevBuf<double> lmr_val;
  DevBuf<int> inj_list, add_list;
  DevBuf<long long> inj_pre, add_pre;
  int n_inj = 0, n_add = 0;
  long long inj_items = 0, add_items = 0;
};

struct View {
  std::vector<BlockStore *> blk;      // view position -> block
  std::vector<int> blk_dom;           // view position -> view domain
  std::vector<DomainStore *> dom;     // view domain -> domain
  int Lmax = 0;
  std::vector<ViewLevel> lv;          // [1..Lmax]
  std::vector<BlkFld> hf;
  DevBuf<BlkFld> df;
  DevBuf<Tile> t_int, t_zint, t_l1cells, t_faces, t_planes, t_pairs, t_vfaces;
  DevBuf<Tile> t_bcax[3];             // bounds mode: 3 components x 2 faces x ttc plane per block, per axis
  int n_bcax[3] = {0, 0, 0};
  bool bc_periodic[3] = {false, false, false};  // some block has a periodic face along the axis
  int n_pairs = 0, pairs_kch = 1;
  int n_int = 0, n_zint = 0, n_l1cells = 0, n_faces = 0, n_planes = 0, n_vfaces = 0;
  // field exchanges as copy maps (a view over one domain that has them):
  // exchange(1..3) of u, v, w and exchange(4) + pbound of p
  const FxCopy *fx_uvw = nullptr, *fx_p = nullptr, *fxe_sub = nullptr, *fxe_chain = nullptr;
  const FxCell *fxe_cells = nullptr;
  long long nfx_uvw = 0, nsfx_uvw = 0, nfx_p = 0, nsfx_p = 0;
  long long nfxe_sub = 0, nsfxe_sub = 0, nfxe_chain = 0, nfxe_cells = 0;
  bool fx_per_iteration = false;      // u, v, w exchanged whole at every calvel point (4th-order calmas)
  DevBuf<double> fx_stage, fx_prev;   // staged sources; chained sources before the last exchange
  // the coarse end of the red-black V-cycle in one cluster launch (k_coarse_cycle):
  // levels cc_g0..Lmax, 0 = off
  int cc_g0 = 0;
  size_t cc_smem = 0;
  CcArgs cc_args;
  // the middle levels in one cooperative launch per direction (k_mid_cycle):
  // phases down (levels 2 .. first cluster level - 1, or the coarsest) and up
  bool mid_on = false;
  DevBuf<MidPhase> mid_down, mid_up;
  int n_mid_down = 0, n_mid_up = 0, mid_grid = 0;
  std::vector<DevBuf<int>> mid_lists;
  std::vector<DevBuf<long long>> mid_pres;
  DevBuf<MidBar> mid_bar;
  DevBuf<CcHalo> cc_halo;
  DevBuf<HaloCopy> cc_pairs;
  DevBuf<DomState> ds;
  DevBuf<int> act, ones;
  DevBuf<int> err;                    // device error code (a TMA wait that gave up)
  DevBuf<int> budget;                 // iterations left in the server's bounded loop
  DevBuf<CUtensorMap> fmaps;          // per block: p, ustar, vstar, wstar (bound fields)
  bool fields_tma = false;            // bound fields admit the TMA calvel/calmas
  bool wall_law = false;              // some block has wall-function faces (BlkFld::wtau)
  DevBuf<unsigned long long> rmax, rmax_scratch;
  DevBuf<double> hist;
  int hcap = 0;
  long long n_l1 = 0;
  // graphs: the whole outer loop (WHILE node) and a single iteration
  cudaGraph_t g_loop = nullptr, g_once = nullptr;
  cudaGraphExec_t x_loop = nullptr, x_once = nullptr;
  cudaGraphConditionalHandle cond = 0;
  long long launches_per_iter = 0;
  void drop_graphs() {
    if (x_loop) cudaGraphExecDestroy(x_loop);
    if (g_loop) cudaGraphDestroy(g_loop);
    if (x_once) cudaGraphExecDestroy(x_once);
    if (g_once) cudaGraphDestroy(g_once);
    x_loop = x_once = nullptr;
    g_loop = g_once = nullptr;
  }
  ~View() { drop_graphs(); }
};

}  // namespace mf3d

using namespace mf3d;

namespace mf3d {
struct SipState;
}

struct mf3d_ctx {
  mf3d_params prm;
  int device = 0;
  int elem = 8;
  bool coarse64 = false;    // FP32 V-cycle with the coarsest level (and its sweeps) in FP64
  bool lmr = false;         // blocks of different refinement (LMR): the V-cycle only
  int nsm = 148;            // SMs of the device
  int sweep_occ = 4;        // resident sweep CTAs per SM
  cudaStream_t stream = nullptr;
  // host entry point: u, v, w travel on a side stream while the solve runs
  // (only the final calvel needs them); their wall values go straight into
  // the face planes first
  cudaStream_t side = nullptr;
  cudaEvent_t ev_side = nullptr;
  cudaEvent_t ev_in = nullptr;  // host entry: the solve's inputs are on the device
  bool walls_given = false, wait_side = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  long long launches = 0;
  std::vector<std::unique_ptr<DomainStore>> doms;
  std::unique_ptr<View> view;
  bool use_graph = true;
  // kernel timing (mf3d_profile)
  int prof_kind = 0;
  std::vector<cudaEvent_t> prof_ev;
  std::vector<double> prof_pending_bytes;
  double prof_ms = 0.0, prof_bytes = 0.0;
  long long prof_n = 0;
  // solver 1 (SIP): factors, residual, the substitution graph
  std::unique_ptr<mf3d::SipState> sip;
  long long sip_sweeps = 0;
  // host entry point mirrors
  DevBuf<double> mirror;
  std::vector<size_t> mirror_off;
  DevBuf<double *> ptrs;
  // mf3d_mgkcyc_device_noalloc: device address of its fixed pointer tables
  void *noalloc_tab = nullptr;
  // mf3d_bind_old_velocity: uoo, voo, woo per block (view order) for the
  // convective outflow of the solve's boundu/v/w; empty = none bound
  std::vector<std::array<const double *, 3>> oo_bound;
  // mf3d_set_wall_model: Re and fric (control.cin) of the wall functions
  double wall_re = 0.0, wall_fric = 0.0;
};

namespace mf3d {

// Kernel timing: bracket one launch of the profiled class with events.
static void prof_begin(mf3d_ctx *C, int kind, double bytes) {
  if (C->prof_kind != kind || kind == 0) return;
  size_t q = C->prof_pending_bytes.size();
  while (C->prof_ev.size() < 2 * (q + 1)) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    C->prof_ev.push_back(e);
  }
  cudaEventRecord(C->prof_ev[2 * q], C->stream);
  C->prof_pending_bytes.push_back(bytes);
}
static void prof_end(mf3d_ctx *C, int kind) {
  if (C->prof_kind != kind || kind == 0 || C->prof_pending_bytes.empty()) return;
  cudaEventRecord(C->prof_ev[2 * (C->prof_pending_bytes.size() - 1) + 1], C->stream);
}
static void prof_collect(mf3d_ctx *C) {
  for (size_t q = 0; q < C->prof_pending_bytes.size(); ++q) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, C->prof_ev[2 * q], C->prof_ev[2 * q + 1]) == cudaSuccess) {
      C->prof_ms += ms;
      C->prof_bytes += C->prof_pending_bytes[q];
      C->prof_n += 1;
    }
  }
  C->prof_pending_bytes.clear();
}

// Levels with at most this many interior cells sweep with k_rbgs_small.
constexpr long long kSmallLevelCells = 1ll << 19;

// Red-black sweep segments of a set of blocks (k_rbgs).  A column is 32
// lanes over q (ceil(nx/2) per row) by RB_RJ rows of one block.  Schedules:
//   0  the planes of all columns laid end to end and cut into equal runs, one
//      per CTA: as many CTAs as the device holds at once (whole multiples of
//      that when a run would exceed RB_KMAX planes), so the launch has no
//      partial wave; a run that crosses a column boundary becomes two
//      segments;
//   1  the same over twice as many CTAs (two waves);
//   2  each column cut into c equal runs, c = resident CTAs / columns (at
//      least 1): no run crosses a column, at most one wave;
//   3  the same with c + 1 runs per column;
//   4  runs of kch planes in several waves, kch in {2, 4, 8, 16, 32} the
//      one whose estimated time ceil(CTAs / resident) * (kch + ring fill) is
//      least (concurrent CTAs cover neighbouring columns of the same planes).
// Runs are at least kMinRun planes (shorter ones would be mostly ring fill)
// and at most RB_KMAX.  Returns the CTA count; first[c] .. first[c+1]-1 are
// CTA c's segments; the CTAs run columns in order of their first plane.
constexpr long long kMinRun = 4;
constexpr int kSweepSchedules = 5;
static int sweep_segments(const mf3d_ctx *C, const std::vector<BlkLev> &tab, const std::vector<int> &blocks,
                          std::vector<RbSeg> &segs, std::vector<int> &first, int sched = 0) {
  segs.clear();
  first.assign(1, 0);
  long long planes = 0, columns = 0;
  for (int b : blocks) {
    const BlkLev &B = tab[b];
    const long long cols = (long long)((B.nx + 1) / 2 + RB_TX - 1) / RB_TX * ((B.ny + RB_RJ - 1) / RB_RJ);
    columns += cols;
    planes += cols * B.nz;
  }
  if (planes == 0) return 0;
  const long long resident = (long long)C->nsm * C->sweep_occ;
  if (sched >= 2) {
    // per block, runs of `run` planes; CTAs ordered plane run first, so the
    // CTAs resident together share planes (their halo rows meet in L2)
    auto run_of = [&](const BlkLev &B) -> long long {
      if (sched == 4) return 0;
      const long long c = std::max(1LL, resident / columns) + (sched == 3 ? 1 : 0);
      return std::min<long long>(RB_KMAX, std::max(kMinRun, (B.nz + c - 1) / c));
    };
    long long kch4 = 2;
    if (sched == 4) {
      double best = 1e300;
      for (long long kc : {2LL, 4LL, 8LL, 16LL, (long long)std::min(32, RB_KMAX)}) {
        long long n = 0;
        for (int b : blocks) {
          const BlkLev &B = tab[b];
          n += (long long)((B.nx + 1) / 2 + RB_TX - 1) / RB_TX * ((B.ny + RB_RJ - 1) / RB_RJ) * ((B.nz + kc - 1) / kc);
        }
        const double cost = (double)((n + resident - 1) / resident) * (kc + RB_PD);
        if (cost <= best) { best = cost; kch4 = kc; }
      }
    }
    for (int b : blocks) {
      const BlkLev &B = tab[b];
      const long long run = sched == 4 ? kch4 : run_of(B);
      for (int k = 1; k <= B.nz; k += (int)run)
        for (int j0 = 1; j0 <= B.ny; j0 += RB_RJ)
          for (int q0 = 0; q0 < (B.nx + 1) / 2; q0 += RB_TX) {
            segs.push_back(RbSeg{b, k, (int)std::min<long long>(k + run - 1, B.nz), j0, q0, 0, 0, 0});
            first.push_back((int)segs.size());
          }
    }
    return (int)first.size() - 1;
  }
  const long long target = resident * (sched == 1 ? 2 : 1);
  const long long waves = (planes + target * RB_KMAX - 1) / (target * RB_KMAX);
  const long long run = std::max(kMinRun, (planes + target * waves - 1) / (target * waves));
  long long left = run;
  for (int b : blocks) {
    const BlkLev &B = tab[b];
    for (int j0 = 1; j0 <= B.ny; j0 += RB_RJ)
      for (int q0 = 0; q0 < (B.nx + 1) / 2; q0 += RB_TX)
        for (int k = 1; k <= B.nz;) {
          const int take = (int)std::min<long long>(left, B.nz - k + 1);
          segs.push_back(RbSeg{b, k, k + take - 1, j0, q0, 0, 0, 0});
          k += take;
          left -= take;
          if (left == 0) {
            first.push_back((int)segs.size());
            left = run;
          }
        }
  }
  if (first.back() != (int)segs.size()) first.push_back((int)segs.size());
  return (int)first.size() - 1;
}

// TMA restriction tiles into a coarse level: 32 x RB_RJ/2 coarse cells, kch
// planes; kch = 0 picks it as for the sweep's estimate (2 resident CTAs per
// SM: the ring takes ~110 KB).  Returns kch.
static int rtma_tiles(const mf3d_ctx *C, const std::vector<BlkLev> &tab, const std::vector<int> &blocks, int kch,
                      std::vector<Tile> &out) {
  out.clear();
  if (kch <= 0) {
    const long long resident = (long long)C->nsm * 2;
    kch = 2;
    double best_cost = 1e300;
    for (int kc : {2, 4, 8, 16, 32}) {
      long long n = 0;
      for (int b : blocks) {
        const BlkLev &B = tab[b];
        n += (long long)((B.nx + 31) / 32) * ((B.ny + RB_RJ / 2 - 1) / (RB_RJ / 2)) * ((B.nz + kc - 1) / kc);
      }
      const double cost = (double)((n + resident - 1) / resident) * (kc + 3);
      if (cost <= best_cost) { best_cost = cost; kch = kc; }
    }
  }
  for (int b : blocks) {
    const BlkLev &B = tab[b];
    add_tiles_2d(out, b, Box{1, B.nx, 1, B.ny, 1, B.nz}, 32, RB_RJ / 2, kch);
  }
  return kch;
}

// Plane tiles of kTile consecutive columns of a GX x GY plane and kch planes
// of K0..K1, per block; kch as for the sweep (few waves of resident CTAs).
struct PlaneExt {
  int blk, gx, gy, k0, k1;
};
static int plane_tiles(const mf3d_ctx *C, const std::vector<PlaneExt> &ext, std::vector<Tile> &out) {
  out.clear();
  if (ext.empty()) return 1;
  const long long resident = (long long)C->nsm * 6;
  int best = 2;
  double best_cost = 1e300;
  for (int kch : {2, 4, 8, 16}) {
    long long n = 0;
    for (const auto &e : ext)
      n += ((long long)e.gx * e.gy + kTile - 1) / kTile * ((e.k1 - e.k0 + 1 + kch - 1) / kch);
    const double cost = (double)((n + resident - 1) / resident) * (kch + 2);
    if (cost <= best_cost) { best_cost = cost; best = kch; }
  }
  for (const auto &e : ext)
    for (int k = e.k0; k <= e.k1; k += best)
      for (long long q = 0; q < (long long)e.gx * e.gy; q += kTile) out.push_back(Tile{e.blk, k, 0, (int)q});
  return best;
}

// Line relaxation (mg_itrsch 2) on level g: room for every listed block's
// TDMA factors (six arrays of its cells, k_tdma_factor), pointed to from its
// table entry, and the shape of k_tdma_lines.  A block whose diagonals hold
// fewer than 32 lines is one CTA; larger ones take a cluster of 4 CTAs or
// more (below), each CTA owning a slice of at least 8 line positions of
// every diagonal.
static int tdma_layout(mf3d_ctx *C, View &V, int g, std::vector<BlkLev> &tab) {
  ViewLevel &L = V.lv[g];
  const int nb = (int)V.blk.size();
  L.td_fp64 = C->elem == 8 || (C->coarse64 && g >= V.Lmax);
  const size_t sz = L.td_fp64 ? 8 : 4;
  size_t bytes = 0;
  std::vector<size_t> off(nb, 0);
  int numax = 1, nmax = 1;
  L.td_lines[0] = L.td_lines[1] = L.td_lines[2] = 0;
  for (int b = 0; b < nb; ++b) {
    if (g > V.blk[b]->ngrid) continue;
    const BlkLev &B = tab[b];
    off[b] = bytes;
    bytes += ((size_t)6 * B.nx * B.ny * B.nz * sz + 255) / 256 * 256;
    numax = std::max(numax, std::max(B.nx, B.ny));
    nmax = std::max(nmax, std::max(B.nx, std::max(B.ny, B.nz)));
    L.td_lines[0] = std::max(L.td_lines[0], B.nx * B.nz);
    L.td_lines[1] = std::max(L.td_lines[1], B.ny * B.nz);
    L.td_lines[2] = std::max(L.td_lines[2], B.nx * B.ny);
  }
  int st;
  if ((st = L.tdf.alloc(std::max<size_t>(bytes, 256)))) return st;
  for (int b = 0; b < nb; ++b)
    if (g <= V.blk[b]->ngrid) tab[b].tdf = L.tdf.p + off[b];
  const size_t cap = 200 * 1024;
  // the kernel's limits (the attributes are the kernel's, not the launch's)
  void (*kern)(const BlkLev *, const int *, const int *, int, int, int) =
      L.td_fp64 ? (void (*)(const BlkLev *, const int *, const int *, int, int, int))k_tdma_lines<double>
                : (void (*)(const BlkLev *, const int *, const int *, int, int, int))k_tdma_lines<float>;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap));
  // shape for cl CTAs per block: lines staged at a time and shared memory
  auto shape = [&](int cl, int &gmax, size_t &smem) {
    const int per = (numax + cl - 1) / cl;
    gmax = (int)std::max<size_t>(1, std::min<size_t>(per, cap / ((7 * (size_t)nmax + 9) * sz)));
    smem = (7 * (size_t)gmax * (nmax + 1) + 2 * (size_t)gmax) * sz;
  };
  // Up to 8 CTAs per block (portable clusters); more (non-portable, up to
  // 16) only where the device holds a cluster for every block of the level
  // at once - 16 with too few resident measured slower (18.1 against 11.2 ms
  // per finest-level relaxation of 2x2x2 blocks of 128^3; 12 CTAs, of which
  // fewer than 8 clusters fit: 19.6 ms).  There the query picks 10: 10.5 ms.
  L.td_cl = numax >= 32 ? std::min(8, numax / 8) : 1;
  int nblk = 0;
  for (int b = 0; b < nb; ++b) nblk += g <= V.blk[b]->ngrid;
  if (numax >= 128 && cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
    for (int cl = std::min(16, numax / 8); cl > 8; --cl) {
      int gm;
      size_t sm;
      shape(cl, gm, sm);
      cudaLaunchAttribute at;
      at.id = cudaLaunchAttributeClusterDimension;
      at.val.clusterDim.x = (unsigned)cl;
      at.val.clusterDim.y = at.val.clusterDim.z = 1;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)cl);
      cfg.blockDim = dim3(TD_THREADS);
      cfg.dynamicSmemBytes = sm;
      cfg.attrs = &at;
      cfg.numAttrs = 1;
      int ncl = 0;
      if (cudaOccupancyMaxActiveClusters(&ncl, kern, &cfg) == cudaSuccess && ncl >= nblk) {
        L.td_cl = cl;
        break;
      }
    }
    cudaGetLastError();  // a refused query leaves no error behind
  }
  if (const char *e = std::getenv("MF3D_TD_CLUSTER")) L.td_cl = std::max(1, std::min(16, std::atoi(e)));  // tuning
  shape(L.td_cl, L.td_gmax, L.td_smem);
  L.td_nmax = nmax;
  L.td_numax = numax;
  if (L.td_smem > cap) {
    set_error("line relaxation: a line of " + std::to_string(nmax) + " cells does not fit in shared memory");
    return MF3D_E_UNSUPPORTED;
  }
  return MF3D_OK;
}

// The TDMA factors of every level of the view (after its coefficients).
static void tdma_factors(mf3d_ctx *C, View &V) {
  for (int g = 1; g <= V.Lmax; ++g) {
    ViewLevel &L = V.lv[g];
    if (!L.n_list[SUB_A]) continue;
    for (int dir = 0; dir < 3; ++dir) {
      const dim3 grid((unsigned)((L.td_lines[dir] + 127) / 128), (unsigned)L.n_list[SUB_A]);
      if (L.td_fp64) launch(k_tdma_factor<double>, grid, 128, 0, C->stream, L.tab.p, L.list[SUB_A].p, dir);
      else launch(k_tdma_factor<float>, grid, 128, 0, C->stream, L.tab.p, L.list[SUB_A].p, dir);
      ++C->launches;
    }
  }
}

// The coarse levels of a red-black V-cycle as one cluster launch
// (k_coarse_cycle): a view over one domain of at most CC_MAX_BLOCKS blocks,
// with ir >= 1; g0 = the finest level from which every block's levels (phi
// and rhs) and halo staging fit one CTA's shared memory.  The domain's halo
// pairs of those levels are regrouped by destination block.
// MF3D_COARSE_CLUSTER=0 turns it off.
constexpr size_t kCcSmemCap = 200 * 1024;
static int coarse_cycle_plan(mf3d_ctx *C, View &V) {
  V.cc_g0 = 0;
  if (C->lmr) return MF3D_OK;  // the cluster kernel holds no LMR halo programs
  const char *e = std::getenv("MF3D_COARSE_CLUSTER");
  if (e && e[0] == '0') return MF3D_OK;
  const int nb = (int)V.blk.size();
  if (V.dom.size() != 1 || C->prm.mg_itrsch != 3 || C->prm.lsm || C->prm.irestr < 1 || nb > CC_MAX_BLOCKS ||
      V.Lmax < 3)
    return MF3D_OK;
  const DomainStore &D = *V.dom[0];
  const int Lc = C->coarse64 ? V.Lmax : V.Lmax + 1;
  auto elem_of = [&](int g) { return (C->elem == 8 || g >= Lc) ? 8 : 4; };
  int g0 = 0;
  size_t smem = 0;
  int bufn = 0;
  for (int g = 2; g < V.Lmax && !g0; ++g) {
    if (V.Lmax - g + 1 > CC_MAX_LEVELS) continue;
    int bn = 0;
    for (int l = g; l <= V.Lmax; ++l) {
      std::vector<int> cnt(nb, 0);
      for (const auto &h : D.halo[l]) cnt[h.dblk]++;
      for (int c : cnt) bn = std::max(bn, c);
    }
    size_t worst = 0;
    for (int b = 0; b < nb; ++b) {
      long long bytes = 0, coef = 0;
      for (int l = g; l <= V.Lmax; ++l) {
        bytes += 2 * cc_level_bytes(V.lv[l].htab[b], elem_of(l));
        coef += cc_coef_bytes(V.lv[l].htab[b], elem_of(l));
      }
      worst = std::max(worst, (size_t)((bytes + 15) / 16 * 16 + ((long long)bn * 8 + 15) / 16 * 16 + coef));
    }
    if (worst <= kCcSmemCap) { g0 = g; smem = worst; bufn = bn; }
  }
  if (!g0) return MF3D_OK;
  long long coef_off = 0;
  // the coefficient region follows the largest block's levels and halo
  // buffer (every CTA gets the same dynamic size)
  {
    long long worst = 0;
    for (int b = 0; b < nb; ++b) {
      long long bytes = 0;
      for (int l = g0; l <= V.Lmax; ++l) bytes += 2 * cc_level_bytes(V.lv[l].htab[b], elem_of(l));
      worst = std::max(worst, (bytes + 15) / 16 * 16 + ((long long)bufn * 8 + 15) / 16 * 16);
    }
    coef_off = worst;
    long long coef = 0;
    for (int b = 0; b < nb; ++b) {
      long long c = 0;
      for (int l = g0; l <= V.Lmax; ++l) c += cc_coef_bytes(V.lv[l].htab[b], elem_of(l));
      coef = std::max(coef, c);
    }
    smem = (size_t)(worst + coef);
    if (smem > kCcSmemCap) return MF3D_OK;  // the launch path stays
  }
  void (*kern)(const CcArgs, const int *) = C->elem == 8 ? k_coarse_cycle<double> : k_coarse_cycle<float>;
  // the device holds such a cluster at all (else the launch path stays)
  {
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeClusterDimension;
    at.val.clusterDim.x = (unsigned)nb;
    at.val.clusterDim.y = at.val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)nb);
    cfg.blockDim = dim3(CC_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.attrs = &at;
    cfg.numAttrs = 1;
    int ncl = 0;
    if (cudaOccupancyMaxActiveClusters(&ncl, kern, &cfg) != cudaSuccess || ncl < 1) {
      cudaGetLastError();
      return MF3D_OK;
    }
  }
  // halo pairs of the held levels grouped by destination block
  std::vector<HaloCopy> pairs;
  std::vector<CcHalo> hs((size_t)(V.Lmax - g0 + 1) * nb);
  std::vector<long long> start(hs.size());
  for (int l = g0; l <= V.Lmax; ++l)
    for (int b = 0; b < nb; ++b) {
      start[(size_t)(l - g0) * nb + b] = (long long)pairs.size();
      for (const auto &h : D.halo[l])
        if (h.dblk == b) pairs.push_back(HaloCopy{h.dblk, h.doff, h.sblk, h.soff});
      hs[(size_t)(l - g0) * nb + b].n = (int)(pairs.size() - start[(size_t)(l - g0) * nb + b]);
    }
  int st;
  if ((st = V.cc_pairs.upload(pairs, C->stream))) return st;
  for (size_t q = 0; q < hs.size(); ++q) hs[q].pairs = V.cc_pairs.p + start[q];
  if ((st = V.cc_halo.upload(hs, C->stream))) return st;
  CcArgs &a = V.cc_args;
  std::memset(&a, 0, sizeof a);
  for (int l = g0; l <= V.Lmax; ++l) a.tab[l - g0] = V.lv[l].tab.p;
  a.halo = V.cc_halo.p;
  a.blk0 = 0;
  a.nb = nb;
  a.nlev = V.Lmax - g0 + 1;
  a.g0 = g0;
  a.lc = Lc;
  a.ir = C->prm.irestr;
  a.ip = C->prm.iproln;
  a.dom = 0;
  a.bufn = bufn;
  a.coef_off = coef_off;
  V.cc_g0 = g0;
  V.cc_smem = smem;
  CK(cudaStreamSynchronize(C->stream));  // the host vectors are locals
  return MF3D_OK;
}

// The phases of the middle levels (k_mid_cycle), in vcycle's order: down,
// for levels 2 .. gtop, the pre-smoothing of every present block (the first
// red half-sweep came with the restriction into the level), the extra
// sweeps of blocks bottoming out there, the restriction into the next
// level; up, from the level above the cluster (or the one above the
// coarsest) to 2, the prolongation from below and the post-smoothing.  Red-
// black smoothing without L_LSM, levels of one element type, the levels'
// items below 2^31; otherwise the launch path stays.
static int mid_cycle_plan(mf3d_ctx *C, View &V) {
  V.mid_on = false;
  if (C->lmr) return MF3D_OK;
  // off unless MF3D_MID_CYCLE=1: on 2x2x2 blocks of 128^3 the launch path
  // measured 85.7 ms a solve against 92.9 for this one (its grid barriers
  // cost more than the launches they replace)
  const char *e = std::getenv("MF3D_MID_CYCLE");
  if (!(e && e[0] == '1')) return MF3D_OK;
  const int sch = C->prm.mg_itrsch, ir = C->prm.irestr, ip = C->prm.iproln;
  if (sch != 3 || C->prm.lsm || V.Lmax < 2 || ir < 1) return MF3D_OK;
  const int Lc = C->coarse64 ? V.Lmax : V.Lmax + 1;
  const int gtop = V.cc_g0 ? V.cc_g0 - 1 : V.Lmax;
  if (gtop < 2) return MF3D_OK;
  const int glast = V.cc_g0 ? V.cc_g0 : V.Lmax;  // deepest level a mid phase touches
  const bool f64 = C->elem == 8;
  if (!f64)
    for (int g = 2; g <= glast; ++g)
      if (g >= Lc) return MF3D_OK;  // an FP64 coarsest level among FP32 ones: the launch path
  int occ = 0;
  void (*kern)(const MidPhase *, int, const int *, MidBar *, int *) = f64 ? k_mid_cycle<double> : k_mid_cycle<float>;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, MID_THREADS, 0) != cudaSuccess || occ < 1) {
    cudaGetLastError();
    return MF3D_OK;
  }
  std::vector<MidPhase> down, up;
  int st;
  // a device list of blocks and its item prefix
  auto make_list = [&](const std::vector<int> &blocks, const std::function<long long(int)> &items,
                       const int *&lp, const long long *&pp, int &n, long long &total) -> int {
    std::vector<long long> pre(1, 0);
    for (int b : blocks) pre.push_back(pre.back() + items(b));
    n = (int)blocks.size();
    total = pre.back();
    V.mid_lists.emplace_back();
    V.mid_pres.emplace_back();
    int r;
    if ((r = V.mid_lists.back().upload(blocks, C->stream))) return r;
    if ((r = V.mid_pres.back().upload(pre, C->stream))) return r;
    lp = V.mid_lists.back().p;
    pp = V.mid_pres.back().p;
    return MF3D_OK;
  };
  auto add_sweeps = [&](std::vector<MidPhase> &out, int g, int q, int it, bool fz, bool red_done) -> int {
    ViewLevel &L = V.lv[g];
    if (!L.n_list[q] || it <= 0) return MF3D_OK;
    MidPhase sw = {};
    sw.kind = MID_SWEEP;
    sw.tab = L.tab.p;
    int r;
    if ((r = make_list(L.hblk[q], [&](int b) { const BlkLev &B = L.htab[b]; return (long long)((B.nx + 1) / 2) * B.ny * B.nz; },
                       sw.list, sw.pre, sw.nlist, sw.items)))
      return r;
    for (int itr = 0; itr < it; ++itr) {
      const bool f = fz && itr == 0;
      if (!(f && red_done)) {
        MidPhase red = sw;
        red.colour = 0;
        red.fz = f ? 1 : 0;
        out.push_back(red);
      }
      MidPhase black = sw;
      black.colour = 1;
      black.fz = 0;
      out.push_back(black);
      if (L.n_halo[q]) {
        MidPhase h = {};
        h.tab = L.tab.p;
        h.seg = L.hseg[q].p;
        h.nseg = L.n_hseg[q];
        h.nstaged = L.n_staged[q];
        h.items = L.n_halo[q];
        h.buf = L.stage[q].p;
        if (L.n_staged[q]) {
          h.kind = MID_HALO_STAGE;
          out.push_back(h);
        }
        h.kind = MID_HALO_APPLY;
        out.push_back(h);
      }
    }
    return MF3D_OK;
  };
  for (int g = 2; g <= gtop; ++g) {
    if ((st = add_sweeps(down, g, SUB_A, ir, true, true))) return st;
    if ((st = add_sweeps(down, g, SUB_C, ip, ir == 0, false))) return st;
    if (g < V.Lmax && V.lv[g + 1].n_list[SUB_A]) {
      ViewLevel &Cl = V.lv[g + 1];
      MidPhase rs = {};
      rs.kind = MID_RESTRICT;
      rs.tab = V.lv[g].tab.p;
      rs.tab2 = Cl.tab.p;
      if ((st = make_list(Cl.hblk[SUB_A], [&](int b) { const BlkLev &B = Cl.htab[b]; return (long long)(B.nx + 2) * (B.ny + 2) * (B.nz + 2); },
                          rs.list, rs.pre, rs.nlist, rs.items)))
        return st;
      down.push_back(rs);
    }
  }
  for (int g = V.cc_g0 ? gtop : V.Lmax - 1; g >= 2; --g) {
    ViewLevel &F = V.lv[g], &Cl = V.lv[g + 1];
    if (F.n_list[SUB_D]) {
      MidPhase pr = {};
      pr.kind = MID_PROLONG;
      pr.tab = F.tab.p;
      pr.tab2 = Cl.tab.p;
      if ((st = make_list(F.hblk[SUB_D], [&](int b) { const BlkLev &B = Cl.htab[b]; return (long long)(B.nx + 1) * (B.ny + 1) * (B.nz + 1); },
                          pr.list, pr.pre, pr.nlist, pr.items)))
        return st;
      up.push_back(pr);
    }
    if ((st = add_sweeps(up, g, SUB_D, ip, false, false))) return st;
  }
  // the kernel splits item indices with 32-bit high multiplies: exact while
  // a block's items times the divisor (a row or plane extent) stay below 2^32
  for (const auto &ph : down)
    if (ph.items >= (1LL << 31) || ph.nlist > MID_MAX_LIST) return MF3D_OK;
  for (const auto &ph : up)
    if (ph.items >= (1LL << 31) || ph.nlist > MID_MAX_LIST) return MF3D_OK;
  for (int g = 2; g <= glast; ++g)
    for (const BlkLev &B : V.lv[g].htab)
      if ((long long)(B.nx + 2) * (B.ny + 2) * (B.nz + 2) * (std::max(B.nx, B.ny) + 2) >= (1LL << 32)) return MF3D_OK;
  if ((st = V.mid_down.upload(down, C->stream))) return st;
  if ((st = V.mid_up.upload(up, C->stream))) return st;
  if ((st = V.mid_bar.alloc(1))) return st;
  CK(cudaMemsetAsync(V.mid_bar.p, 0, sizeof(MidBar), C->stream));
  CK(cudaStreamSynchronize(C->stream));  // the host vectors are locals
  V.n_mid_down = (int)down.size();
  V.n_mid_up = (int)up.size();
  V.mid_grid = C->nsm * std::min(occ, MID_CTAS_PER_SM);
  V.mid_on = V.n_mid_down > 0;
  return MF3D_OK;
}

// Build the launch tables of a view over `doms` (all of one precision).
static int build_view(mf3d_ctx *C, View &V, const std::vector<DomainStore *> &doms, int hcap) {
  cudaStream_t s = C->stream;
  V.drop_graphs();
  V.blk.clear(); V.blk_dom.clear(); V.dom = doms; V.Lmax = 0; V.n_l1 = 0;
  std::vector<int> dom_base;
  for (size_t d = 0; d < doms.size(); ++d) {
    dom_base.push_back((int)V.blk.size());
    for (auto &b : doms[d]->blocks) {
      V.blk.push_back(b.get());
      V.blk_dom.push_back((int)d);
    }
    V.Lmax = std::max(V.Lmax, doms[d]->ngrid);
  }
  const int nb = (int)V.blk.size(), nd = (int)doms.size();
  V.lv.clear();
  V.lv.resize(V.Lmax + 1);
  int st;
  for (int g = 1; g <= V.Lmax; ++g) {
    ViewLevel &L = V.lv[g];
    std::vector<BlkLev> tab(nb);
    std::vector<RbSeg> sw[3];
    std::vector<Tile> ce[3];
    std::vector<int> li[3], sblk[3];
    for (int b = 0; b < nb; ++b) {
      const BlockStore &S = *V.blk[b];
      BlkLev B;
      std::memset(&B, 0, sizeof B);
      if (g <= S.ngrid) B = S.lv[g].desc;
      B.dom = V.blk_dom[b];
      tab[b] = B;
      if (g > S.ngrid) continue;
      const int sub_extra = (g == S.ngrid) ? SUB_C : SUB_D;
      const Box bce{0, B.nx + 1, 0, B.ny + 1, 0, B.nz + 1};
      for (int q : {(int)SUB_A, sub_extra}) {
        sblk[q].push_back(b);
        add_tiles_2d(ce[q], b, bce, RW_TX, RW_RJ, RW_KCH);
        li[q].push_back(b);
        L.cells_sub[q] += (long long)B.nx * B.ny * B.nz;
      }
    }
    if (C->prm.mg_itrsch == 2 && (st = tdma_layout(C, V, g, tab))) return st;
    if (C->prm.mg_itrsch == 1) {
      // slices of k of at least 8 planes: up to 8 CTAs per block, up to 16
      // (non-portable) where the device holds a cluster for every block at once
      int nzmax = 1, nblk = 0;
      for (int b = 0; b < nb; ++b)
        if (g <= V.blk[b]->ngrid) { nzmax = std::max(nzmax, tab[b].nz); ++nblk; }
      L.lx_cl = nzmax >= 32 ? std::min(8, nzmax / 8) : 1;
      void (*kern)(const BlkLev *, const int *, const int *, int) =
          C->elem == 8 ? (void (*)(const BlkLev *, const int *, const int *, int))k_lexgs<double>
                       : (void (*)(const BlkLev *, const int *, const int *, int))k_lexgs<float>;
      if (nzmax >= 128 && cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
        for (int cl = std::min(16, nzmax / 8); cl > 8; --cl) {
          cudaLaunchAttribute at;
          at.id = cudaLaunchAttributeClusterDimension;
          at.val.clusterDim.x = (unsigned)cl;
          at.val.clusterDim.y = at.val.clusterDim.z = 1;
          cudaLaunchConfig_t cfg = {};
          cfg.gridDim = dim3((unsigned)cl);
          cfg.blockDim = dim3(1024);
          cfg.attrs = &at;
          cfg.numAttrs = 1;
          int ncl = 0;
          if (cudaOccupancyMaxActiveClusters(&ncl, kern, &cfg) == cudaSuccess && ncl >= nblk) {
            L.lx_cl = cl;
            break;
          }
        }
        cudaGetLastError();  // a refused query leaves no error behind
      }
      if (const char *e = std::getenv("MF3D_LX_CLUSTER")) L.lx_cl = std::max(1, std::min(16, std::atoi(e)));  // tuning
    }
    if ((st = L.tab.upload(tab, s))) return st;
    {
      // restriction into level g (g > 1): every block present here; prolongation
      // from level g+1 into g: every block continuing down
      std::vector<PlaneExt> re, pe;
      std::vector<int> inj, add, rblk;
      std::vector<long long> inj_pre(1, 0), add_pre(1, 0);
      for (int b = 0; b < nb; ++b) {
        const BlkLev &B = tab[b];
        const BlockStore &S = *V.blk[b];
        if (g > S.ngrid) continue;
        const long long cells = (long long)(B.nx + 2) * (B.ny + 2) * (B.nz + 2);
        if (g > 1 && g > S.own) {  // LMR: into a level of the same size
          inj.push_back(b);
          inj_pre.push_back(inj_pre.back() + cells);
        } else if (g > 1) {
          re.push_back(PlaneExt{b, B.nx + 2, B.ny + 2, 0, B.nz + 1});
        }
        if (g < S.ngrid && g >= S.own) {  // LMR: from a level of the same size
          add.push_back(b);
          add_pre.push_back(add_pre.back() + cells);
        } else if (g < S.ngrid) {
          pe.push_back(PlaneExt{b, B.nx / 2 + 1, B.ny / 2 + 1, 0, B.nz / 2});
        }
      }
      for (int b : sblk[SUB_A])
        if (!(g > 1 && g > V.blk[b]->own)) rblk.push_back(b);
      L.n_inj = (int)inj.size();
      L.n_add = (int)add.size();
      L.inj_items = inj_pre.back();
      L.add_items = add_pre.back();
      if ((st = L.inj_list.upload(inj, s))) return st;
      if ((st = L.inj_pre.upload(inj_pre, s))) return st;
      if ((st = L.add_list.upload(add, s))) return st;
      if ((st = L.add_pre.upload(add_pre, s))) return st;
      std::vector<Tile> rt, pt;
      L.rkch = plane_tiles(C, re, rt);
      L.pkch = plane_tiles(C, pe, pt);
      L.n_rtile = (int)rt.size();
      L.n_ptile = (int)pt.size();
      if ((st = L.rtile.upload(rt, s))) return st;
      if ((st = L.ptile.upload(pt, s))) return st;
      std::vector<Tile> rm;
      if (g > 1 && !rblk.empty()) L.rtma_kch = rtma_tiles(C, tab, rblk, 0, rm);
      L.n_rtma = (int)rm.size();
      if ((st = L.rtma.upload(rm, s))) return st;
    }
    // level 1 always takes the pipelined sweep; MF3D_SMALL_LEVEL_CELLS overrides the limit
    long long small_limit = kSmallLevelCells;
    if (const char *e = std::getenv("MF3D_SMALL_LEVEL_CELLS")) small_limit = std::atoll(e);
    // under L_LSM every level sweeps with the plain-load kernel (per-cell coefficients)
    L.small = C->prm.lsm || (g > 1 && L.cells_sub[SUB_A] <= small_limit);
    for (int q = 0; q < 3; ++q) {
      std::vector<int> pre(1, 0);
      for (int b : li[q]) {
        const BlkLev &B = tab[b];
        pre.push_back(pre.back() + ((B.nx + 1) / 2) * B.ny * B.nz);
      }
      L.small_items[q] = pre.back();
      if ((st = L.spre[q].upload(pre, s))) return st;
    }
    L.htab = tab;
    for (int q = 0; q < 3; ++q) {
      L.hblk[q] = sblk[q];
      std::vector<int> sf;
      L.n_sweep[q] = sweep_segments(C, tab, sblk[q], sw[q], sf, L.sched);
      if ((st = L.sfirst[q].upload(sf, s))) return st;
      L.n_cells[q] = (int)ce[q].size();
      L.n_list[q] = (int)li[q].size();
      if ((st = L.sweep[q].upload(sw[q], s))) return st;
      if ((st = L.cells[q].upload(ce[q], s))) return st;
      if ((st = L.list[q].upload(li[q], s))) return st;
    }
    // LMR: the level's halo program (single-domain views)
    L.lmr_depth.clear();
    L.lmr_nwrites = 0;
    if (nd == 1 && (int)doms[0]->lmr.size() > g && !doms[0]->lmr[g].depth_start.empty()) {
      const DomainStore::LmrLevel &M = doms[0]->lmr[g];
      L.lmr_terms = M.terms.p;
      L.lmr_nodes = M.nodes.p;
      L.lmr_writes = M.writes.p;
      L.lmr_depth = M.depth_start;
      L.lmr_nwrites = M.n_writes;
      if ((st = L.lmr_val.alloc((size_t)std::max(M.depth_start.back(), 1)))) return st;
    }
    // halo segments: the domains' resident pair lists
    for (int q = 0; q < 3; ++q) {
      std::vector<HaloSeg> segs;
      long long n = 0, ns = 0;
      for (int d = 0; d < nd; ++d) {
        const DomainStore &D = *doms[d];
        if (g > D.ngrid) continue;
        const bool in = q == SUB_A || (q == SUB_C ? g == D.ngrid : g < D.ngrid);
        if (!in || D.halo[g].empty()) continue;
        HaloSeg sg;
        sg.pairs = D.dhalo[g].p;
        sg.start = n;
        sg.sstart = ns;
        sg.n = (int)D.halo[g].size();
        sg.nstaged = D.nstaged[g];
        sg.blk_base = dom_base[d];
        sg.dom = d;
        n += sg.n;
        ns += sg.nstaged;
        segs.push_back(sg);
      }
      L.n_hseg[q] = (int)segs.size();
      L.n_halo[q] = n;
      L.n_staged[q] = ns;
      if ((st = L.hseg[q].upload(segs, s))) return st;
      if ((st = L.stage[q].alloc((size_t)std::max<long long>(ns, 1) * 8))) return st;
    }
  }
  // level-1 field tables
  V.hf.resize(nb);
  std::vector<Tile> t1, t2, t5;
  std::vector<long long> it_faces, it_planes, it_vfaces, it_bcax[3];
  for (int b = 0; b < nb; ++b) {
    const BlockStore &S = *V.blk[b];
    BlkFld F = S.fld;
    const int d = V.blk_dom[b];
    F.dom = d;
    F.L1 = S.lv[1].desc;
    F.L1.dom = d;
    for (int f = 0; f < 6; ++f) {
      const FaceRule &r = doms[d]->rules[6 * (b - dom_base[d]) + f];
      F.wall[f] = r.kind == FACE_WALL;
      F.src[f] = r.kind == FACE_WALL ? b : dom_base[d] + r.src;
    }
    V.hf[b] = F;
    V.wall_law |= F.wtau != nullptr;
    const mf3d_block_desc &x = S.d;
    add_tiles_2d(t1, b, Box{1, x.nx, 1, x.ny, 1, x.nz}, RW_TX, RW_RJ, RW_KCH);
    add_tiles_2d(t2, b, Box{0, x.nx + 1, 0, x.ny + 1, 0, x.nz + 1}, RW_TX, RW_RJ, RW_KCH);
    add_tiles_2d(t5, b, Box{1, x.nx, 1, x.ny, 1, x.nz}, OZ_TX, OZ_RJ, OZ_KCH);
    it_faces.push_back(2 * ((long long)x.ny * x.nz + (long long)x.nx * x.nz + (long long)x.nx * x.ny));
    it_planes.push_back((long long)x.ny * x.nz + (long long)x.nx * x.nz + (long long)x.nx * x.ny);
    it_vfaces.push_back((long long)(C->prm.pl_ex + 1) * it_faces.back());
    {
      const long long ti = x.nx + 2 * (long long)F.pl, tj = x.ny + 2 * (long long)F.pl, tk = x.nz + 2 * (long long)F.pl;
      it_bcax[0].push_back(6 * tj * tk);
      it_bcax[1].push_back(6 * ti * tk);
      it_bcax[2].push_back(6 * ti * tj);
      for (int f = 0; f < 6; ++f) V.bc_periodic[f / 2] |= F.pface[f] != 0;
    }
    V.n_l1 += (long long)x.nx * x.ny * x.nz;
  }
  {
    std::vector<PlaneExt> pe;
    for (int b = 0; b < nb; ++b) {
      const mf3d_block_desc &x = V.blk[b]->d;
      pe.push_back(PlaneExt{b, (x.nx + 3) / 2, x.ny + 2, 0, x.nz + 1});
    }
    std::vector<Tile> tp;
    V.pairs_kch = plane_tiles(C, pe, tp);
    V.n_pairs = (int)tp.size();
    if ((st = V.t_pairs.upload(tp, s))) return st;
  }
  auto t3 = make_tiles(it_faces), t4 = make_tiles(it_planes), t6 = make_tiles(it_vfaces);
  V.n_int = (int)t1.size(); V.n_l1cells = (int)t2.size(); V.n_faces = (int)t3.size();
  V.n_planes = (int)t4.size(); V.n_zint = (int)t5.size(); V.n_vfaces = (int)t6.size();
  if ((st = V.df.upload(V.hf, s))) return st;
  if ((st = V.t_int.upload(t1, s))) return st;
  if ((st = V.t_zint.upload(t5, s))) return st;
  if ((st = V.t_l1cells.upload(t2, s))) return st;
  if ((st = V.t_faces.upload(t3, s))) return st;
  if ((st = V.t_planes.upload(t4, s))) return st;
  if ((st = V.t_vfaces.upload(t6, s))) return st;
  if (C->prm.bounds)
    for (int a = 0; a < 3; ++a) {
      auto tb = make_tiles(it_bcax[a]);
      V.n_bcax[a] = (int)tb.size();
      if ((st = V.t_bcax[a].upload(tb, s))) return st;
    }
  if ((st = coarse_cycle_plan(C, V))) return st;
  if ((st = mid_cycle_plan(C, V))) return st;
  V.fx_uvw = V.fx_p = V.fxe_sub = V.fxe_chain = nullptr;
  V.fxe_cells = nullptr;
  V.nfx_uvw = V.nsfx_uvw = V.nfx_p = V.nsfx_p = 0;
  V.nfxe_sub = V.nsfxe_sub = V.nfxe_chain = V.nfxe_cells = 0;
  V.fx_per_iteration = false;
  if (nd == 1 && doms[0]->nfx_uvw + doms[0]->nfx_p > 0) {
    const DomainStore &D = *doms[0];
    V.fx_uvw = D.fx_uvw.p; V.nfx_uvw = D.nfx_uvw; V.nsfx_uvw = D.nsfx_uvw;
    V.fx_p = D.fx_p.p; V.nfx_p = D.nfx_p; V.nsfx_p = D.nsfx_p;
    V.fxe_sub = D.fxe_sub.p; V.nfxe_sub = D.nfxe_sub; V.nsfxe_sub = D.nsfxe_sub;
    V.fxe_chain = D.fxe_chain.p; V.nfxe_chain = D.nfxe_chain;
    V.fxe_cells = D.fxe_cells.p; V.nfxe_cells = D.nfxe_cells;
    V.fx_per_iteration = D.fx_per_iteration;
    const long long ns = std::max(std::max(V.nsfx_uvw, V.nsfx_p), V.nsfxe_sub);
    if ((st = V.fx_stage.alloc((size_t)std::max<long long>(ns, 1)))) return st;
    if ((st = V.fx_prev.alloc((size_t)std::max<long long>(V.nfxe_chain, 1)))) return st;
  }
  // per-domain solve state
  std::vector<int> ones(std::max(nd, 1), 1);
  if ((st = V.ds.alloc(std::max(nd, 1)))) return st;
  if ((st = V.act.upload(ones, s))) return st;
  if ((st = V.ones.upload(ones, s))) return st;
  if ((st = V.err.alloc(1))) return st;
  CK(cudaMemsetAsync(V.err.p, 0, sizeof(int), s));
  if ((st = V.budget.alloc(1))) return st;
  CK(cudaMemsetAsync(V.budget.p, 0, sizeof(int), s));
  if ((st = V.rmax.alloc(std::max(nd, 1)))) return st;
  if ((st = V.rmax_scratch.alloc(std::max(nd, 1)))) return st;
  CK(cudaMemsetAsync(V.rmax.p, 0, V.rmax.n * sizeof(unsigned long long), s));
  V.hcap = std::max(hcap, 1);
  if ((st = V.hist.alloc((size_t)std::max(nd, 1) * V.hcap))) return st;
  // the line relaxation's factors; under L_LSM every solve forms them anew
  if (C->prm.mg_itrsch == 2 && !C->prm.lsm) tdma_factors(C, V);
  CK(cudaStreamSynchronize(s));
  return MF3D_OK;
}

// ---------------------------------------------------------------------------
// V-cycle over a view.
// ---------------------------------------------------------------------------
template <typename T>
static void halo(mf3d_ctx *C, View &V, int g, int q) {
  ViewLevel &L = V.lv[g];
  if (!L.lmr_depth.empty()) {
    // LMR: the nodes depth by depth from the pre-exchange state, then the writes
    for (size_t d = 1; d < L.lmr_depth.size(); ++d) {
      const int n0 = L.lmr_depth[d - 1], n1 = L.lmr_depth[d];
      if (n1 <= n0) continue;
      launch(k_lmr_nodes<T>, grid_of(n1 - n0, 256), 256, 0, C->stream, L.tab.p, (int)V.blk.size(), L.lmr_terms,
             L.lmr_nodes, n0, n1, L.lmr_val.p);
      ++C->launches;
    }
    if (L.lmr_nwrites) {
      launch(k_lmr_write<T>, grid_of(L.lmr_nwrites, 256), 256, 0, C->stream, L.tab.p, (int)V.blk.size(),
             L.lmr_writes, L.lmr_nwrites, (const double *)L.lmr_val.p);
      ++C->launches;
    }
    return;
  }
  if (!L.n_halo[q]) return;
  T *buf = (T *)L.stage[q].p;
  if (L.n_staged[q]) {
    launch(k_halo_stage<T>, grid_of(L.n_staged[q], 256), 256, 0, C->stream, L.tab.p, L.hseg[q].p, L.n_hseg[q],
                                                                       L.n_staged[q], V.act.p, buf);
    ++C->launches;
  }
  launch(k_halo_apply<T>, grid_of(L.n_halo[q], 256), 256, 0, C->stream, L.tab.p, L.hseg[q].p, L.n_hseg[q],
                                                                   L.n_halo[q], V.act.p, buf);
  ++C->launches;
}

// mgrelax(g, it) (mgsolver.for:371-617) on subset q: `it` sweeps, each
// followed by the halo refresh (mgbound + exchangepp + exchbc_mgpp).
template <typename T>
static void relax(mf3d_ctx *C, View &V, int g, int q, int it, bool from_zero, bool red_done = false) {
  ViewLevel &L = V.lv[g];
  if (!L.n_list[q]) return;
  const int sch = C->prm.mg_itrsch;
  for (int itr = 0; itr < it; ++itr) {
    if (sch == 3) {
      // timed (mf3d_profile): level 1's half-sweeps that read the other
      // colour, rhs and write their own (12 B per cell in FP64), pre- and
      // post-smoothing; not the from-zero red half-sweep (8 B per cell)
      const int pk = (g == 1 && q != SUB_C) ? MF3D_PROF_SMOOTH_L1 : 0;
      const double half = 0.5 * (double)L.cells_sub[q] * sizeof(T);
      const bool fz = from_zero && itr == 0;
      const bool skip_red = fz && red_done;  // the restriction formed the red half-sweep
      prof_begin(C, fz ? 0 : pk, 3 * half);
      const dim3 grid(L.n_sweep[q]), cta(RB_TX, RB_TY);
      if (L.small) {
        const int g2 = grid_of(L.small_items[q], kTile);
        if (skip_red)
          ;
        else if (fz)
          launch(k_rbgs_small<T, true>, g2, kTile, 0, C->stream, L.tab.p, L.spre[q].p, L.list[q].p, L.n_list[q], V.act.p, 0);
        else
          launch(k_rbgs_small<T, false>, g2, kTile, 0, C->stream, L.tab.p, L.spre[q].p, L.list[q].p, L.n_list[q], V.act.p,
                                                             0);
        prof_end(C, fz ? 0 : pk);
        prof_begin(C, pk, 3 * half);
        launch(k_rbgs_small<T, false>, g2, kTile, 0, C->stream, L.tab.p, L.spre[q].p, L.list[q].p, L.n_list[q], V.act.p, 1);
        prof_end(C, pk);
        C->launches += skip_red ? 1 : 2;
        halo<T>(C, V, g, q);
        continue;
      }
      if (skip_red)
        ;
      else if (fz)
        launch(k_rbgs<T, true>, grid, cta, 0, C->stream, L.tab.p, L.sweep[q].p, L.sfirst[q].p, V.act.p, 0, V.err.p);
      else
        launch(k_rbgs<T, false>, grid, cta, 0, C->stream, L.tab.p, L.sweep[q].p, L.sfirst[q].p, V.act.p, 0, V.err.p);
      prof_end(C, fz ? 0 : pk);
      prof_begin(C, pk, 3 * half);
      launch(k_rbgs<T, false>, grid, cta, 0, C->stream, L.tab.p, L.sweep[q].p, L.sfirst[q].p, V.act.p, 1, V.err.p);
      prof_end(C, pk);
      C->launches += skip_red ? 1 : 2;
    } else if (sch == 1) {
      launch_cl(k_lexgs<T>, L.n_list[q] * L.lx_cl, 1024, 0, C->stream, L.lx_cl, L.tab.p, L.list[q].p, V.act.p,
                L.lx_cl);
      ++C->launches;
    } else {
      // three passes, each reading rhs and phi and writing phi once
      const int pk = (g == 1 && q == SUB_A) ? MF3D_PROF_SMOOTH_L1 : 0;
      prof_begin(C, pk, 9.0 * (double)L.cells_sub[q] * sizeof(T));
      launch_cl(k_tdma_lines<T>, L.n_list[q] * L.td_cl, TD_THREADS, L.td_smem, C->stream, L.td_cl, L.tab.p,
                L.list[q].p, V.act.p, L.td_cl, L.td_gmax, L.td_nmax);
      prof_end(C, pk);
      ++C->launches;
    }
    halo<T>(C, V, g, q);
  }
}

template <typename T, typename TC>
static void restr(mf3d_ctx *C, View &V, int g) {  // level g -> g+1, blocks continuing down
  ViewLevel &F = V.lv[g], &Cl = V.lv[g + 1];
  if (Cl.n_inj) {  // LMR: blocks past their own last level
    launch(k_lmr_inject<T, TC>, grid_of(Cl.inj_items, 256), 256, 0, C->stream, F.tab.p, Cl.tab.p, Cl.inj_list.p,
           Cl.inj_pre.p, Cl.n_inj, V.act.p, (C->prm.mg_itrsch == 3 && C->prm.irestr > 0) ? 1 : 0);
    ++C->launches;
  }
  if (!Cl.n_rtile) return;
  const int pk = g == 1 ? MF3D_PROF_RESTRICT_L1 : 0;
  prof_begin(C, pk, (double)F.cells_sub[SUB_D] * sizeof(T) * (2.0 + 2.0 / 8.0));  // fine phi, rhs in; coarse out
  if (C->prm.mg_itrsch == 3 && C->prm.irestr > 0 && Cl.n_rtma && !C->prm.lsm) {
    // red-black from zero: the coarse interior phi is never read before it
    // is written, so only its ghost shell is zeroed (the kernel's shared
    // memory limit is raised on the context's device in ctx_init)
    launch(k_restrict_tma<T, TC>, Cl.n_rtma, kTile, RsShape<T>::SMEM, C->stream, F.tab.p, Cl.tab.p, Cl.rtma.p, V.act.p,
                                                                              Cl.rtma_kch, V.err.p, 1);
    prof_end(C, pk);
    ++C->launches;
    return;
  }
  launch(k_restrict<T, TC>, Cl.n_rtile, kTile, 0, C->stream, F.tab.p, Cl.tab.p, Cl.rtile.p, V.act.p, Cl.rkch,
         (C->prm.mg_itrsch == 3 && C->prm.irestr > 0) ? 1 : 0);
  prof_end(C, pk);
  ++C->launches;
}

template <typename T, typename TC>
static void corr(mf3d_ctx *C, View &V, int g) {  // level g+1 -> g, blocks continuing down
  ViewLevel &F = V.lv[g], &Cl = V.lv[g + 1];
  if (F.n_add) {  // LMR: blocks past their own last level
    for (int mode = 0; mode < 2; ++mode)
      launch(k_lmr_add<T, TC>, grid_of(F.add_items, 256), 256, 0, C->stream, F.tab.p, Cl.tab.p, F.add_list.p,
             F.add_pre.p, F.n_add, V.act.p, mode);
    C->launches += 2;
  }
  if (!F.n_ptile) return;
  const int pk = g == 1 ? MF3D_PROF_PROLONG_L1 : 0;
  prof_begin(C, pk, (double)F.cells_sub[SUB_D] * sizeof(T) * (2.0 + 1.0 / 8.0));  // fine in/out, coarse in
  launch(k_prolong<T, TC>, F.n_ptile, kTile, 0, C->stream, F.tab.p, Cl.tab.p, F.ptile.p, V.act.p, F.pkch);
  prof_end(C, pk);
  ++C->launches;
}

// mgkcyc (mgsolver.for:224-369, kcycle = 1) for every domain of the view,
// each with its own depth: down the levels with irestr sweeps, irestr +
// iproln sweeps where a domain bottoms out, back up with iproln sweeps.
// Every domain sees exactly the operation sequence of its own V-cycle.
// On entry the level-1 rhs holds su and the level-1 ghost shell holds zeros.
template <typename T>
static void vcycle(mf3d_ctx *C, View &V) {
  const int sch = C->prm.mg_itrsch, ir = C->prm.irestr, ip = C->prm.iproln;
  // pp = 0 (newsolv_mg.for:19-21, :44): the red-black path never reads the
  // level-1 interior before overwriting it; the other smoothers, or no
  // pre-smoothing, need real zeros.
  const bool need_zero = sch != 3 || ir == 0;
  if (need_zero)
    for (size_t b = 0; b < V.blk.size(); ++b) {
      const BlkLev &B = V.blk[b]->lv[1].desc;
      cudaMemsetAsync(B.phi, 0, (size_t)2 * B.cstr * sizeof(T), C->stream);
    }
  // levels >= Lc hold FP64 (the coarsest level of an FP32 V-cycle)
  const int Lc = C->coarse64 ? V.Lmax : V.Lmax + 1;
  auto relax_g = [&](int g, int q, int it, bool fz, bool red_done = false) {
    if (g >= Lc) relax<double>(C, V, g, q, it, fz, red_done);
    else relax<T>(C, V, g, q, it, fz, red_done);
  };
  // with red-black pre-smoothing the restriction also forms the coarse
  // level's first (from-zero) red half-sweep
  const bool red_in_restr = sch == 3 && ir > 0;
  // levels cc_g0.. run as one cluster launch (k_coarse_cycle) where planned,
  // levels 2 .. cc_g0-1 (or the coarsest) as one cooperative launch per
  // direction (k_mid_cycle) where planned
  const int gtop = V.cc_g0 ? V.cc_g0 - 1 : V.Lmax;
  for (int g = 1; g <= (V.mid_on ? 1 : gtop); ++g) {
    relax_g(g, SUB_A, ir, sch == 3, g > 1 && red_in_restr);  // a level starts from zero (pp = 0; mgrestr)
    relax_g(g, SUB_C, ip, sch == 3 && ir == 0);
    if (g < V.Lmax) {
      if (g + 1 >= Lc) restr<T, double>(C, V, g);
      else restr<T, T>(C, V, g);
    }
  }
  if (V.mid_on) {
    // the barrier's count starts at 0 even after a launch that gave up waiting
    cudaMemsetAsync(V.mid_bar.p, 0, sizeof(MidBar), C->stream);
    launch_coop(k_mid_cycle<T>, V.mid_grid, MID_THREADS, 0, C->stream, (const MidPhase *)V.mid_down.p, V.n_mid_down,
                (const int *)V.act.p, V.mid_bar.p, V.err.p);
    ++C->launches;
  }
  if (V.cc_g0) {
    launch_cl(k_coarse_cycle<T>, (int)V.blk.size(), CC_THREADS, V.cc_smem, C->stream, (int)V.blk.size(), V.cc_args,
              (const int *)V.act.p);
    ++C->launches;
  }
  if (V.mid_on && V.n_mid_up) {
    cudaMemsetAsync(V.mid_bar.p, 0, sizeof(MidBar), C->stream);
    launch_coop(k_mid_cycle<T>, V.mid_grid, MID_THREADS, 0, C->stream, (const MidPhase *)V.mid_up.p, V.n_mid_up,
                (const int *)V.act.p, V.mid_bar.p, V.err.p);
    ++C->launches;
  }
  for (int g = V.mid_on ? 1 : gtop - (V.cc_g0 ? 0 : 1); g >= 1; --g) {
    if (g + 1 >= Lc) corr<T, double>(C, V, g);
    else corr<T, T>(C, V, g);
    relax_g(g, SUB_D, ip, false);
  }
}

// ---------------------------------------------------------------------------
// Autotuner.  Per level it picks, by timing the candidates on the view's own
// arrays, (a) the schedule of the red-black half-sweep (sweep_segments: one
// wave of equal plane runs across columns, two waves, or c / c+1 runs per
// column), (b) for levels between 64 K and 4 M cells, the sweep kernel
// (TMA-staged k_rbgs or the plain-load k_rbgs_small), (c) the planes per CTA
// of the TMA restriction into the level, and (d) the CTAs per block of the
// line and lexicographic relaxations.  Every candidate computes the same
// values bit for bit - a half-sweep updates each cell from the other colour
// alone, a restriction each coarse cell from its own children, a line or
// lexicographic sweep keeps its recurrence order whatever the CTA split -
// so the choice changes only the time.  Choices are cached for the process
// by device, precision, smoother and the level's block shapes; a context
// whose levels are all cached times nothing.  The server's lanes look the
// cache up and keep the defaults on a miss.  MF3D_AUTOTUNE=0 turns it off.
// ---------------------------------------------------------------------------
static std::mutex g_tune_mu;
static std::map<std::string, int> g_tune;

static bool autotune_enabled() {
  const char *e = std::getenv("MF3D_AUTOTUNE");
  return !(e && e[0] == '0');
}
static std::string tune_key(const mf3d_ctx *C, const ViewLevel &L, const char *what, int elem) {
  std::string k = std::string(what) + "|dev" + std::to_string(C->device) + "|e" + std::to_string(elem) + "|s" +
                  std::to_string(C->prm.mg_itrsch) + "|occ" + std::to_string(C->sweep_occ);
  for (int b : L.hblk[SUB_A]) {
    const BlkLev &B = L.htab[b];
    k += "|" + std::to_string(B.nx) + "x" + std::to_string(B.ny) + "x" + std::to_string(B.nz);
  }
  return k;
}
static bool tune_get(const std::string &k, int &v) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(k);
  if (it == g_tune.end()) return false;
  v = it->second;
  return true;
}
static void tune_put(const std::string &k, int v) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[k] = v;
}
// MF3D_TUNE_LOG=1 prints each choice the tuner makes to stderr.
static void tune_log(const mf3d_ctx *C, int g, const char *what, int v) {
  static const bool on = [] {
    const char *e = std::getenv("MF3D_TUNE_LOG");
    return e && e[0] == '1';
  }();
  if (on) std::fprintf(stderr, "mf3d tune: device %d level %d %s = %d\n", C->device, g, what, v);
}
// Mean device milliseconds of f() over kTuneReps runs after one warm-up
// run; a failed launch counts as infinitely slow.
constexpr int kTuneReps = 3, kTuneTrials = 3;
constexpr double kTuneMargin = 0.03;  // a candidate must beat the default by 3 %
template <class Fn>
static double tune_time(mf3d_ctx *C, Fn &&f) {
  f();
  if (cudaEventRecord(C->ev0, C->stream) != cudaSuccess) return 1e30;
  for (int r = 0; r < kTuneReps; ++r) f();
  if (cudaEventRecord(C->ev1, C->stream) != cudaSuccess || cudaEventSynchronize(C->ev1) != cudaSuccess) {
    cudaGetLastError();
    return 1e30;
  }
  if (cudaGetLastError() != cudaSuccess) return 1e30;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, C->ev0, C->ev1);
  return ms / kTuneReps;
}
// Picks one of n candidates: set(c) installs candidate c, run() is the work
// it is timed on.  The candidates are timed in kTuneTrials interleaved
// rounds and each keeps its fastest round, so a slow moment of the GPU
// (another context, a clock change) hits every candidate alike and no single
// run decides.  The default def stays unless the fastest candidate beats it
// by kTuneMargin: a close call keeps the shape that was chosen by measuring
// whole solves.  Installs the pick; returns a status.
template <class Set, class Run>
static int tune_pick(mf3d_ctx *C, int n, int def, Set &&set, Run &&run, int &pick) {
  std::vector<double> t(n, 1e30);
  int st;
  for (int tr = 0; tr < kTuneTrials; ++tr)
    for (int c = 0; c < n; ++c) {
      if ((st = set(c))) return st;
      t[c] = std::min(t[c], tune_time(C, run));
    }
  int best = def;
  for (int c = 0; c < n; ++c)
    if (t[c] < t[best]) best = c;
  pick = t[best] < (1.0 - kTuneMargin) * t[def] ? best : def;
  return set(pick);
}
static int upload_sweeps(mf3d_ctx *C, ViewLevel &L, int sched, int only_q = -1) {
  for (int q = 0; q < 3; ++q) {
    if (only_q >= 0 && q != only_q) continue;
    std::vector<RbSeg> sw;
    std::vector<int> sf;
    L.n_sweep[q] = sweep_segments(C, L.htab, L.hblk[q], sw, sf, sched);
    int st;
    if ((st = L.sweep[q].upload(sw, C->stream))) return st;
    if ((st = L.sfirst[q].upload(sf, C->stream))) return st;
  }
  L.sched = sched;
  return MF3D_OK;
}
// line relaxation shape for cl CTAs per block (as tdma_layout's)
static void td_shape(ViewLevel &L, int cl) {
  const size_t sz = L.td_fp64 ? 8 : 4, cap = 200 * 1024;
  const int per = (L.td_numax + cl - 1) / cl;
  L.td_gmax = (int)std::max<size_t>(1, std::min<size_t>(per, cap / ((7 * (size_t)L.td_nmax + 9) * sz)));
  L.td_smem = (7 * (size_t)L.td_gmax * (L.td_nmax + 1) + 2 * (size_t)L.td_gmax) * sz;
  L.td_cl = cl;
}

template <typename T>
static int autotune_level(mf3d_ctx *C, View &V, int g, bool time_new) {
  ViewLevel &L = V.lv[g];
  if (!L.n_list[SUB_A]) return MF3D_OK;
  cudaStream_t s = C->stream;
  const int sch = C->prm.mg_itrsch;
  int st;
  const dim3 cta(RB_TX, RB_TY);
  if (sch == 3 && !C->prm.lsm) {
    // (a) sweep schedule, (b) sweep kernel
    const std::string ks = tune_key(C, L, "sweep", sizeof(T));
    int v;
    const char *forced = std::getenv("MF3D_SWEEP_SCHED");  // a fixed schedule (tuning comparisons)
    if (forced) {
      if ((st = upload_sweeps(C, L, std::max(0, std::min(kSweepSchedules - 1, std::atoi(forced)))))) return st;
    } else if (g == 1) {
      // level 1 keeps the default: timed on its own (no outer kernels
      // around it, no fields bound yet) it ranks the schedules differently
      // from whole solves, where schedule 0 measured 52.1 us a half-sweep
      // against 46.6 us for the default on 2x2x2 blocks of 128^3
    } else if (tune_get(ks, v)) {
      if ((st = upload_sweeps(C, L, v & 7))) return st;
      L.small = (v >> 3) & 1;
    } else if (time_new) {
      // candidates 0 .. kSweepSchedules-1: k_rbgs with that schedule;
      // kSweepSchedules: k_rbgs_small (levels of 64 K to 4 M cells)
      const long long cells = L.cells_sub[SUB_A];
      const bool small_ok = g > 1 && cells >= (1LL << 16) && cells <= (1LL << 22);
      const int n = kSweepSchedules + (small_ok ? 1 : 0);
      const int Lc = C->coarse64 ? V.Lmax : V.Lmax + 1;
      const int ir = std::max(C->prm.irestr, 1), ip = C->prm.iproln;
      // the level's share of a V-cycle: pre-smoothing from zero, the
      // restriction below it and the correction from below, post-smoothing
      // (the kernels around the half-sweeps set the L2 contents and the
      // launch overlap that the sweeps meet in a solve)
      auto pass = [&] {
        relax<T>(C, V, g, SUB_A, ir, true, false);
        if (g < V.Lmax) {
          if (g + 1 >= Lc) { restr<T, double>(C, V, g); corr<T, double>(C, V, g); }
          else { restr<T, T>(C, V, g); corr<T, T>(C, V, g); }
        }
        relax<T>(C, V, g, SUB_D, ip, false);
      };
      auto set = [&](int c) {
        L.small = c == kSweepSchedules ? 1 : 0;
        return upload_sweeps(C, L, L.small ? kDefaultSweepSchedule : c);
      };
      int pick;
      if ((st = tune_pick(C, n, kDefaultSweepSchedule, set, pass, pick))) return st;
      tune_log(C, g, L.small ? "sweep kernel: plain loads" : "sweep schedule", L.sched);
      tune_put(ks, L.sched | (L.small << 3));
    }
  }
  if ((sch == 2 || sch == 1) && !C->prm.lsm) {
    // (d) CTAs per block of the line / lexicographic relaxation: the
    // default and the portable sizes below it
    const std::string kl = tune_key(C, L, sch == 2 ? "tdma" : "lex", sizeof(T));
    const int def = sch == 2 ? L.td_cl : L.lx_cl;
    int v;
    auto set_cl = [&](int cl) {
      if (sch == 2) td_shape(L, cl);
      else L.lx_cl = cl;
    };
    if (tune_get(kl, v)) {
      if (v <= def) set_cl(v);
    } else if (time_new && def > 1) {
      // the default and the portable cluster sizes below it
      std::vector<int> cls{def};
      for (int cl : {8, 4})
        if (cl < def) cls.push_back(cl);
      int pick;
      if ((st = tune_pick(
               C, (int)cls.size(), 0, [&](int c) { set_cl(cls[c]); return (int)MF3D_OK; },
               [&] {
                 if (sch == 2)
                   launch_cl(k_tdma_lines<T>, L.n_list[SUB_A] * L.td_cl, TD_THREADS, L.td_smem, s, L.td_cl, L.tab.p,
                             L.list[SUB_A].p, V.act.p, L.td_cl, L.td_gmax, L.td_nmax);
                 else
                   launch_cl(k_lexgs<T>, L.n_list[SUB_A] * L.lx_cl, 1024, 0, s, L.lx_cl, L.tab.p, L.list[SUB_A].p,
                             V.act.p, L.lx_cl);
               },
               pick)))
        return st;
      tune_log(C, g, sch == 2 ? "line CTAs per block" : "lex CTAs per block", cls[pick]);
      tune_put(kl, cls[pick]);
    }
  }
  return MF3D_OK;
}

// (c) planes per CTA of the TMA restriction into level g (from g-1).
static int autotune_restrict(mf3d_ctx *C, View &V, int g, bool time_new) {
  ViewLevel &L = V.lv[g];
  if (!(C->prm.mg_itrsch == 3 && C->prm.irestr > 0 && g > 1 && L.n_rtma && !C->prm.lsm)) return MF3D_OK;
  const int Lc = C->coarse64 ? V.Lmax : V.Lmax + 1;
  const bool f64 = C->elem == 8 || g - 1 >= Lc, c64 = C->elem == 8 || g >= Lc;
  const std::string kr = tune_key(C, L, "restrict", (f64 ? 80 : 40) + (c64 ? 8 : 4));
  // kch < 0: the plain-load restriction (k_restrict over the level's plane
  // tiles), which small levels can prefer to the TMA ring's fill latency
  auto set_kch = [&](int kch) {
    std::vector<Tile> rm;
    if (kch >= 0) L.rtma_kch = rtma_tiles(C, L.htab, L.hblk[SUB_A], kch, rm);
    L.n_rtma = (int)rm.size();
    return L.rtma.upload(rm, C->stream);
  };
  int v, st;
  if (tune_get(kr, v)) return set_kch(v);
  if (!time_new) return MF3D_OK;
  static const int kch_of[6] = {2, 4, 8, 16, 32, -1};
  int def = 0;
  for (int c = 0; c < 5; ++c)
    if (kch_of[c] == L.rtma_kch) def = c;  // the wave model's choice (rtma_tiles)
  int pick;
  if ((st = tune_pick(
           C, 6, def, [&](int c) { return set_kch(kch_of[c]); },
           [&] {
             if (f64) restr<double, double>(C, V, g - 1);
             else if (c64) restr<float, double>(C, V, g - 1);
             else restr<float, float>(C, V, g - 1);
           },
           pick)))
    return st;
  tune_log(C, g, "restrict planes", kch_of[pick]);
  tune_put(kr, kch_of[pick]);
  return MF3D_OK;
}

// Tunes (or looks up) every level of the view; time_new = false only looks
// the cache up.  The arrays are scratch at this point (the solve writes every
// value it reads) except the level-1 ghost shell, which must hold zeros: the
// timed corrections write it, so level 1's phi is cleared at the end.  The
// restrictions are tuned first, since a level's sweep is timed together with
// the restriction below it.  Levels inside the coarse cluster launch
// (k_coarse_cycle) run no sweep or restriction of their own.
static int autotune_view(mf3d_ctx *C, View &V, bool time_new) {
  if (!autotune_enabled() || C->lmr) return MF3D_OK;
  if (C->prm.mg_itrsch == 2 && C->prm.lsm) return MF3D_OK;
  const int Lc = C->coarse64 ? V.Lmax : V.Lmax + 1;
  // last level with its own sweep launches (the middle-level launch and the
  // coarse cluster compute per cell, untuned)
  const int gl = V.mid_on ? 1 : V.cc_g0 ? V.cc_g0 - 1 : V.Lmax;
  int st;
  for (int g = 2; g <= std::min(gl + 1, V.Lmax); ++g)
    if ((st = autotune_restrict(C, V, g, time_new))) return st;
  for (int g = 1; g <= gl; ++g) {
    const bool fp64 = C->elem == 8 || g >= Lc;
    if ((st = fp64 ? autotune_level<double>(C, V, g, time_new) : autotune_level<float>(C, V, g, time_new))) return st;
  }
  if (!time_new) return MF3D_OK;
  CK(cudaStreamSynchronize(C->stream));
  const size_t e1 = (C->elem == 8 || 1 >= Lc) ? 8 : 4;
  for (size_t b = 0; b < V.blk.size(); ++b) {
    const BlkLev &B = V.blk[b]->lv[1].desc;
    CK(cudaMemsetAsync(B.phi, 0, (size_t)2 * B.cstr * e1, C->stream));
  }
  CK(cudaMemsetAsync(V.err.p, 0, sizeof(int), C->stream));
  CK(cudaStreamSynchronize(C->stream));
  return MF3D_OK;
}

// A field exchange copy map (k_fx_stage + k_fx_apply); returns the launches.
static int field_exchange(mf3d_ctx *C, View &V, const FxCopy *pairs, long long n, long long nstaged,
                          const int *only, const double *prev = nullptr) {
  if (!n) return 0;
  if (nstaged)
    launch(k_fx_stage, grid_of(nstaged, kTile), kTile, 0, C->stream, V.df.p, pairs, nstaged, only, V.fx_stage.p,
           prev);
  launch(k_fx_apply, grid_of(n, kTile), kTile, 0, C->stream, V.df.p, pairs, n, nstaged, only, V.fx_stage.p, prev);
  return nstaged ? 2 : 1;
}

// exchange(4) + pbound after p += pp: the whole copy map where the view has
// one (every ghost the reference writes), else the face ghosts calvel reads.
static void p_exchange(mf3d_ctx *C, View &V, const int *act) {
  if (V.nfx_p) {
    C->launches += field_exchange(C, V, V.fx_p, V.nfx_p, V.nsfx_p, act);
  } else {
    launch(k_p_faces, V.n_faces, kTile, 0, C->stream, V.df.p, V.t_faces.p, act);
    ++C->launches;
  }
}

// At a calvel point of the fused path (the initial calvel, each outer
// iteration), the chained ghosts of exchange(1..3): k_fx_evolve + the
// sub-map (see k_fx_evolve).  Nothing when the layout has no such chains.
static void field_evolve(mf3d_ctx *C, View &V, const int *act) {
  if (V.fx_per_iteration) return;
  const long long n1 = V.nfxe_cells + V.nfxe_chain + V.nsfxe_sub;
  if (n1) {
    launch(k_fx_evolve, grid_of(n1, kTile), kTile, 0, C->stream, V.df.p, V.ds.p, act, V.fxe_cells, V.nfxe_cells,
           V.fxe_chain, V.nfxe_chain, V.fx_prev.p, V.fxe_sub, V.nsfxe_sub, V.fx_stage.p);
    ++C->launches;
  }
  if (V.nfxe_sub) {
    launch(k_fx_apply, grid_of(V.nfxe_sub, kTile), kTile, 0, C->stream, V.df.p, V.fxe_sub, V.nfxe_sub, V.nsfxe_sub,
           act, V.fx_stage.p, (const double *)nullptr);
    ++C->launches;
  }
}

// Fused calvel + calmas over the view (the TMA-staged kernel when the bound
// fields admit it).
template <typename T>
static void calvel_calmas(mf3d_ctx *C, View &V, const int *act, unsigned long long *slot, int write_su,
                          bool exchange = true) {
  if (C->prm.differencing == 2) {
    // the 4th-order divergence reads two face layers past the cell: calvel,
    // its exchange(1..3) and calmas in the reference's order (the whole
    // exchange where the view has its copy map; `exchange` false when the
    // velocities are already this calvel point's, exchanged)
    launch(k_calvel, V.n_int, dim3(RW_TX, RW_RJ), 0, C->stream, V.df.p, V.t_int.p, V.ds.p, act);
    ++C->launches;
    if (exchange && V.nfx_uvw) {
      C->launches += field_exchange(C, V, V.fx_uvw, V.nfx_uvw, V.nsfx_uvw, act);
    } else if (exchange) {
      launch(k_vel_faces, V.n_vfaces, kTile, 0, C->stream, V.df.p, V.t_vfaces.p, act, C->prm.pl_ex);
      ++C->launches;
    }
    launch(k_calmas4<T>, V.n_int, dim3(RW_TX, RW_RJ), 0, C->stream, V.df.p, V.t_int.p, V.ds.p, act, slot, write_su);
    return;
  }
  if (C->prm.lsm) {
    launch(k_calvel_calmas_lsm, V.n_zint, dim3(OZ_TX, OZ_RJ), 0, C->stream, V.df.p, V.t_zint.p, V.ds.p, act, slot,
           write_su);
  } else if (V.fields_tma) {
    // axes that are uniform with a power-of-two spacing in every block
    int mask = 7;
    for (const auto &F : V.hf)
      for (int a = 0; a < 3; ++a)
        if (F.pinv[a] == 0.0) mask &= ~(1 << a);
    const dim3 grid(V.n_zint), cta(OZ_TX, CV_TY);
#define MF3D_CV(M)                                                                                              \
  case M:                                                                                                        \
    launch(k_calvel_calmas_tma<T, M>, grid, cta, 0, C->stream, V.df.p, V.t_zint.p, V.ds.p, act, slot, write_su, OZ_KCH, \
                                                           V.err.p);                                             \
    break;
    switch (mask) { MF3D_CV(0) MF3D_CV(1) MF3D_CV(2) MF3D_CV(3) MF3D_CV(4) MF3D_CV(5) MF3D_CV(6) MF3D_CV(7) }
#undef MF3D_CV
  } else
    launch(k_calvel_calmas<T>, V.n_zint, dim3(OZ_TX, OZ_RJ), 0, C->stream, V.df.p, V.t_zint.p, V.ds.p, act, slot,
                                                                      write_su);
}

// One outer iteration of newsolv_mg (newsolv_mg.for:25-58) for every active
// domain: V-cycle, p += pp, p halo + pbound, calvel + calmas, bookkeeping.
template <typename T>
static void iteration_body(mf3d_ctx *C, View &V, int loop_graph) {
  cudaStream_t s = C->stream;
  vcycle<T>(C, V);
  launch(k_add_correction<T>, V.n_pairs, kTile, 0, s, V.df.p, V.t_pairs.p, V.act.p, V.pairs_kch);
  p_exchange(C, V, V.act.p);
  prof_begin(C, MF3D_PROF_CALMAS, (double)V.n_l1 * (4 * sizeof(double) + sizeof(T)));  // p, u*, v*, w* in; su out
  calvel_calmas<T>(C, V, V.act.p, V.rmax.p, 0);
  prof_end(C, MF3D_PROF_CALMAS);
  field_evolve(C, V, V.act.p);
  launch(k_iter_end, 1, 256, 0, s, V.ds.p, (int)V.dom.size(), V.rmax.p, V.hist.p, V.hcap, V.act.p, V.cond,
                               loop_graph, V.budget.p);
  C->launches += 3;
}

template <typename T>
static int build_graphs(mf3d_ctx *C, View &V) {
  if (V.x_loop && V.x_once) return MF3D_OK;
  const int saved_prof = C->prof_kind;
  const long long saved_launches = C->launches;
  C->prof_kind = 0;  // no event records inside graphs
  // the whole outer loop: a conditional WHILE node around one iteration
  CK(cudaGraphCreate(&V.g_loop, 0));
  CK(cudaGraphConditionalHandleCreate(&V.cond, V.g_loop, 1u, cudaGraphCondAssignDefault));
  cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
  np.conditional.handle = V.cond;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, V.g_loop, nullptr, 0, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  // a failed capture leaves no partial graph and the counters as they were
  auto fail = [&](cudaError_t e, const char *what) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    C->launches = saved_launches;
    C->prof_kind = saved_prof;
    V.drop_graphs();
    return MF3D_E_CUDA;
  };
  cudaError_t e = cudaStreamBeginCaptureToGraph(C->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) return fail(e, "cudaStreamBeginCaptureToGraph");
  C->launches = 0;
  iteration_body<T>(C, V, 1);
  V.launches_per_iter = C->launches;
  cudaGraph_t captured = nullptr;
  if ((e = cudaStreamEndCapture(C->stream, &captured)) != cudaSuccess) return fail(e, "capture of the outer loop");
  if ((e = cudaGraphInstantiate(&V.x_loop, V.g_loop, 0)) != cudaSuccess) return fail(e, "cudaGraphInstantiate");
  // one iteration (the server's per-cycle step)
  if ((e = cudaStreamBeginCapture(C->stream, cudaStreamCaptureModeRelaxed)) != cudaSuccess)
    return fail(e, "cudaStreamBeginCapture");
  iteration_body<T>(C, V, 0);
  if ((e = cudaStreamEndCapture(C->stream, &V.g_once)) != cudaSuccess) return fail(e, "capture of one iteration");
  if ((e = cudaGraphInstantiate(&V.x_once, V.g_once, 0)) != cudaSuccess) return fail(e, "cudaGraphInstantiate");
  C->launches = saved_launches;
  C->prof_kind = saved_prof;
  return MF3D_OK;
}

// The server's cycle: a WHILE node around one iteration that runs until a
// domain stops, none is left, or V.budget iterations have run.
template <typename T>
static int build_server_graph(mf3d_ctx *C, View &V) {
  if (V.x_loop) return MF3D_OK;
  CK(cudaGraphCreate(&V.g_loop, 0));
  CK(cudaGraphConditionalHandleCreate(&V.cond, V.g_loop, 1u, cudaGraphCondAssignDefault));
  cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
  np.conditional.handle = V.cond;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, V.g_loop, nullptr, 0, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  CK(cudaStreamBeginCaptureToGraph(C->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  const long long saved = C->launches;
  iteration_body<T>(C, V, 2);
  V.launches_per_iter = C->launches - saved;
  C->launches = saved;
  cudaGraph_t captured;
  CK(cudaStreamEndCapture(C->stream, &captured));
  CK(cudaGraphInstantiate(&V.x_loop, V.g_loop, 0));
  return MF3D_OK;
}

// Bind the caller's field pointers (ttc layout, device) to the view blocks.
static int bind_fields(mf3d_ctx *C, View &V, const mf3d_fields *f) {
  for (size_t b = 0; b < V.blk.size(); ++b) {
    BlkFld &F = V.hf[b];
    // the old velocities of mf3d_bind_old_velocity, unless this call (the
    // velocity predictor) bound its own
    if (!C->oo_bound.empty() && !F.oo[0])
      for (int a = 0; a < 3; ++a) F.oo[a] = C->oo_bound[b][a];
    F.ustar = f[b].ustar; F.vstar = f[b].vstar; F.wstar = f[b].wstar;
    F.u = f[b].u; F.v = f[b].v; F.w = f[b].w; F.p = f[b].p; F.su = f[b].su;
    F.dens = C->prm.lsm ? f[b].dens : nullptr;
    if (!F.ustar || !F.vstar || !F.wstar || !F.u || !F.v || !F.w || !F.p || (C->prm.lsm && !F.dens)) {
      set_error("mf3d_fields: a required pointer is NULL");
      return MF3D_E_INVALID;
    }
  }
  // TMA staging of p, ustar, vstar, wstar needs 16-byte aligned bases and rows
  // of a multiple of 16 bytes (ttc_i even); otherwise the plain-load kernel runs
  const size_t nb = V.blk.size();
  bool tma = tensor_map_encoder() != nullptr;
  for (size_t b = 0; b < nb && tma; ++b) {
    const BlkFld &F = V.hf[b];
    const double *fp[4] = {F.p, F.ustar, F.vstar, F.wstar};
    tma = F.ti % 2 == 0;
    for (const double *q : fp) tma = tma && ((uintptr_t)q % 16 == 0);
  }
  if (tma) {
    std::vector<CUtensorMap> maps(4 * nb);
    const int rows[4] = {CvShape::PR, CvShape::UR, CvShape::VR, CvShape::WR};
    int st;
    for (size_t b = 0; b < nb; ++b) {
      BlkFld &F = V.hf[b];
      const double *fp[4] = {F.p, F.ustar, F.vstar, F.wstar};
      const int tk = F.nz + 2 * F.pl;
      for (int a = 0; a < 4; ++a)
        if ((st = field_map(&maps[4 * b + a], fp[a], F.ti, F.tj, tk, rows[a]))) return st;
    }
    if (V.fmaps.n != maps.size() && (st = V.fmaps.alloc(maps.size()))) return st;
    CK(cudaMemcpyAsync(V.fmaps.p, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice,
                       C->stream));
    CK(cudaStreamSynchronize(C->stream));  // maps is a local
    for (size_t b = 0; b < nb; ++b) V.hf[b].fm = V.fmaps.p + 4 * b;
  } else {
    for (size_t b = 0; b < nb; ++b) V.hf[b].fm = nullptr;
  }
  if (tma != V.fields_tma) {
    V.fields_tma = tma;
    V.drop_graphs();  // the captured iteration names the calvel/calmas variant
  }
  CK(cudaMemcpyAsync(V.df.p, V.hf.data(), V.hf.size() * sizeof(BlkFld), cudaMemcpyHostToDevice, C->stream));
  return MF3D_OK;
}

// L_LSM: `coeff` at the start of every solve (newsolv_mg.for:12-14): the
// level densities from the bound dens field, then every level's per-cell
// coefficients (mgsolver.for:69-203).
static void lsm_coefficients(mf3d_ctx *C, View &V) {
  cudaStream_t s = C->stream;
  for (size_t b = 0; b < V.blk.size(); ++b) {
    const BlockStore &S = *V.blk[b];
    const BlkFld &F = V.hf[b];
    const double cx = S.d.dy * S.d.dz / S.d.dx, cy = S.d.dx * S.d.dz / S.d.dy, cz = S.d.dx * S.d.dy / S.d.dz;
    const long long ps = (long long)F.ti * F.tj;
    DensView d{F.dens, (long long)(F.pl - 1) * (1 + F.ti + ps), F.ti, ps};
    for (int g = 1; g <= S.ngrid; ++g) {
      const BlkLev &B = S.lv[g].desc;
      const long long n = (long long)B.nx * B.ny * B.nz;
      if (g > 1) {
        launch(k_lsm_coarsen, grid_of(n, 256), 256, 0, s, d, S.lv[g].dens.p, B.nx, B.ny, B.nz);
        const long long sy = B.nx, sz = (long long)B.nx * B.ny;
        d = DensView{S.lv[g].dens.p, -(1 + sy + sz), sy, sz};
        ++C->launches;
      }
      launch(k_lsm_coef, grid_of(n, 256), 256, 0, s, B, d, cx, cy, cz);
      ++C->launches;
    }
  }
}

// Start the solve of every domain of the view: state, face planes, the
// initial calvel/calmas (newsolv_mg.for:16-17; p's ghosts used as given),
// rmax0 and the thresholds.  Everything stays on the device.
template <typename T>
static int solve_begin(mf3d_ctx *C, View &V, const double *dt, const double *alfapr) {
  cudaStream_t s = C->stream;
  const int nd = (int)V.dom.size();
  std::vector<DomState> hs(nd);
  for (int d = 0; d < nd; ++d) {
    std::memset(&hs[d], 0, sizeof(DomState));
    hs[d].dt = dt[d];
    hs[d].dtinv = pow2_inverse(dt[d]);
    hs[d].rdt = div_reciprocal(dt[d]);
    hs[d].alfapr = alfapr[d];
    hs[d].tol = C->prm.eps;
    hs[d].eps_relative = C->prm.eps_relative;
    hs[d].maxcy = std::min(std::max(C->prm.maxcy, 0), V.hcap);
  }
  CK(cudaMemcpyAsync(V.ds.p, hs.data(), nd * sizeof(DomState), cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));  // hs is a local
  CK(cudaMemsetAsync(V.rmax.p, 0, nd * sizeof(unsigned long long), s));
  if (C->prm.lsm) {
    lsm_coefficients(C, V);
    if (C->prm.mg_itrsch == 2) tdma_factors(C, V);
  }
  launch(k_face_planes, V.n_planes, kTile, 0, s, V.df.p, V.t_planes.p, C->walls_given ? 1 : 0);
  // the 4th-order calmas, and the chained ghosts of the exchange, read the
  // caller's u, v, w from the first calvel point on
  if (C->wait_side && (C->prm.differencing == 2 || V.nfxe_chain + V.nfxe_sub))
    CK(cudaStreamWaitEvent(s, C->ev_side, 0));
  calvel_calmas<T>(C, V, V.ones.p, V.rmax.p, 0);
  field_evolve(C, V, V.ones.p);
  launch(k_dom_init, 1, 256, 0, s, V.ds.p, nd, V.rmax.p, V.act.p);
  C->launches += 3;
  return MF3D_OK;
}

// exchange_bc of u, v, w with every block on one rank (exchange_bc.for:
// 16-838): per layer, the first walk's self-copies, the second walk's
// self-copies and packs, the third walk's unpacks, each over x, y, z.
// A face code whose boundu/v/w branch needs data the library does not hold:
// the convective outflow of the east face (21, uoo; bounds.for:143-170)
// without the old velocities, wall functions above 65 (no branch) or under
// L_LSM (mu/dens, log_law.for:22), and under L_LSM the inflow and outflow
// faces, which phi gates (bounds.for:43-50, 146-158).  The inlet files of
// the west codes 7 and 8 come through mf3d_set_inlet, Re and fric of the
// wall functions through mf3d_set_wall_model.
static bool bounds_code_unsupported(int f, int code, bool lsm, int alfabc, bool have_oo = false) {
  if (code >= 61 && (code > 65 || lsm)) return true;
  if (f == 1 && code == 21 && alfabc == 1 && !have_oo) return true;
  if (lsm && ((f == 0 && code == 1) || (f == 1 && (code == 2 || code == 21) && alfabc == 1))) return true;
  return false;
}

// exchange_bc of u, v, w (only >= 0: of that component alone)
static void bc_walks(mf3d_ctx *C, View &V, int only = -1) {
  for (int ly = 0; ly <= C->prm.pl_ex; ++ly)
    for (int mode = 0; mode < 3; ++mode)
      for (int a = 0; a < 3; ++a) {
        if (!V.bc_periodic[a]) continue;
        launch(k_bc_walk, V.n_bcax[a], kTile, 0, C->stream, V.df.p, V.t_bcax[a].p, V.ds.p, a, ly, mode, only);
        ++C->launches;
      }
}
// the faces without a neighbour by their code, layers 0..pl_ex (only as above);
// dt < 0: the solve's dt and alfapr.  The wall functions of a tangential
// component (one component at a time) run their face law first, on layer 0.
static void bound_faces(mf3d_ctx *C, View &V, int alfabc, int only = -1, double dt = 0.0, double alfapr = 0.0) {
  for (int ly = 0; ly <= C->prm.pl_ex; ++ly)
    for (int a = 0; a < 3; ++a) {
      if (V.wall_law && ly == 0 && only >= 0 && only != a) {
        launch(k_wall_law, V.n_bcax[a], kTile, 0, C->stream, V.df.p, V.t_bcax[a].p, V.ds.p, a, C->wall_re,
               C->wall_fric, V.err.p);
        ++C->launches;
      }
      launch(k_bound_faces, V.n_bcax[a], kTile, 0, C->stream, V.df.p, V.t_bcax[a].p, V.ds.p, a, ly, C->prm.ubulk,
             alfabc, only, dt, alfapr);
      ++C->launches;
    }
}

// Finish: optional su, the final calvel (u, v, w from the final p).
template <typename T>
static int solve_end(mf3d_ctx *C, View &V) {
  cudaStream_t s = C->stream;
  bool want_su = false;
  for (auto &F : V.hf) want_su |= F.su != nullptr;
  if (want_su) {
    calvel_calmas<T>(C, V, V.ones.p, V.rmax_scratch.p, 1, false);
    ++C->launches;
  }
  if (C->wait_side) CK(cudaStreamWaitEvent(s, C->ev_side, 0));  // the host entry's u, v, w
  launch(k_calvel, V.n_int, dim3(RW_TX, RW_RJ), 0, s, V.df.p, V.t_int.p, V.ds.p, nullptr);
  C->launches += 1;
  // exchange(1..3) of the last calvel (press.for:196-198): the copy map of
  // every ghost it writes where the view has one, chained sources from
  // their state before that exchange (the 4th-order path has exchanged
  // already); else the full periodic planes (bounds mode) and the face ghosts
  if (V.nfx_uvw) {
    if (!V.fx_per_iteration)
      C->launches += field_exchange(C, V, V.fx_uvw, V.nfx_uvw, V.nsfx_uvw, nullptr, V.fx_prev.p);
  } else {
    if (C->prm.bounds) bc_walks(C, V);
    launch(k_vel_faces, V.n_vfaces, kTile, 0, s, V.df.p, V.t_vfaces.p, nullptr, C->prm.pl_ex);
    ++C->launches;
  }
  if (C->prm.bounds) {
    // boundu/boundv/boundw (newsolv_mg.for:86-88); a convective outflow
    // takes the solve's dt and alfapr (dt < 0) and the bound old velocities.
    // The components are independent but for the wall functions, whose laws
    // read all three: then boundu, boundv, boundw one after the other, each
    // with its own periodic copy first, as the reference runs them
    if (V.wall_law) {
      for (int comp = 0; comp < 3; ++comp) {
        bc_walks(C, V, comp);
        bound_faces(C, V, C->prm.alfabc, comp, -1.0, 0.0);
      }
    } else {
      bc_walks(C, V);
      bound_faces(C, V, C->prm.alfabc, -1, -1.0, 0.0);
    }
  }
  return MF3D_OK;
}

// A kernel that gave up waiting (a TMA copy that never landed) leaves its
// code in V.err; the results of that call are not valid.
static int check_device_error(View &V) {
  int e = 0;
  CK(cudaMemcpy(&e, V.err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (e == 0) return MF3D_OK;
  CK(cudaMemset(V.err.p, 0, sizeof(int)));
  if (e == ERR_WALL_LAW) {
    set_error("log_law: USTAR DOESNT CONVERGE (a smooth-wall law took 10 steps, log_law.for:47-62)");
    return MF3D_E_INVALID;
  }
  if (e == ERR_MID_BARRIER) {
    set_error("a grid barrier of the middle-level V-cycle launch did not complete within its time limit");
    return MF3D_E_TIMEOUT;
  }
  set_error("a device copy did not complete within its time limit (code " + std::to_string(e) + ")");
  return MF3D_E_TIMEOUT;
}

// Fold the device state of every domain into the caller's infos/history.
static int collect(mf3d_ctx *C, View &V, mf3d_solve_info *infos, double *hist, int hcap, float ms) {
  const int nd = (int)V.dom.size();
  std::vector<DomState> hs(nd);
  CK(cudaMemcpy(hs.data(), V.ds.p, nd * sizeof(DomState), cudaMemcpyDeviceToHost));
  if (int st = check_device_error(V)) return st;
  int worst = MF3D_OK;
  for (int d = 0; d < nd; ++d) {
    const DomState &D = hs[d];
    int status = MF3D_OK;
    if (D.done == 2) status = MF3D_E_NONFINITE;
    else if (D.done != 1) status = MF3D_NOT_CONVERGED;
    const double rmax = D.iter > 0 ? D.rmax : D.rmax0;
    if (status >= 0 && rmax > 100.0) status = MF3D_DIVERGED;  // newsolv_mg.for:64
    if (infos) {
      infos[d].rmax = rmax; infos[d].rmax0 = D.rmax0; infos[d].iter = D.iter;
      infos[d].status = status; infos[d].ms_device = ms;
    }
    if (hist && hcap > 0 && D.iter > 0)
      CK(cudaMemcpy(hist + (size_t)d * hcap, V.hist.p + (size_t)d * V.hcap, std::min(D.iter, hcap) * sizeof(double),
                    cudaMemcpyDeviceToHost));
    if (status < 0) worst = worst < 0 ? worst : status;
    else if (worst >= 0) worst = std::max(worst, status);
  }
  if (worst == MF3D_E_NONFINITE) set_error("non-finite rmax");
  return worst;
}

template <typename T>
static int solve_view(mf3d_ctx *C, View &V, const double *dt, const double *alfapr, mf3d_solve_info *infos,
                      double *hist, int hcap) {
  cudaStream_t s = C->stream;
  C->launches = 0;
  const int nd = (int)V.dom.size();
  CK(cudaEventRecord(C->ev0, s));
  int st = solve_begin<T>(C, V, dt, alfapr);
  if (st) return st;
  const int maxcy = std::min(std::max(C->prm.maxcy, 0), V.hcap);
  long long iters_run = 0;
  if (maxcy > 0) {
    if (C->use_graph && C->prof_kind == 0) {
      if ((st = build_graphs<T>(C, V)) && V.mid_on) {
        // a driver that does not capture the cooperative middle-level launch
        // into the loop graph: the launch path instead
        V.mid_on = false;
        cudaGetLastError();
        st = build_graphs<T>(C, V);
      }
      if (st) return st;
      CK(cudaGraphLaunch(V.x_loop, s));
    } else {
      std::vector<int> act(nd);
      for (int it = 1; it <= maxcy; ++it) {
        iteration_body<T>(C, V, 0);
        CK(cudaMemcpyAsync(act.data(), V.act.p, nd * sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        prof_collect(C);
        bool any = false;
        for (int a : act) any |= a != 0;
        if (!any) break;
      }
    }
  }
  if ((st = solve_end<T>(C, V))) return st;
  CK(cudaEventRecord(C->ev1, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  prof_collect(C);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, C->ev0, C->ev1);
  const int res = collect(C, V, infos, hist, hcap, ms);
  if (C->use_graph && C->prof_kind == 0 && maxcy > 0) {
    // every domain's iterations ran inside the graph: count the body launches
    std::vector<DomState> hs(nd);
    if (cudaMemcpy(hs.data(), V.ds.p, nd * sizeof(DomState), cudaMemcpyDeviceToHost) == cudaSuccess)
      for (auto &D : hs) iters_run = std::max<long long>(iters_run, D.iter);
    C->launches += std::max(iters_run, 1LL) * V.launches_per_iter;
  }
  return res;
}

}  // namespace mf3d
#include "sip.cuh"
namespace mf3d {

template <typename T>
static int mgkcyc_view(mf3d_ctx *C, View &V, double *const *su, double *const *pp) {
  cudaStream_t s = C->stream;
  const int nb = (int)V.blk.size();
  C->launches = 0;
  if (C->ptrs.n < (size_t)2 * nb && C->ptrs.alloc(2 * nb)) return MF3D_E_OOM;
  CK(cudaMemcpyAsync(C->ptrs.p, su, nb * sizeof(double *), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(C->ptrs.p + nb, pp, nb * sizeof(double *), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(V.df.p, V.hf.data(), nb * sizeof(BlkFld), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(V.act.p, V.ones.p, V.ones.n * sizeof(int), cudaMemcpyDeviceToDevice, s));
  launch(k_load_rhs<T>, V.n_int, dim3(RW_TX, RW_RJ), 0, s, V.df.p, V.t_int.p, C->ptrs.p);
  vcycle<T>(C, V);
  launch(k_store_pp<T>, V.n_l1cells, dim3(RW_TX, RW_RJ), 0, s, V.df.p, V.t_l1cells.p, C->ptrs.p + nb);
  // restore the invariant: the level-1 ghost shell holds zeros between calls
  ViewLevel &L1 = V.lv[1];
  launch(k_zero_ghosts<T>, dim3(64, L1.n_list[SUB_A]), kTile, 0, s, L1.tab.p, L1.list[SUB_A].p, L1.n_list[SUB_A]);
  C->launches += 3;
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return check_device_error(V);
}

// ---------------------------------------------------------------------------
// mf3d_mgkcyc_device_noalloc: the pointer tables in a fixed device array.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double *g_noalloc_ptrs[2 * MF3D_NOALLOC_MAX_BLOCKS];

// Device address of g_noalloc_ptrs in the current device's context, looked
// up when a context is created (ctx_init), with its device current.  The
// address is kept in the context, so a context created after a device reset
// (which reloads the module, possibly elsewhere) holds the new address.
static int noalloc_tables(void **out) {
  void *a = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&a, g_noalloc_ptrs);
  if (e != cudaSuccess || !a) {
    set_error(std::string("mf3d_mgkcyc_device_noalloc set-up: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    return MF3D_E_CUDA;
  }
  *out = a;
  return MF3D_OK;
}

// Loads every kernel a V-cycle call can launch (cudaFuncGetAttributes forces
// a lazily loaded module function in), so that no later call - in particular
// mf3d_mgkcyc_device_noalloc - makes the driver load code on first use.
template <typename T>
static int preload_vcycle_kernels() {
  cudaFuncAttributes fa;
  const void *k[] = {
      (const void *)k_rbgs<T, true>, (const void *)k_rbgs<T, false>, (const void *)k_rbgs_small<T, true>,
      (const void *)k_rbgs_small<T, false>, (const void *)k_rbgs_small<double, true>,
      (const void *)k_rbgs_small<double, false>, (const void *)k_rbgs<double, true>,
      (const void *)k_rbgs<double, false>, (const void *)k_lexgs<T>, (const void *)k_lexgs<double>,
      (const void *)k_tdma_factor<T>, (const void *)k_tdma_factor<double>, (const void *)k_tdma_lines<T>,
      (const void *)k_tdma_lines<double>, (const void *)k_restrict<T, T>, (const void *)k_restrict<T, double>,
      (const void *)k_restrict_tma<T, T>, (const void *)k_restrict_tma<T, double>, (const void *)k_prolong<T, T>,
      (const void *)k_prolong<T, double>, (const void *)k_halo_stage<T>, (const void *)k_halo_apply<T>,
      (const void *)k_halo_stage<double>, (const void *)k_halo_apply<double>, (const void *)k_zero_ghosts<T>,
      (const void *)k_load_rhs<T>, (const void *)k_store_pp<T>};
  for (const void *f : k) CK(cudaFuncGetAttributes(&fa, f));
  return MF3D_OK;
}

template <typename T>
static int mgkcyc_view_noalloc(mf3d_ctx *C, View &V, double *const *su, double *const *pp) {
  cudaStream_t s = C->stream;
  const int nb = (int)V.blk.size();
  if (nb > MF3D_NOALLOC_MAX_BLOCKS) {
    set_error("mf3d_mgkcyc_device_noalloc: " + std::to_string(nb) + " blocks exceed MF3D_NOALLOC_MAX_BLOCKS (" +
              std::to_string(MF3D_NOALLOC_MAX_BLOCKS) + ")");
    return MF3D_E_INVALID;
  }
  double **tab = (double **)C->noalloc_tab;
  C->launches = 0;
  CK(cudaMemcpyAsync(tab, su, nb * sizeof(double *), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(tab + nb, pp, nb * sizeof(double *), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(V.df.p, V.hf.data(), nb * sizeof(BlkFld), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(V.act.p, V.ones.p, V.ones.n * sizeof(int), cudaMemcpyDeviceToDevice, s));
  launch(k_load_rhs<T>, V.n_int, dim3(RW_TX, RW_RJ), 0, s, V.df.p, V.t_int.p, tab);
  vcycle<T>(C, V);
  launch(k_store_pp<T>, V.n_l1cells, dim3(RW_TX, RW_RJ), 0, s, V.df.p, V.t_l1cells.p, tab + nb);
  // restore the invariant: the level-1 ghost shell holds zeros between calls
  ViewLevel &L1 = V.lv[1];
  launch(k_zero_ghosts<T>, dim3(64, L1.n_list[SUB_A]), kTile, 0, s, L1.tab.p, L1.list[SUB_A].p, L1.n_list[SUB_A]);
  C->launches += 3;
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return check_device_error(V);
}

static size_t ttc_elems(int pl, const mf3d_block_desc &d) {
  return (size_t)(d.nx + 2 * pl) * (d.ny + 2 * pl) * (d.nz + 2 * pl);
}

static int check_params(const mf3d_params *prm) {
  if (!prm) { set_error("params: NULL"); return MF3D_E_INVALID; }
  if (prm->ngrid < 1 || prm->ngrid > 16) { set_error("ngrid out of range"); return MF3D_E_INVALID; }
  if (prm->mg_itrsch < 1 || prm->mg_itrsch > 3) { set_error("error about mg iteration selection (mg_itrsch)"); return MF3D_E_INVALID; }
  if (prm->irestr < 0 || prm->iproln < 0 || prm->maxcy < 0) { set_error("negative sweep/cycle count"); return MF3D_E_INVALID; }
  if (prm->pl < 1) { set_error("pl must be >= 1"); return MF3D_E_INVALID; }
  if (prm->pl_ex < 0 || prm->pl_ex >= prm->pl) { set_error("pl_ex must satisfy 0 <= pl_ex < pl"); return MF3D_E_INVALID; }
  // calmas takes its 4th-order branch for differencing 2 (press.for:13-35)
  // and the 2nd-order one otherwise; 3 (WENO convection) is the one L_LSM needs
  if (prm->differencing < 1 || prm->differencing > 3) { set_error("differencing must be 1, 2 or 3"); return MF3D_E_INVALID; }
  if (prm->differencing == 2 && prm->pl < 2) {
    set_error("differencing = 2: the 4th-order divergence reads u(i-2), which needs pl >= 2");
    return MF3D_E_INVALID;
  }
  if (prm->differencing == 2 && prm->lsm) { set_error("differencing = 2 with lsm (L_LSM needs WENO, 3)"); return MF3D_E_INVALID; }
  if (prm->precision < 0 || prm->precision > 1) { set_error("precision mode not supported"); return MF3D_E_UNSUPPORTED; }
  if (prm->lsm && prm->precision != MF3D_PREC_FP64) { set_error("lsm runs in FP64 only"); return MF3D_E_UNSUPPORTED; }
  if (prm->solver != 0 && prm->solver != 1 && prm->solver != 2) { set_error("solver must be 1 or 2"); return MF3D_E_INVALID; }
  if (prm->solver == 1) {
    if (prm->nswp < 1) { set_error("solver 1: nswp must be >= 1"); return MF3D_E_INVALID; }
    if (prm->precision != MF3D_PREC_FP64 || prm->lsm) {
      set_error("solver 1 (SIP) runs in FP64 without lsm");
      return MF3D_E_UNSUPPORTED;
    }
  }
  return MF3D_OK;
}

static int ctx_init(mf3d_ctx *C, const mf3d_params *prm, bool nonblocking = false, bool high_priority = false) {
  C->prm = *prm;
  C->device = prm->device;
  C->elem = prm->precision == MF3D_PREC_FP64 ? 8 : 4;
  CK(cudaSetDevice(C->device));
  // A blocking stream orders after work the caller queued on the legacy
  // default stream (e.g. the copies that produced the device inputs).  The
  // server's lanes use non-blocking streams, so that no lane waits for the
  // caller's or the other lane's work through the legacy stream.
  int lo = 0, hi = 0;
  CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  CK(cudaStreamCreateWithPriority(&C->stream, nonblocking ? cudaStreamNonBlocking : cudaStreamDefault,
                                  high_priority ? hi : lo));
  CK(cudaEventCreate(&C->ev0));
  CK(cudaEventCreate(&C->ev1));
  const char *e = getenv("MF3D_NO_GRAPH");
  C->use_graph = !(e && e[0] == '1');
  CK(cudaDeviceGetAttribute(&C->nsm, cudaDevAttrMultiProcessorCount, C->device));
  int occ = 0;
  if (C->elem == 8) CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rbgs<double, false>, RB_TX * RB_TY, 0));
  else CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rbgs<float, false>, RB_TX * RB_TY, 0));
  C->sweep_occ = std::max(occ, 1);
  // Per-device kernel attributes: every context sets them on its own device
  // (an attribute set on one device does not carry to another).
  CK(cudaFuncSetAttribute(k_restrict_tma<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          RsShape<double>::SMEM));
  CK(cudaFuncSetAttribute(k_restrict_tma<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          RsShape<float>::SMEM));
  CK(cudaFuncSetAttribute(k_restrict_tma<float, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          RsShape<float>::SMEM));
  CK(cudaFuncSetAttribute(k_coarse_cycle<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCcSmemCap));
  CK(cudaFuncSetAttribute(k_coarse_cycle<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCcSmemCap));
  if (int st = C->elem == 8 ? preload_vcycle_kernels<double>() : preload_vcycle_kernels<float>()) return st;
  return noalloc_tables(&C->noalloc_tab);
}

static int make_view(mf3d_ctx *C) {
  std::vector<DomainStore *> doms;
  for (auto &d : C->doms) doms.push_back(d.get());
  C->view.reset(new View());
  int st = build_view(C, *C->view, doms, std::max(C->prm.maxcy, 1));
  if (st) return st;
  return autotune_view(C, *C->view, true);
}

// The west inlets of boundu (bounds.for:55-135) on a block without a west
// neighbour.  Codes 12 and 13 are the 1/7 power law of the wall distance in
// y (13), times the same law in z (12):
//   u = ubulk*(1+1/7)*|2*yc/H|^(1/7)          yc < H/2
//   u = ubulk*(1+1/7)*|2*(H-yc)/H|^(1/7)      otherwise, H = yen - yst
//   u = u*(1+1/7)*|zc/(zen-zst)|^(1/7)        code 12
// formed once on the host in that order, from the cell centres the
// reference forms (a running sum, initial.for:341-365) and the extents of the
// whole domain (alloc_dom.for:427-439).  Code 7 takes u, v and w from the
// caller's inlet file, code 8 v and w from the SEM file and u as its
// fluctuation up added to ubulk or to the code-12 profile (UPROF_SEM = 12),
// both through mf3d_set_inlet.  A component's plane covers its rows
// js-1..je+1 and planes ks-1..ke+1 (code 8: js-1..je, ks-1..ke,
// bounds.for:84-86) at the ghost layers 0..pl_ex.
struct Extents {
  double yst, yen, zst, zen;
};
static Extents domain_extents(const mf3d_block_desc *blocks, int nb) {
  Extents e{blocks[0].ysl, blocks[0].yel, blocks[0].zsl, blocks[0].zel};
  for (int b = 1; b < nb; ++b) {
    e.yst = std::min(e.yst, blocks[b].ysl); e.yen = std::max(e.yen, blocks[b].yel);
    e.zst = std::min(e.zst, blocks[b].zsl); e.zen = std::max(e.zen, blocks[b].zel);
  }
  return e;
}
static double cell_centre(double lo, double h, int pl, int c) {  // field index c, 1-based
  double x = lo + (double)(-pl + 1) * h;
  for (int i = 2; i <= c; ++i) x = x + h;
  return x - 0.5 * h;
}
static double power_law_y(double ubulk, const Extents &e, double yc) {
  const double H = e.yen - e.yst;
  if (yc < H / 2) return ubulk * (1.0 + 1.0 / 7.0) * std::pow(std::fabs(2 * yc / H), 1. / 7.);
  return ubulk * (1.0 + 1.0 / 7.0) * std::pow(std::fabs(2 * (H - yc) / H), 1.0 / 7.0);
}
static double power_law_z(double u, const Extents &e, double zc) {
  return u * (1.0 + 1. / 7.) * std::pow(std::fabs(zc / (e.zen - e.zst)), 1. / 7.);
}
// The last local row and plane of component c (0 u, 1 v, 2 w) on a west
// face: v stops one row short of a north wall, w one plane short of a top
// wall (jsv..jev, ksw..kew; localparameters.for:185-190).
static void west_ranges(const mf3d_block_desc &d, int c, int &je, int &ke) {
  je = d.ny - ((c == 1 && d.jnext < 0 && d.bc_north != MF3D_BC_PERIODIC) ? 1 : 0);
  ke = d.nz - ((c == 2 && d.knext < 0 && d.bc_top != MF3D_BC_PERIODIC) ? 1 : 0);
}
// Values a west inlet of code 7 or 8 reads, u, v, w one after the other:
// code 7 each component over rows js-1..je+1 and planes ks-1..ke+1 of its
// own ranges, code 8 over js-1..je and ks-1..ke (bounds.for:84-86).
static long long inlet_count(const mf3d_block_desc &d, int code) {
  long long n = 0;
  for (int c = 0; c < 3; ++c) {
    int je, ke;
    west_ranges(d, c, je, ke);
    n += code == 7 ? (long long)(je + 2) * (ke + 2) : (long long)(je + 1) * (ke + 1);
  }
  return n;
}
// Forms (codes 12, 13) or installs (7, 8: vals, inlet_count of them) the
// inlet planes of block S.
static int install_inlet(mf3d_ctx *C, BlockStore &S, const Extents &e, int code, int uprof, const double *vals) {
  const mf3d_block_desc &d = S.d;
  const int pl = C->prm.pl, rows = d.ny + 2;
  const size_t pn = (size_t)rows * (d.nz + 2);
  std::vector<double> pln(3 * pn, 0.0);
  int s1[3] = {-1, -1, -1}, t1[3] = {-1, -1, -1};
  if (code == 7 || code == 8) {
    size_t r = 0;
    for (int c = 0; c < 3; ++c) {
      int je, ke;
      west_ranges(d, c, je, ke);
      s1[c] = code == 7 ? je + 1 : je;
      t1[c] = code == 7 ? ke + 1 : ke;
      for (int t = 0; t <= t1[c]; ++t)
        for (int q = 0; q <= s1[c]; ++q) {
          double u = vals[r++];
          if (code == 8 && c == 0) {  // u = up + ubulk, or up + the code-12 profile
            const double up = u;
            if (uprof == 12) {
              u = power_law_y(C->prm.ubulk, e, cell_centre(d.ysl, d.dy, pl, q + pl));
              u = power_law_z(u, e, cell_centre(d.zsl, d.dz, pl, t + pl)) + up;
            } else {
              u = C->prm.ubulk + up;
            }
          }
          pln[c * pn + (size_t)t * rows + q] = u;
        }
    }
  } else {
    s1[0] = d.ny + 1;
    t1[0] = d.nz + 1;
    for (int t = 0; t <= d.nz + 1; ++t)
      for (int q = 0; q <= d.ny + 1; ++q) {
        double u = power_law_y(C->prm.ubulk, e, cell_centre(d.ysl, d.dy, pl, q + pl));
        if (code == 12) u = power_law_z(u, e, cell_centre(d.zsl, d.dz, pl, t + pl));
        pln[(size_t)t * rows + q] = u;
      }
  }
  int st;
  if ((st = S.inlet.upload(pln, C->stream))) return st;
  CK(cudaStreamSynchronize(C->stream));  // pln is a local
  S.fld.inl = S.inlet.p;
  for (int c = 0; c < 3; ++c) {
    S.fld.inl_s1[c] = s1[c];
    S.fld.inl_t1[c] = t1[c];
  }
  return MF3D_OK;
}
static bool inlet_code(const mf3d_block_desc &d) {
  return d.iprev < 0 && (d.bc_west == 7 || d.bc_west == 8 || d.bc_west == 12 || d.bc_west == 13);
}
// The wall-function codes (61 to 65) of a block's faces without a neighbour:
// bit f set for face f; `rough` when one of them is 62.
static int wall_law_faces(const mf3d_block_desc &d, bool *rough = nullptr) {
  const int bcs[6] = {d.bc_west, d.bc_east, d.bc_south, d.bc_north, d.bc_bottom, d.bc_top};
  const int nbrs[6] = {d.iprev, d.inext, d.jprev, d.jnext, d.kprev, d.knext};
  int m = 0;
  for (int f = 0; f < 6; ++f)
    if (nbrs[f] < 0 && bcs[f] >= 61 && bcs[f] <= 65) {
      m |= 1 << f;
      if (rough && bcs[f] == 62) *rough = true;
    }
  return m;
}
// Every code-7 and code-8 inlet of a bounds context has its plane, every
// wall-function face its Re (and fric); with `outflow` (bounds run with
// alfabc = 1), every convective outflow face (code 21) has the old
// velocities (mf3d_bind_old_velocity).
static int inlets_ready(const mf3d_ctx *C, bool outflow = false) {
  if (!C->prm.bounds) return MF3D_OK;
  for (const auto &D : C->doms)
    for (const auto &S : D->blocks) {
      if (inlet_code(S->d) && !S->fld.inl) {
        set_error("bounds: block " + std::to_string(S->d.id) + " has west code " + std::to_string(S->d.bc_west) +
                  " and no inlet values (mf3d_set_inlet)");
        return MF3D_E_INVALID;
      }
      if (outflow && S->d.inext < 0 && S->d.bc_east == 21 && C->oo_bound.empty()) {
        set_error("bounds: block " + std::to_string(S->d.id) +
                  " has a convective outflow (code 21, alfabc 1) and no old velocities (mf3d_bind_old_velocity)");
        return MF3D_E_INVALID;
      }
      bool rough = false;
      if (wall_law_faces(S->d, &rough) && (C->wall_re <= 0.0 || (rough && C->wall_fric <= 0.0))) {
        set_error("bounds: block " + std::to_string(S->d.id) +
                  " has wall-function faces and no Re (or no fric for code 62): mf3d_set_wall_model");
        return MF3D_E_INVALID;
      }
    }
  return MF3D_OK;
}

// LMR (localparameters.for:26-102): a block's refinement rdiv is the
// coarsest block's spacing over its own, a power of two; params.ngrid is
// ngrd_gl = ngrid_input + log2(max rdiv), and a block of refinement r keeps
// ngrid_input + log2(r) levels of its own size (`own`).  rdv[b][g]
// (localparameters.for:47-57): r on the levels every block has, halving on
// the block's extra levels, 1 below its own.  Returns whether the layout
// mixes refinements; the rules of alloc_dom.for:12-230 (neighbours at most
// 2:1 apart, periodic partners equal) and the scope of the restatement (the
// V-cycle in FP64 on uniform blocks) are checked here.
static int lmr_plan(const mf3d_block_desc *blocks, int nb, const mf3d_params *prm, bool &lmr, std::vector<int> &own,
                    std::vector<std::vector<int>> &rdv) {
  lmr = false;
  own.assign(nb, prm->ngrid);
  rdv.assign(nb, std::vector<int>(prm->ngrid + 1, 1));
  double hmax = 0.0;
  for (int b = 0; b < nb; ++b) hmax = std::max(hmax, blocks[b].dx);
  std::vector<int> r(nb, 1), lg(nb, 0);
  int lg_max = 0;
  for (int b = 0; b < nb; ++b) {
    const mf3d_block_desc &d = blocks[b];
    const double x = hmax / d.dx;
    const long q = std::lround(x);
    if (!(d.dx > 0.0) || q < 1 || (q & (q - 1)) || std::fabs(x - (double)q) > 1e-8 * x ||
        std::fabs(blocks[0].dx / blocks[0].dy * d.dy - d.dx) > 1e-8 * d.dx ||
        std::fabs(blocks[0].dx / blocks[0].dz * d.dz - d.dx) > 1e-8 * d.dx) {
      set_error("block " + std::to_string(d.id) + ": spacings are not the coarsest block's over a power of two");
      return MF3D_E_INVALID;
    }
    r[b] = (int)q;
    while ((1 << lg[b]) < r[b]) ++lg[b];
    lg_max = std::max(lg_max, lg[b]);
    lmr |= q > 1;
  }
  if (!lmr) return MF3D_OK;
  if (prm->ngrid - lg_max < 1) {
    set_error("LMR: ngrid (ngrd_gl) must exceed log2 of the largest refinement");
    return MF3D_E_INVALID;
  }
  if (prm->lsm || prm->solver == 1 || prm->bounds) {
    set_error("LMR: the V-cycle runs without lsm, bounds or solver 1");
    return MF3D_E_UNSUPPORTED;
  }
  std::map<int, int> pos;
  for (int b = 0; b < nb; ++b) pos[blocks[b].id] = b;
  const int act = prm->ngrid - lg_max;
  for (int b = 0; b < nb; ++b) {
    const mf3d_block_desc &d = blocks[b];
    if (d.hx || d.hy || d.hz) {
      set_error("LMR: uniform spacing only (block " + std::to_string(d.id) + ")");
      return MF3D_E_UNSUPPORTED;
    }
    std::vector<int> nbr = {d.iprev, d.inext, d.jprev, d.jnext, d.kprev, d.knext};
    for (int q = 0; q < 4; ++q) { nbr.push_back(d.corprev[q]); nbr.push_back(d.cornext[q]); }
    for (int q = 0; q < 6; ++q) { nbr.push_back(d.edgprev[q]); nbr.push_back(d.edgnext[q]); }
    for (int id : nbr) {
      if (id < 0) continue;
      auto it = pos.find(id);
      if (it == pos.end()) { set_error("neighbour id " + std::to_string(id) + " not in the layout"); return MF3D_E_INVALID; }
      const int o = r[it->second];
      if (o != r[b] && o != 2 * r[b] && 2 * o != r[b]) {
        set_error("====ERROR===>  wrong rdiv " + std::to_string(d.id) + " (neighbours more than 2:1 apart)");
        return MF3D_E_INVALID;
      }
    }
    for (int id : {d.per_ip, d.per_in, d.per_jp, d.per_jn, d.per_kp, d.per_kn}) {
      auto it = pos.find(id);
      if (id >= 0 && it != pos.end() && r[it->second] != r[b]) {
        set_error("==ERROR==>wrong rdiv for a periodic partner of block " + std::to_string(d.id));
        return MF3D_E_INVALID;
      }
    }
    own[b] = act + lg[b];
    for (int g = 1; g <= prm->ngrid; ++g)
      rdv[b][g] = g > own[b] ? 1 : g <= act ? r[b] : rdv[b][g - 1] / 2;
  }
  return MF3D_OK;
}

static int create(const mf3d_block_desc *blocks, int nb, const mf3d_params *prm, mf3d_ctx **out) {
  if (!blocks || nb <= 0 || !out) { set_error("mf3d_create: bad arguments"); return MF3D_E_INVALID; }
  int st = check_params(prm);
  if (st) return st;
  bool lmr = false;
  std::vector<int> own;
  std::vector<std::vector<int>> rdv;
  if ((st = lmr_plan(blocks, nb, prm, lmr, own, rdv))) return st;
  for (int b = 0; b < nb; ++b) {
    const auto &d = blocks[b];
    const int pow2 = 1 << (own[b] - 1);
    if (d.nx < 1 || d.ny < 1 || d.nz < 1 || d.nx % pow2 || d.ny % pow2 || d.nz % pow2) {  // localparameters.for:201-206
      set_error("2:the given number not correct for mgsolver! (block " + std::to_string(d.id) +
                " not divisible by 2^(ngrid-1))");
      return MF3D_E_INVALID;
    }
    if (d.nx <= prm->pl_ex || d.ny <= prm->pl_ex || d.nz <= prm->pl_ex) {
      set_error("block " + std::to_string(d.id) + ": an edge does not exceed pl_ex");
      return MF3D_E_INVALID;
    }
    if (prm->bounds) {
      const int bcs[6] = {d.bc_west, d.bc_east, d.bc_south, d.bc_north, d.bc_bottom, d.bc_top};
      const int nbrs[6] = {d.iprev, d.inext, d.jprev, d.jnext, d.kprev, d.knext};
      for (int f = 0; f < 6; ++f)
        if (nbrs[f] < 0 && bounds_code_unsupported(f, bcs[f], prm->lsm != 0, prm->alfabc, true)) {
          set_error("bounds: block " + std::to_string(d.id) + " face " + std::to_string(f) + " has code " +
                    std::to_string(bcs[f]) + ", whose boundu/v/w branch needs data the library does not hold");
          return MF3D_E_UNSUPPORTED;
        }
    }
    if (prm->bounds && wall_law_faces(d)) {
      const int m = wall_law_faces(d);
      const int n[3] = {d.nx, d.ny, d.nz};
      for (int f = 0; f < 6; ++f)
        if (((m >> f) & 1) && n[f / 2] < 2) {
          set_error("bounds: a wall-function face of block " + std::to_string(d.id) +
                    " with one cell along its normal (the two faces' laws would read each other's updates)");
          return MF3D_E_UNSUPPORTED;
        }
      if (d.hx || d.hy || d.hz) {
        set_error("bounds: the wall functions of block " + std::to_string(d.id) + " read uniform spacings");
        return MF3D_E_UNSUPPORTED;
      }
    }
    if (prm->bounds && inlet_code(d) && d.bc_west != 7 && (d.hy || d.hz)) {
      set_error("bounds: the power-law inlet of block " + std::to_string(d.id) +
                " reads uniform cell centres (initial.for:341-365)");
      return MF3D_E_UNSUPPORTED;
    }
    if (prm->solver == 1 && (d.hx || d.hy || d.hz)) {
      set_error("solver 1 (SIP): uniform spacing only (pressure_1sweep, press.for:294-320)");
      return MF3D_E_UNSUPPORTED;
    }
    if (prm->lsm && (d.hx || d.hy || d.hz)) {
      set_error("lsm: uniform spacing only (the reference's variable-density branch)");
      return MF3D_E_UNSUPPORTED;
    }
    if (prm->differencing == 2 && (d.hx || d.hy || d.hz)) {
      set_error("differencing = 2: uniform spacing only (the reference's 4th-order divergence)");
      return MF3D_E_UNSUPPORTED;
    }
  }
  {
    std::vector<mf3d_block_desc> descs(blocks, blocks + nb);
    std::vector<FaceRule> rules;
    if ((st = face_rules(descs, rules))) return st;
  }
  auto C = std::make_unique<mf3d_ctx>();
  if ((st = ctx_init(C.get(), prm))) return st;
  AllocScope scope(C->stream);
  C->doms.emplace_back(new DomainStore());
  C->coarse64 = C->elem == 4 && prm->ngrid > 1;
  C->lmr = lmr;
  if ((st = build_domain(*C->doms[0], blocks, nb, prm->ngrid, C->elem, C->coarse64 ? 8 : C->elem, prm->pl,
                         C->stream, prm->lsm != 0, prm->bounds != 0, lmr ? -1 : prm->pl_ex, prm->differencing == 2,
                         lmr ? &own : nullptr, lmr ? &rdv : nullptr)))
    return st;
  if (prm->bounds) {
    const Extents e = domain_extents(blocks, nb);
    for (auto &S : C->doms[0]->blocks) {
      if (inlet_code(S->d) && (S->d.bc_west == 12 || S->d.bc_west == 13) &&
          (st = install_inlet(C.get(), *S, e, S->d.bc_west, 0, nullptr)))
        return st;
      if (wall_law_faces(S->d)) {
        // the wall stresses of the six faces, zero at the start
        // (initial.for:878-883) and kept across calls
        const long long ti = S->d.nx + 2 * prm->pl, tj = S->d.ny + 2 * prm->pl, tk = S->d.nz + 2 * prm->pl;
        S->fld.wplane = std::max(tj * tk, std::max(ti * tk, ti * tj));
        if ((st = S->wall.alloc((size_t)12 * S->fld.wplane))) return st;
        CK(cudaMemsetAsync(S->wall.p, 0, S->wall.n * sizeof(double), C->stream));
        S->fld.wtau = S->wall.p;
      }
    }
    CK(cudaStreamSynchronize(C->stream));
  }
  if ((st = make_view(C.get()))) return st;
  *out = C.release();
  return MF3D_OK;
}

// LMR contexts run the V-cycle only: the outer loop's field exchanges at
// refinement interfaces (exchangep.for, exchangeu/v/w.for) are not restated.
static int lmr_refused(const mf3d_ctx *C, const char *what) {
  if (!C || !C->lmr) return MF3D_OK;
  set_error(std::string(what) +
            ": an LMR layout (blocks of different refinement) runs mf3d_mgkcyc_device only; the field exchanges "
            "at refinement interfaces (exchangep.for, exchangeu/v/w.for) are not restated");
  return MF3D_E_UNSUPPORTED;
}

}  // namespace mf3d

// The deepest level count a domain allows: every edge divisible by 2^(L-1)
// with the coarsest edge >= 4 (at least one level).
int mf3d_max_levels(int nx, int ny, int nz) {
  int L = 1;
  while (true) {
    const int m = 1 << L;
    if (nx % m || ny % m || nz % m) break;
    if (nx / m < 4 || ny / m < 4 || nz / m < 4) break;
    ++L;
  }
  return L;
}

namespace mf3d {

// One block alone: no neighbours, periodic axes wrap onto itself.
static mf3d_block_desc lone_block(const mf3d_domain_desc &x) {
  mf3d_block_desc d;
  std::memset(&d, 0, sizeof d);
  d.id = 0;
  d.nx = x.nx; d.ny = x.ny; d.nz = x.nz;
  d.dx = x.dx; d.dy = x.dy; d.dz = x.dz;
  d.xel = x.nx * x.dx; d.yel = x.ny * x.dy; d.zel = x.nz * x.dz;
  d.iprev = d.inext = d.jprev = d.jnext = d.kprev = d.knext = -1;
  for (int q = 0; q < 4; ++q) d.corprev[q] = d.cornext[q] = -1;
  for (int q = 0; q < 6; ++q) d.edgprev[q] = d.edgnext[q] = -1;
  d.per_ip = d.per_in = d.per_jp = d.per_jn = d.per_kp = d.per_kn = -1;
  d.bc_west = d.bc_east = x.bc[0];
  d.bc_south = d.bc_north = x.bc[1];
  d.bc_bottom = d.bc_top = x.bc[2];
  d.hx = x.hx; d.hy = x.hy; d.hz = x.hz;
  return d;
}

// The final exchange(1..3) reads planes 1..pl_ex+1 inside each face.
static bool edges_exceed(const mf3d_domain_desc &x, int pl_ex) {
  return x.nx > pl_ex && x.ny > pl_ex && x.nz > pl_ex;
}

static int domain_ngrid(const mf3d_domain_desc &x) {
  if (x.nx < 1 || x.ny < 1 || x.nz < 1) return -1;
  if (x.ngrid <= 0) return mf3d_max_levels(x.nx, x.ny, x.nz);
  const int pow2 = 1 << (x.ngrid - 1);
  if (x.nx % pow2 || x.ny % pow2 || x.nz % pow2) return -1;
  return x.ngrid;
}

static int batch_create(const mf3d_domain_desc *doms, int nd, const mf3d_params *prm, mf3d_ctx **out) {
  if (!doms || nd <= 0 || !out) { set_error("mf3d_batch_create: bad arguments"); return MF3D_E_INVALID; }
  int st = check_params(prm);
  if (st) return st;
  if (prm->lsm || prm->bounds || prm->solver == 1) {
    set_error("lsm, bounds and solver 1: single-problem contexts (mf3d_create) only");
    return MF3D_E_UNSUPPORTED;
  }
  for (int d = 0; d < nd; ++d) {
    if (domain_ngrid(doms[d]) < 1) {
      set_error("domain " + std::to_string(d) + ": sizes not divisible by 2^(ngrid-1)");
      return MF3D_E_INVALID;
    }
    if (!edges_exceed(doms[d], prm->pl_ex)) {
      set_error("domain " + std::to_string(d) + ": an edge does not exceed pl_ex");
      return MF3D_E_INVALID;
    }
    if (prm->differencing == 2 && (doms[d].hx || doms[d].hy || doms[d].hz)) {
      set_error("differencing = 2: uniform spacing only (the reference's 4th-order divergence)");
      return MF3D_E_UNSUPPORTED;
    }
  }
  auto C = std::make_unique<mf3d_ctx>();
  if ((st = ctx_init(C.get(), prm))) return st;
  AllocScope scope(C->stream);
  // FP32 V-cycles keep an FP64 coarsest level when every domain bottoms out
  // on the same level (one launch per level needs one element type)
  bool same_depth = true;
  for (int d = 1; d < nd; ++d) same_depth &= domain_ngrid(doms[d]) == domain_ngrid(doms[0]);
  C->coarse64 = C->elem == 4 && same_depth && domain_ngrid(doms[0]) > 1;
  for (int d = 0; d < nd; ++d) {
    mf3d_block_desc b = lone_block(doms[d]);
    C->doms.emplace_back(new DomainStore());
    if ((st = build_domain(*C->doms.back(), &b, 1, domain_ngrid(doms[d]), C->elem, C->coarse64 ? 8 : C->elem,
                           prm->pl, C->stream)))
      return st;
  }
  if ((st = make_view(C.get()))) return st;
  *out = C.release();
  return MF3D_OK;
}

static int run_solve(mf3d_ctx *C, const double *dt, const double *alfapr, mf3d_solve_info *infos, double *hist,
                     int hcap) {
  if (C->prm.solver == 1) return solve_view_sip(C, *C->view, dt, alfapr, infos, hist, hcap);
  if (C->elem == 8) return solve_view<double>(C, *C->view, dt, alfapr, infos, hist, hcap);
  return solve_view<float>(C, *C->view, dt, alfapr, infos, hist, hcap);
}

// Host entry: mirror host arrays on the device (8 per block), solve, copy back.
static int host_solve(mf3d_ctx *C, const mf3d_fields *fields, const double *dt, const double *alfapr,
                      mf3d_solve_info *infos, double *hist, int hcap) {
  View &V = *C->view;
  cudaStream_t s = C->stream;
  const int nb = (int)V.blk.size();
  const int pl = C->prm.pl;
  if (!C->mirror.p) {
    size_t tot = 0;
    C->mirror_off.resize(nb);
    const size_t arrays = C->prm.lsm ? 9 : 8;  // + dens under L_LSM
    for (int b = 0; b < nb; ++b) { C->mirror_off[b] = tot; tot += arrays * ttc_elems(pl, V.blk[b]->d); }
    int st = C->mirror.alloc(tot);
    if (st) return st;
    CK(cudaStreamSynchronize(s));  // the side stream writes into it too
  }
  // ustar, vstar, wstar, p (and dens) on the solve stream.  u, v, w are
  // read only by the final calvel (and boundu/v/w), so they travel on a
  // side stream while the solve runs; the solve waits for them just before
  // that calvel.  Their wall values - all the solve reads of them earlier,
  // through the face planes - go straight from the caller's arrays into
  // those planes on the solve stream.  The side copies start only once the
  // inputs are in: both go host to device over one link, and the solve
  // waits for the inputs, not for u, v, w.
  if (!C->side) {
    CK(cudaStreamCreateWithFlags(&C->side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&C->ev_side, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&C->ev_in, cudaEventDisableTiming));
  }
  for (int b = 0; b < nb; ++b) {  // every pointer before any copy is queued
    const mf3d_fields &f = fields[b];
    if (!f.ustar || !f.vstar || !f.wstar || !f.u || !f.v || !f.w || !f.p) {
      set_error("mf3d_fields: a required pointer is NULL");
      return MF3D_E_INVALID;
    }
    if (C->prm.lsm && !f.dens) { set_error("mf3d_fields: dens is NULL under lsm"); return MF3D_E_INVALID; }
  }
  std::vector<mf3d_fields> dev(nb);
  for (int b = 0; b < nb; ++b) {
    const size_t n = ttc_elems(pl, V.blk[b]->d);
    double *m = C->mirror.p + C->mirror_off[b];
    double *const hsrc[4] = {fields[b].ustar, fields[b].vstar, fields[b].wstar, fields[b].p};
    const int q_of[4] = {0, 1, 2, 6};
    for (int q = 0; q < 4; ++q)
      CK(cudaMemcpyAsync(m + q_of[q] * n, hsrc[q], n * sizeof(double), cudaMemcpyHostToDevice, s));
    dev[b] = mf3d_fields{m, m + n, m + 2 * n, m + 3 * n, m + 4 * n, m + 5 * n, m + 6 * n,
                         fields[b].su ? m + 7 * n : nullptr, nullptr};
    if (C->prm.lsm) {
      CK(cudaMemcpyAsync(m + 8 * n, fields[b].dens, n * sizeof(double), cudaMemcpyHostToDevice, s));
      dev[b].dens = m + 8 * n;
    }
    // the wall planes of the normal velocity component, interior tangential
    // range, into lo / hi as k_face_planes lays them out
    const BlkFld &F = V.hf[b];
    const mf3d_block_desc &d = V.blk[b]->d;
    const size_t ti = d.nx + 2 * pl, tj = d.ny + 2 * pl;
    for (int f = 0; f < 6; ++f) {
      if (!F.wall[f]) continue;
      const int ax = f / 2, side = f & 1;
      const double *vel = ax == 0 ? fields[b].u : ax == 1 ? fields[b].v : fields[b].w;
      const int g = side ? (ax == 0 ? d.nx : ax == 1 ? d.ny : d.nz) : 0;  // local index of the wall face
      double *dst = side ? F.hi[ax] : F.lo[ax];
      // host element of local (i, j, k): (i+pl-1) + ti*((j+pl-1) + tj*(k+pl-1))
      auto at = [&](int i, int j, int k) {
        return vel + (size_t)(i + pl - 1) + ti * ((size_t)(j + pl - 1) + tj * (size_t)(k + pl - 1));
      };
      if (ax == 1) {  // rows of nx along i, one per k
        CK(cudaMemcpy2DAsync(dst, d.nx * sizeof(double), at(1, g, 1), ti * tj * sizeof(double), d.nx * sizeof(double),
                             d.nz, cudaMemcpyHostToDevice, s));
      } else if (ax == 2) {  // rows of nx along i, one per j
        CK(cudaMemcpy2DAsync(dst, d.nx * sizeof(double), at(1, 1, g), ti * sizeof(double), d.nx * sizeof(double),
                             d.ny, cudaMemcpyHostToDevice, s));
      } else {  // single values strided by ti along j and ti*tj along k
        cudaMemcpy3DParms p3;
        std::memset(&p3, 0, sizeof p3);
        p3.srcPtr = make_cudaPitchedPtr((void *)at(g, 1, 1), ti * sizeof(double), sizeof(double), tj);
        p3.dstPtr = make_cudaPitchedPtr(dst, sizeof(double), sizeof(double), d.ny);
        p3.extent = make_cudaExtent(sizeof(double), d.ny, d.nz);
        p3.kind = cudaMemcpyHostToDevice;
        CK(cudaMemcpy3DAsync(&p3, s));
      }
    }
  }
  CK(cudaEventRecord(C->ev_in, s));
  CK(cudaStreamWaitEvent(C->side, C->ev_in, 0));
  for (int b = 0; b < nb; ++b) {
    const size_t n = ttc_elems(pl, V.blk[b]->d);
    double *m = C->mirror.p + C->mirror_off[b];
    double *const hsrc[3] = {fields[b].u, fields[b].v, fields[b].w};
    for (int q = 0; q < 3; ++q)
      CK(cudaMemcpyAsync(m + (3 + q) * n, hsrc[q], n * sizeof(double), cudaMemcpyHostToDevice, C->side));
  }
  CK(cudaEventRecord(C->ev_side, C->side));
  C->walls_given = true;
  C->wait_side = true;
  int st = bind_fields(C, V, dev.data());
  if (!st) st = run_solve(C, dt, alfapr, infos, hist, hcap);
  C->walls_given = false;
  C->wait_side = false;
  if (st < 0) cudaStreamSynchronize(C->side);  // no copy outlives the call
  if (st < 0 && st != MF3D_E_NONFINITE) return st;
  for (int b = 0; b < nb; ++b) {
    const size_t n = ttc_elems(pl, V.blk[b]->d);
    double *m = C->mirror.p + C->mirror_off[b];
    double *const hdst[5] = {fields[b].u, fields[b].v, fields[b].w, fields[b].p, fields[b].su};
    const int q_of[5] = {3, 4, 5, 6, 7};
    for (int q = 0; q < 5; ++q) {
      if (!hdst[q]) continue;
      CK(cudaMemcpyAsync(hdst[q], m + q_of[q] * n, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
  }
  CK(cudaStreamSynchronize(s));
  return st;
}

}  // namespace mf3d

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int mf3d_abi_version(void) { return MF3D_ABI_VERSION; }

const char *mf3d_last_error(void) { return mf3d::g_err.c_str(); }

const char *mf3d_status_string(int s) {
  switch (s) {
    case MF3D_OK: return "ok";
    case MF3D_NOT_CONVERGED: return "not converged";
    case MF3D_DIVERGED: return "diverged (rmax > 100)";
    case MF3D_E_INVALID: return "invalid configuration";
    case MF3D_E_CUDA: return "CUDA error";
    case MF3D_E_OOM: return "out of device memory";
    case MF3D_E_TIMEOUT: return "device wait timed out";
    case MF3D_E_NONFINITE: return "non-finite residual";
    case MF3D_E_UNSUPPORTED: return "unsupported feature";
    default: return "unknown status";
  }
}

int mf3d_build_topology(int nblocks, const double *extents, const int *bc6, double dx, double dy, double dz,
                        mf3d_block_desc *out) {
  return mf3d::build_topology(nblocks, extents, bc6, dx, dy, dz, out);
}

int mf3d_create(const mf3d_block_desc *blocks, int nblocks, const mf3d_params *params, mf3d_ctx **ctx) {
  try {
    return mf3d::create(blocks, nblocks, params, ctx);
  } catch (const std::exception &e) {
    mf3d::set_error(std::string("mf3d_create: ") + e.what());
    return MF3D_E_OOM;
  }
}

int mf3d_batch_create(const mf3d_domain_desc *domains, int ndomains, const mf3d_params *params, mf3d_ctx **ctx) {
  try {
    return mf3d::batch_create(domains, ndomains, params, ctx);
  } catch (const std::exception &e) {
    mf3d::set_error(std::string("mf3d_batch_create: ") + e.what());
    return MF3D_E_OOM;
  }
}

int mf3d_destroy(mf3d_ctx *ctx) {
  if (!ctx) return MF3D_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->side) {
    cudaStreamSynchronize(ctx->side);
    cudaStreamDestroy(ctx->side);
  }
  if (ctx->ev_side) cudaEventDestroy(ctx->ev_side);
  if (ctx->ev_in) cudaEventDestroy(ctx->ev_in);
  ctx->view.reset();
  ctx->doms.clear();
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  for (auto e : ctx->prof_ev) cudaEventDestroy(e);
  cudaStream_t s = ctx->stream;
  delete ctx;
  if (s) cudaStreamDestroy(s);
  return MF3D_OK;
}

int mf3d_newsolv_mg_device(mf3d_ctx *C, const mf3d_fields *fields, double dt, double alfapr, mf3d_solve_info *info,
                           double *hist, int cap) {
  if (!C || !fields) { mf3d::set_error("mf3d_newsolv_mg_device: bad arguments"); return MF3D_E_INVALID; }
  if (int st_lmr = mf3d::lmr_refused(C, "mf3d_newsolv_mg_device")) return st_lmr;
  if (C->view->dom.size() != 1) { mf3d::set_error("a batch context: use mf3d_batch_solve_device"); return MF3D_E_INVALID; }
  if (cudaSetDevice(C->device) != cudaSuccess) { mf3d::set_error("cudaSetDevice failed"); return MF3D_E_CUDA; }
  mf3d::AllocScope scope(C->stream);
  int st = mf3d::inlets_ready(C, C->prm.alfabc == 1);
  if (st) return st;
  if ((st = mf3d::bind_fields(C, *C->view, fields))) return st;
  return mf3d::run_solve(C, &dt, &alfapr, info, hist, cap);
}

int mf3d_rungek_2nd_device(mf3d_ctx *C, const mf3d_fields *fields, const mf3d_rk_fields *rk, double dt,
                           double alfapr, int alfabc, int pressureforce, double forcn) {
  using namespace mf3d;
  if (int st_lmr = mf3d::lmr_refused(C, "mf3d_rungek_2nd_device")) return st_lmr;
  if (!C || !fields || !rk) { set_error("mf3d_rungek_2nd_device: bad arguments"); return MF3D_E_INVALID; }
  if (C->view->dom.size() != 1) { set_error("mf3d_rungek_2nd_device: mf3d_create contexts only"); return MF3D_E_INVALID; }
  if (!C->prm.bounds || C->prm.lsm || C->elem != 8) {
    set_error("mf3d_rungek_2nd_device: needs a context with bounds = 1, FP64 and no lsm");
    return MF3D_E_UNSUPPORTED;
  }
  if ((C->prm.differencing == 2 || C->prm.differencing == 3) && C->prm.pl < 3) {
    set_error("mf3d_rungek_2nd_device: the 4th-order and WENO stages read three ghost layers (pl >= 3)");
    return MF3D_E_INVALID;
  }
  if (int st = inlets_ready(C)) return st;
  View &V = *C->view;
  for (size_t b = 0; b < V.blk.size(); ++b) {
    const mf3d_block_desc &d = V.blk[b]->d;
    if (d.hx || d.hy || d.hz) { set_error("mf3d_rungek_2nd_device: uniform spacing only"); return MF3D_E_UNSUPPORTED; }
    const int bcs[6] = {d.bc_west, d.bc_east, d.bc_south, d.bc_north, d.bc_bottom, d.bc_top};
    const int nbrs[6] = {d.iprev, d.inext, d.jprev, d.jnext, d.kprev, d.knext};
    for (int f = 0; f < 6; ++f)
      if (nbrs[f] < 0 && bounds_code_unsupported(f, bcs[f], false, alfabc, true)) {
        set_error("mf3d_rungek_2nd_device: face code " + std::to_string(bcs[f]) + " with alfabc " +
                  std::to_string(alfabc) + " reads data the library does not hold");
        return MF3D_E_UNSUPPORTED;
      }
    if (!rk[b].uoo || !rk[b].voo || !rk[b].woo || !rk[b].vis) {
      set_error("mf3d_rk_fields: a pointer is NULL");
      return MF3D_E_INVALID;
    }
  }
  // Every entry is valid: bind the caller's buffers for this call only; the
  // guard unbinds them on every way out, so no later upload of the field
  // table carries a pointer the caller may have freed.
  struct Unbind {
    View &V;
    ~Unbind() {
      for (auto &F : V.hf) {
        F.oo[0] = F.oo[1] = F.oo[2] = nullptr;
        F.vis = nullptr;
      }
    }
  } unbind{V};
  for (size_t b = 0; b < V.blk.size(); ++b) {
    for (int a = 0; a < 3; ++a) V.hf[b].oo[a] = a == 0 ? rk[b].uoo : a == 1 ? rk[b].voo : rk[b].woo;
    V.hf[b].vis = rk[b].vis;
  }
  if (cudaSetDevice(C->device) != cudaSuccess) { set_error("cudaSetDevice failed"); return MF3D_E_CUDA; }
  AllocScope scope(C->stream);
  int st = bind_fields(C, V, fields);
  if (st) return st;
  cudaStream_t s = C->stream;
  C->launches = 0;
  CK(cudaMemsetAsync(V.ds.p, 0, V.ds.n * sizeof(DomState), s));  // no domain marked diverged
  // rungek_conv2nd: boundu, the u loop, boundv, the v loop, boundw, the w
  // loop - each component's predictor sees the other components' ghosts as
  // they were before their own bound; rungek_diff2nd fused per component
  for (int comp = 0; comp < 3; ++comp) {
    bc_walks(C, V, comp);
    bound_faces(C, V, alfabc, comp, dt, alfapr);
    if (C->prm.differencing == 2)
      launch(k_rk4th, V.n_int, dim3(RW_TX, RW_RJ), 0, s, V.df.p, V.t_int.p, comp, dt, alfapr, pressureforce, forcn);
    else if (C->prm.differencing == 3)
      launch(k_rkweno, V.n_int, dim3(RW_TX, RW_RJ), 0, s, V.df.p, V.t_int.p, comp, C->prm.pl_ex, dt, alfapr,
             pressureforce, forcn);
    else
      launch(k_rk2nd, V.n_int, dim3(RW_TX, RW_RJ), 0, s, V.df.p, V.t_int.p, comp, dt, alfapr, pressureforce, forcn);
    ++C->launches;
  }
  const cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) { set_error(std::string("mf3d_rungek_2nd_device: ") + cudaGetErrorString(e)); return MF3D_E_CUDA; }
  return check_device_error(V);
}

int mf3d_bounds_device(mf3d_ctx *C, const mf3d_fields *fields, double dt, double alfapr, int alfabc) {
  using namespace mf3d;
  if (int st_lmr = mf3d::lmr_refused(C, "mf3d_bounds_device")) return st_lmr;
  if (!C || !fields) { set_error("mf3d_bounds_device: bad arguments"); return MF3D_E_INVALID; }
  if (C->view->dom.size() != 1) { set_error("mf3d_bounds_device: mf3d_create contexts only"); return MF3D_E_INVALID; }
  if (!C->prm.bounds || C->elem != 8) {
    set_error("mf3d_bounds_device: needs a context with bounds = 1, FP64");
    return MF3D_E_UNSUPPORTED;
  }
  View &V = *C->view;
  for (size_t b = 0; b < V.blk.size(); ++b) {
    const mf3d_block_desc &d = V.blk[b]->d;
    const int bcs[6] = {d.bc_west, d.bc_east, d.bc_south, d.bc_north, d.bc_bottom, d.bc_top};
    const int nbrs[6] = {d.iprev, d.inext, d.jprev, d.jnext, d.kprev, d.knext};
    for (int f = 0; f < 6; ++f)
      if (nbrs[f] < 0 && bounds_code_unsupported(f, bcs[f], C->prm.lsm != 0, alfabc, true)) {
        set_error("mf3d_bounds_device: face code " + std::to_string(bcs[f]) + " reads data the library does not hold");
        return MF3D_E_UNSUPPORTED;
      }
  }
  if (int st = inlets_ready(C, alfabc == 1)) return st;
  if (cudaSetDevice(C->device) != cudaSuccess) { set_error("cudaSetDevice failed"); return MF3D_E_CUDA; }
  AllocScope scope(C->stream);
  int st = bind_fields(C, V, fields);
  if (st) return st;
  C->launches = 0;
  CK(cudaMemsetAsync(V.ds.p, 0, V.ds.n * sizeof(DomState), C->stream));  // no domain marked diverged
  // boundu, boundv, boundw, each with its periodic copy first
  for (int comp = 0; comp < 3; ++comp) {
    bc_walks(C, V, comp);
    bound_faces(C, V, alfabc, comp, dt, alfapr);
  }
  const cudaError_t e = cudaStreamSynchronize(C->stream);
  if (e != cudaSuccess) { set_error(std::string("mf3d_bounds_device: ") + cudaGetErrorString(e)); return MF3D_E_CUDA; }
  return check_device_error(V);
}

int mf3d_calvel_device(mf3d_ctx *C, const mf3d_fields *fields, double dt, double alfapr) {
  using namespace mf3d;
  if (int st_lmr = mf3d::lmr_refused(C, "mf3d_calvel_device")) return st_lmr;
  if (!C || !fields) { set_error("mf3d_calvel_device: bad arguments"); return MF3D_E_INVALID; }
  if (C->view->dom.size() != 1) { set_error("mf3d_calvel_device: mf3d_create contexts only"); return MF3D_E_INVALID; }
  if (C->prm.lsm || C->elem != 8) { set_error("mf3d_calvel_device: FP64 contexts without lsm"); return MF3D_E_UNSUPPORTED; }
  if (cudaSetDevice(C->device) != cudaSuccess) { set_error("cudaSetDevice failed"); return MF3D_E_CUDA; }
  View &V = *C->view;
  AllocScope scope(C->stream);
  int st = bind_fields(C, V, fields);
  if (st) return st;
  cudaStream_t s = C->stream;
  C->launches = 0;
  DomState d0;
  std::memset(&d0, 0, sizeof d0);
  d0.dt = dt;
  d0.alfapr = alfapr;
  CK(cudaMemcpyAsync(V.ds.p, &d0, sizeof d0, cudaMemcpyHostToDevice, s));
  launch(k_calvel, V.n_int, dim3(RW_TX, RW_RJ), 0, s, V.df.p, V.t_int.p, V.ds.p, nullptr);
  ++C->launches;
  // exchange(1..3) (press.for:196-198): every ghost it writes, edges and
  // corners included, which the next predictor stage reads; its chained
  // sources are the caller's ghosts as they stand (saved first)
  if (V.nfx_uvw) {
    if (V.nfxe_chain && !V.fx_per_iteration) {
      launch(k_fx_evolve, grid_of(V.nfxe_chain, kTile), kTile, 0, s, V.df.p, V.ds.p, (const int *)nullptr,
             V.fxe_cells, 0LL, V.fxe_chain, V.nfxe_chain, V.fx_prev.p, V.fxe_sub, 0LL, V.fx_stage.p);
      ++C->launches;
    }
    C->launches += field_exchange(C, V, V.fx_uvw, V.nfx_uvw, V.nsfx_uvw, nullptr,
                                  V.fx_per_iteration ? nullptr : V.fx_prev.p);
  } else {
    if (C->prm.bounds) bc_walks(C, V);  // the full periodic planes of exchange(1..3)
    launch(k_vel_faces, V.n_vfaces, kTile, 0, s, V.df.p, V.t_vfaces.p, nullptr, C->prm.pl_ex);
    ++C->launches;
  }
  const cudaError_t e = cudaStreamSynchronize(s);  // d0 is a local
  if (e != cudaSuccess) { set_error(std::string("mf3d_calvel_device: ") + cudaGetErrorString(e)); return MF3D_E_CUDA; }
  return MF3D_OK;
}

int mf3d_newsolv_mg(mf3d_ctx *C, const mf3d_fields *fields, double dt, double alfapr, mf3d_solve_info *info,
                    double *hist, int cap) {
  if (!C || !fields) { mf3d::set_error("mf3d_newsolv_mg: bad arguments"); return MF3D_E_INVALID; }
  if (int st_lmr = mf3d::lmr_refused(C, "mf3d_newsolv_mg")) return st_lmr;
  if (C->view->dom.size() != 1) { mf3d::set_error("a batch context: use mf3d_batch_solve_device"); return MF3D_E_INVALID; }
  if (cudaSetDevice(C->device) != cudaSuccess) { mf3d::set_error("cudaSetDevice failed"); return MF3D_E_CUDA; }
  mf3d::AllocScope scope(C->stream);
  if (int st = mf3d::inlets_ready(C, C->prm.alfabc == 1)) return st;
  return mf3d::host_solve(C, fields, &dt, &alfapr, info, hist, cap);
}

int mf3d_batch_solve_device(mf3d_ctx *C, const mf3d_fields *fields, const double *dt, const double *alfapr,
                            mf3d_solve_info *infos, double *hist, int hcap) {
  if (!C || !fields || !dt || !alfapr) { mf3d::set_error("mf3d_batch_solve_device: bad arguments"); return MF3D_E_INVALID; }
  if (cudaSetDevice(C->device) != cudaSuccess) { mf3d::set_error("cudaSetDevice failed"); return MF3D_E_CUDA; }
  mf3d::AllocScope scope(C->stream);
  int st = mf3d::bind_fields(C, *C->view, fields);
  if (st) return st;
  return mf3d::run_solve(C, dt, alfapr, infos, hist, hcap);
}

int mf3d_mgkcyc_device(mf3d_ctx *C, double *const *su, double *const *pp) {
  if (!C || !su || !pp) { mf3d::set_error("mf3d_mgkcyc_device: bad arguments"); return MF3D_E_INVALID; }
  if (C->prm.lsm) { mf3d::set_error("lsm: the coefficients come from a solve's dens"); return MF3D_E_UNSUPPORTED; }
  if (cudaSetDevice(C->device) != cudaSuccess) { mf3d::set_error("cudaSetDevice failed"); return MF3D_E_CUDA; }
  mf3d::AllocScope scope(C->stream);
  if (C->elem == 8) return mf3d::mgkcyc_view<double>(C, *C->view, su, pp);
  return mf3d::mgkcyc_view<float>(C, *C->view, su, pp);
}

int mf3d_mgkcyc_device_noalloc(mf3d_ctx *C, double *const *su, double *const *pp) {
  if (!C || !su || !pp) { mf3d::set_error("mf3d_mgkcyc_device_noalloc: bad arguments"); return MF3D_E_INVALID; }
  if (int st_lmr = mf3d::lmr_refused(C, "mf3d_mgkcyc_device_noalloc")) return st_lmr;
  if (C->prm.lsm) { mf3d::set_error("lsm: the coefficients come from a solve's dens"); return MF3D_E_UNSUPPORTED; }
  if (cudaSetDevice(C->device) != cudaSuccess) { mf3d::set_error("cudaSetDevice failed"); return MF3D_E_CUDA; }
  if (C->elem == 8) return mf3d::mgkcyc_view_noalloc<double>(C, *C->view, su, pp);
  return mf3d::mgkcyc_view_noalloc<float>(C, *C->view, su, pp);
}

long long mf3d_last_launch_count(const mf3d_ctx *C) { return C ? C->launches : 0; }

int mf3d_set_wall_model(mf3d_ctx *C, double re, double fric) {
  if (!C || !C->view || C->doms.size() != 1 || !(re >= 0.0) || !(fric >= 0.0)) {
    mf3d::set_error("mf3d_set_wall_model: bad arguments");
    return MF3D_E_INVALID;
  }
  if (cudaSetDevice(C->device) != cudaSuccess) { mf3d::set_error("cudaSetDevice failed"); return MF3D_E_CUDA; }
  C->wall_re = re;
  C->wall_fric = fric;
  for (auto &S : C->doms[0]->blocks)
    if (S->wall.p && cudaMemsetAsync(S->wall.p, 0, S->wall.n * sizeof(double), C->stream) != cudaSuccess) {
      mf3d::set_error("mf3d_set_wall_model: clearing the wall stresses failed");
      return MF3D_E_CUDA;
    }
  if (cudaStreamSynchronize(C->stream) != cudaSuccess) { mf3d::set_error("mf3d_set_wall_model: sync"); return MF3D_E_CUDA; }
  return MF3D_OK;
}

int mf3d_bind_old_velocity(mf3d_ctx *C, const mf3d_rk_fields *rk) {
  if (!C || !C->view || C->doms.size() != 1) { mf3d::set_error("mf3d_bind_old_velocity: bad arguments"); return MF3D_E_INVALID; }
  mf3d::View &V = *C->view;
  if (!rk) {
    C->oo_bound.clear();
    for (auto &F : V.hf) F.oo[0] = F.oo[1] = F.oo[2] = nullptr;
    return MF3D_OK;
  }
  std::vector<std::array<const double *, 3>> oo(V.blk.size());
  for (size_t b = 0; b < V.blk.size(); ++b) {
    if (!rk[b].uoo || !rk[b].voo || !rk[b].woo) {
      mf3d::set_error("mf3d_bind_old_velocity: a pointer is NULL");
      return MF3D_E_INVALID;
    }
    oo[b] = {rk[b].uoo, rk[b].voo, rk[b].woo};
  }
  C->oo_bound = oo;
  for (size_t b = 0; b < V.blk.size(); ++b)
    for (int a = 0; a < 3; ++a) V.hf[b].oo[a] = oo[b][a];
  return MF3D_OK;
}

int mf3d_set_inlet(mf3d_ctx *C, int block_id, int code, int uprof_sem, const double *values, long long n) {
  if (!C || !values || C->doms.size() != 1 || !C->view) {
    mf3d::set_error("mf3d_set_inlet: bad arguments");
    return MF3D_E_INVALID;
  }
  if (!C->prm.bounds) { mf3d::set_error("mf3d_set_inlet: a context with bounds = 1"); return MF3D_E_INVALID; }
  mf3d::DomainStore &D = *C->doms[0];
  for (size_t b = 0; b < D.blocks.size(); ++b) {
    mf3d::BlockStore &S = *D.blocks[b];
    if (S.d.id != block_id) continue;
    if (S.d.iprev >= 0 || S.d.bc_west != code || (code != 7 && code != 8)) {
      mf3d::set_error("mf3d_set_inlet: block " + std::to_string(block_id) + " has no west face of code " +
                      std::to_string(code) + " (7 or 8)");
      return MF3D_E_INVALID;
    }
    const long long want = mf3d::inlet_count(S.d, code);
    if (n != want) {
      mf3d::set_error("mf3d_set_inlet: " + std::to_string(want) + " values expected, got " + std::to_string(n));
      return MF3D_E_INVALID;
    }
    if (code == 8 && uprof_sem == 12 && (S.d.hy || S.d.hz)) {
      mf3d::set_error("mf3d_set_inlet: the power-law profile reads uniform cell centres");
      return MF3D_E_UNSUPPORTED;
    }
    if (cudaSetDevice(C->device) != cudaSuccess) { mf3d::set_error("cudaSetDevice failed"); return MF3D_E_CUDA; }
    std::vector<mf3d_block_desc> descs;
    for (auto &T : D.blocks) descs.push_back(T->d);
    int st = mf3d::install_inlet(C, S, mf3d::domain_extents(descs.data(), (int)descs.size()), code, uprof_sem, values);
    if (st) return st;
    // the view's copy of the block (the solve uploads it with the fields)
    for (size_t v = 0; v < C->view->blk.size(); ++v)
      if (C->view->blk[v] == &S) {
        C->view->hf[v].inl = S.fld.inl;
        for (int c = 0; c < 3; ++c) {
          C->view->hf[v].inl_s1[c] = S.fld.inl_s1[c];
          C->view->hf[v].inl_t1[c] = S.fld.inl_t1[c];
        }
      }
    return MF3D_OK;
  }
  mf3d::set_error("mf3d_set_inlet: no block " + std::to_string(block_id));
  return MF3D_E_INVALID;
}

int mf3d_tuning(const mf3d_ctx *C, int level, int *sweep_schedule, int *small_sweep, int *restrict_planes,
                int *cluster_ctas) {
  if (!C || !C->view || level < 1 || level > C->view->Lmax) { mf3d::set_error("mf3d_tuning: bad arguments"); return MF3D_E_INVALID; }
  const mf3d::ViewLevel &L = C->view->lv[level];
  if (sweep_schedule) *sweep_schedule = L.sched;
  if (small_sweep) *small_sweep = L.small;
  if (restrict_planes) *restrict_planes = level > 1 ? (L.n_rtma ? L.rtma_kch : -1) : 0;
  if (cluster_ctas) *cluster_ctas = C->prm.mg_itrsch == 2 ? L.td_cl : C->prm.mg_itrsch == 1 ? L.lx_cl : 1;
  return MF3D_OK;
}

int mf3d_test_fail_alloc(long long after) {
  mf3d::g_fail_alloc_countdown.store(after < 0 ? -1 : after);
  return MF3D_OK;
}

int mf3d_test_stall_copy(int device, int bytes) {
  if (bytes < 0 || bytes > 65536) { mf3d::set_error("mf3d_test_stall_copy: bytes out of range"); return MF3D_E_INVALID; }
  if (cudaSetDevice(device) != cudaSuccess) { mf3d::set_error("cudaSetDevice failed"); return MF3D_E_CUDA; }
  const cudaError_t e = cudaMemcpyToSymbol(mf3d::g_test_extra_tx, &bytes, sizeof(int));
  if (e != cudaSuccess) { mf3d::set_error(std::string("mf3d_test_stall_copy: ") + cudaGetErrorString(e)); return MF3D_E_CUDA; }
  return MF3D_OK;
}

int mf3d_profile(mf3d_ctx *C, int kind) {
  if (!C || kind < 0 || kind > MF3D_PROF_PROLONG_L1) { mf3d::set_error("mf3d_profile: bad arguments"); return MF3D_E_INVALID; }
  C->prof_kind = kind;
  C->prof_ms = 0.0; C->prof_bytes = 0.0; C->prof_n = 0;
  C->prof_pending_bytes.clear();
  return MF3D_OK;
}

int mf3d_profile_read(mf3d_ctx *C, double *total_ms, long long *launches, double *bytes) {
  if (!C) { mf3d::set_error("mf3d_profile_read: bad arguments"); return MF3D_E_INVALID; }
  if (total_ms) *total_ms = C->prof_ms;
  if (launches) *launches = C->prof_n;
  if (bytes) *bytes = C->prof_bytes;
  return MF3D_OK;
}

int mf3d_selftest_divide(const double *x, const double *b, long long n, double *q, double *qref, int device) {
  if (!x || !b || !q || !qref || n < 0) { mf3d::set_error("mf3d_selftest_divide: bad arguments"); return MF3D_E_INVALID; }
  if (n == 0) return MF3D_OK;
  CK(cudaSetDevice(device));
  std::vector<double> rb(n);
  for (long long i = 0; i < n; ++i) rb[i] = div_reciprocal(b[i]);
  double *d = nullptr;
  CK(cudaMalloc(&d, (size_t)n * 5 * sizeof(double)));
  std::unique_ptr<double, decltype(&cudaFree)> hold(d, &cudaFree);
  CK(cudaMemcpy(d, x, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d + n, b, n * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d + 2 * n, rb.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  mf3d::k_selftest_divide<<<(int)((n + 255) / 256), 256>>>(d, d + n, d + 2 * n, n, d + 3 * n, d + 4 * n);
  CK(cudaGetLastError());
  CK(cudaMemcpy(q, d + 3 * n, n * sizeof(double), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(qref, d + 4 * n, n * sizeof(double), cudaMemcpyDeviceToHost));
  return MF3D_OK;
}

long long mf3d_halo_map(const mf3d_block_desc *blocks, int nblocks, int ngrid, int level, long long *dst,
                        long long *src) {
  if (!blocks || nblocks <= 0 || level < 1 || level > ngrid) return -1;
  std::vector<mf3d_block_desc> b(blocks, blocks + nblocks);
  std::vector<mf3d::LevelGeom> geom(nblocks);
  std::vector<long long> base(nblocks);
  long long acc = 0;
  for (int q = 0; q < nblocks; ++q) {
    geom[q] = mf3d::LevelGeom{b[q].nx >> (level - 1), b[q].ny >> (level - 1), b[q].nz >> (level - 1)};
    base[q] = acc;
    acc += geom[q].cells();
  }
  auto pairs = mf3d::build_halo_map(b, geom, base);
  if (dst && src)
    for (size_t q = 0; q < pairs.size(); ++q) { dst[q] = pairs[q].dst; src[q] = pairs[q].src; }
  return (long long)pairs.size();
}

int mf3d_halo_refresh_host(const mf3d_block_desc *blocks, int nblocks, int ngrid, int level, double *const *fi) {
  if (!blocks || nblocks <= 0 || !fi || ngrid < 1 || level < 1 || level > ngrid) {
    mf3d::set_error("mf3d_halo_refresh_host: bad arguments");
    return MF3D_E_INVALID;
  }
  try {
    mf3d_params prm;
    std::memset(&prm, 0, sizeof prm);
    prm.ngrid = ngrid;
    prm.mg_itrsch = 3;
    prm.pl = 1;
    prm.differencing = 1;
    bool lmr = false;
    std::vector<int> own;
    std::vector<std::vector<int>> rdv;
    if (int st = mf3d::lmr_plan(blocks, nblocks, &prm, lmr, own, rdv)) return st;
    std::vector<mf3d_block_desc> b(blocks, blocks + nblocks);
    std::vector<mf3d::LevelGeom> geom(nblocks);
    std::vector<long long> base(nblocks);
    std::vector<int> rg(nblocks);
    long long acc = 0;
    bool mixed = false;
    for (int q = 0; q < nblocks; ++q) {
      const int gl = std::min(level, own[q]);
      geom[q] = mf3d::LevelGeom{b[q].nx >> (gl - 1), b[q].ny >> (gl - 1), b[q].nz >> (gl - 1)};
      base[q] = acc;
      acc += geom[q].cells();
      rg[q] = rdv[q][level];
      mixed |= rg[q] != rg[0];
    }
    auto cell = [&](long long id) -> double & {
      const int q = (int)(std::upper_bound(base.begin(), base.end(), id) - base.begin()) - 1;
      return fi[q][id - base[q]];
    };
    if (mixed) {
      // k_lmr_nodes / k_lmr_write on the host
      const mf3d::LmrProgram P = mf3d::build_halo_lmr(b, geom, base, rg);
      std::vector<double> val(P.nodes.size());
      for (size_t n = 0; n < P.nodes.size(); ++n) {
        const auto &N = P.nodes[n];
        double t = 0.0;
        for (int q = 0; q < N.nt; ++q) {
          const auto &a = P.terms[N.t0 + q];
          const double x = a.ref >= 0 ? cell(a.ref) : a.ref == mf3d::kLmrZero ? 0.0 : val[(size_t)(-2 - a.ref)];
          t = q == 0 ? a.w * x : t + a.w * x;
        }
        val[n] = t * N.scale;
      }
      for (auto &w : P.writes) cell(w.first) = val[w.second];
      for (auto &c : P.copies) cell(c.first) = cell(c.second);  // sources no write touches
    } else {
      const auto pairs = mf3d::build_halo_map(b, geom, base);
      std::vector<double> v(pairs.size());
      for (size_t q = 0; q < pairs.size(); ++q) v[q] = cell(pairs[q].src);
      for (size_t q = 0; q < pairs.size(); ++q) cell(pairs[q].dst) = v[q];
    }
  } catch (const std::exception &e) {
    mf3d::set_error(std::string("mf3d_halo_refresh_host: ") + e.what());
    return MF3D_E_OOM;
  }
  return MF3D_OK;
}

long long mf3d_field_exchange_map(const mf3d_block_desc *blocks, int nblocks, int pl, int pl_ex, int op,
                                  long long *dst, long long *src) {
  if (!blocks || nblocks <= 0 || pl < 1 || pl_ex < 0 || pl_ex >= pl || op < 1 || op > 4) return -1;
  std::vector<mf3d_block_desc> b(blocks, blocks + nblocks);
  std::vector<long long> base(nblocks);
  long long acc = 0;
  for (int q = 0; q < nblocks; ++q) {
    if (b[q].nx <= pl_ex || b[q].ny <= pl_ex || b[q].nz <= pl_ex) return -1;
    base[q] = acc;
    acc += (long long)(b[q].nx + 2 * pl) * (b[q].ny + 2 * pl) * (b[q].nz + 2 * pl);
  }
  auto pairs = mf3d::build_field_map(b, base, pl, op, op == 4 ? 0 : pl_ex, op == 4);
  if (dst && src)
    for (size_t q = 0; q < pairs.size(); ++q) { dst[q] = pairs[q].dst; src[q] = pairs[q].src; }
  return (long long)pairs.size();
}

}  // extern "C"

// Serving (request loop over this engine).
#include "server.cuh"
// Restart files of the reference, decoded and encoded on the device.
#include "tecbin.cuh"
