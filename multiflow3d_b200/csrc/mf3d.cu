// libmf3d: B200 (sm_100a) pressure-Poisson multigrid for MultiFlow3D's
// projection step.  Host driver (C++) + C ABI of include/mf3d.h.
//
// One context = one device, one stream, all blocks of the solve resident.
// The reference's per-rank MPI halo traffic becomes on-device copies; its
// module state (vars, multidata) becomes the context.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "kernels.cuh"
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

template <typename T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  ~DevBuf() { if (p) cudaFree(p); }
  int alloc(size_t count) {
    if (p) { cudaFree(p); p = nullptr; }
    n = count;
    if (count == 0) return MF3D_OK;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
      return e == cudaErrorMemoryAllocation ? MF3D_E_OOM : MF3D_E_CUDA;
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

// Tile list: for each block, ceil(items_b / kTile) CTAs.
static std::vector<Tile> make_tiles(const std::vector<long long> &items) {
  std::vector<Tile> t;
  for (size_t b = 0; b < items.size(); ++b)
    for (long long s = 0; s < items[b]; s += kTile) t.push_back(Tile{(int)b, (int)s});
  return t;
}

// One multigrid level of every block, storage type T.
template <typename T>
struct Level {
  int g = 0;
  std::vector<BlkLev> hb;
  DevBuf<BlkLev> db;
  DevBuf<T> phi, rhs, coef, geo;
  DevBuf<Tile> t_sweep, t_cells;
  int n_sweep = 0, n_cells = 0;
  DevBuf<long long> hdst, hsrc;
  DevBuf<T> hbuf;
  int nhalo = 0, nstaged = 0;
  DevBuf<T> tdma_work;
  int ngg = 0;
  bool zero_interior = false;  // interior known to be all zero (right after mgrestr)
};

}  // namespace mf3d

using namespace mf3d;

struct mf3d_ctx {
  mf3d_params prm;
  std::vector<mf3d_block_desc> blocks;
  int nb = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  long long launches = 0;
  // hierarchy (one of the two is used, by precision)
  std::vector<std::unique_ptr<Level<double>>> L64;
  std::vector<std::unique_ptr<Level<float>>> L32;
  // fields
  std::vector<BlkFld> hf;
  DevBuf<BlkFld> df;
  std::vector<FaceRule> rules;
  DevBuf<double> widths, planes;  // geometry, face planes
  DevBuf<double> mirror;          // device mirrors of host fields (host entry point)
  std::vector<size_t> mirror_off;
  DevBuf<Tile> t_int, t_l1cells, t_faces, t_planes;
  int n_int = 0, n_l1cells = 0, n_faces = 0, n_planes = 0;
  DevBuf<unsigned long long> rmax_cur, rmax_scratch;  // atomic-max targets of calmas
  DevBuf<SolveState> st;                     // device-resident solve control
  DevBuf<double> hist_d;                     // rmax after each outer iteration
  unsigned long long *rmax_host = nullptr;  // pinned
  bool use_graph = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraphConditionalHandle cond = 0;
  long long launches_per_iter = 0;
  DevBuf<double *> ptrs;                     // scratch pointer table (mgkcyc_device)
  // kernel timing (mf3d_profile)
  int prof_kind = 0;
  std::vector<cudaEvent_t> prof_ev;          // reusable event pool
  std::vector<double> prof_pending_bytes;    // one entry per bracketed launch
  double prof_ms = 0.0, prof_bytes = 0.0;
  long long prof_n = 0;
  long long n_l1 = 0;                        // finest-level interior cells, all blocks
};

namespace mf3d {

static inline int grid_of(long long n, int tpb) { return (int)((n + tpb - 1) / tpb); }

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
// After a stream synchronize: fold the bracketed launches into the totals.
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

// ---------------------------------------------------------------------------
// Level construction (replaces coeff, mgsolver.for:2-222, and the cof sizing
// of localparameters.for:208-237).
// ---------------------------------------------------------------------------
template <typename T>
static int build_level(mf3d_ctx *C, Level<T> &L, int g) {
  L.g = g;
  const int nb = C->nb;
  const int ngrid = C->prm.ngrid;
  std::vector<T> coef, geo;
  long long phi_off = 0;
  std::vector<long long> it_sweep, it_cells;
  std::vector<LevelGeom> geom(nb);
  std::vector<long long> base(nb);
  long long cell_base = 0;
  L.hb.resize(nb);
  for (int b = 0; b < nb; ++b) {
    const mf3d_block_desc &d = C->blocks[b];
    BlkLev &B = L.hb[b];
    B.nx = d.nx >> (g - 1);
    B.ny = d.ny >> (g - 1);
    B.nz = d.nz >> (g - 1);
    B.hp = hp_of(B.nx);
    B.cstr = (long long)(B.nz + 2) * (B.ny + 2) * B.hp;
    B.cstr = (B.cstr + 31) / 32 * 32;  // 256-byte aligned colour arrays (FP64)
    B.phi0 = phi_off;
    B.rhs0 = phi_off;
    phi_off += 2 * B.cstr;
    B.pos = b;
    B.nmask = 0;
    const int nbr[6] = {d.iprev, d.inext, d.jprev, d.jnext, d.kprev, d.knext};
    const int bc[6] = {d.bc_west, d.bc_east, d.bc_south, d.bc_north, d.bc_bottom, d.bc_top};
    for (int f = 0; f < 6; ++f)
      if (nbr[f] < 0 && bc[f] != MF3D_BC_PERIODIC) B.nmask |= 1 << f;
    // coefficients: aw, ae (x), as, an (y), ab, at (z); Neumann faces zeroed
    B.coef = (int)coef.size();
    const double *ext[3] = {d.hx, d.hy, d.hz};
    const double hh[3] = {d.dx, d.dy, d.dz};
    const int nn[3] = {B.nx, B.ny, B.nz};
    const int nfine[3] = {d.nx, d.ny, d.nz};
    for (int a = 0; a < 3; ++a) {
      std::vector<double> w = level_widths(ext[a], nfine[a], hh[a], ngrid, g);
      const int n = nn[a];
      const double hl = hh[a] * (double)(1 << (g - 1));
      const double dd = hl * hl;
      for (int side = 0; side < 2; ++side) {
        for (int c = 0; c < n + 2; ++c) {
          double v = 0.0;
          if (c >= 1 && c <= n) {
            if (!ext[a]) v = 1.0 / dd;  // mgsolver.for:184-189
            else v = 1.0 / (w[c] * (0.5 * (w[c] + w[side ? c + 1 : c - 1])));
            const int f = 2 * a + side;
            if ((B.nmask >> f & 1) && c == (side ? n : 1)) v = 0.0;  // mgsolver.for:192-203
          }
          coef.push_back((T)v);
        }
      }
    }
    // restriction ratios hf/Hc of this (fine) level, exactly 0.5 on uniform axes
    B.geo = (int)geo.size();
    for (int a = 0; a < 3; ++a) {
      const int n = nn[a];
      if (g < ngrid) {
        std::vector<double> wf = level_widths(ext[a], nfine[a], hh[a], ngrid, g);
        std::vector<double> wc = level_widths(ext[a], nfine[a], hh[a], ngrid, g + 1);
        for (int c = 0; c < n + 2; ++c) geo.push_back((T)((c >= 1 && c <= n) ? wf[c] / wc[(c + 1) >> 1] : 0.0));
      } else {
        for (int c = 0; c < n + 2; ++c) geo.push_back((T)0);
      }
    }
    it_sweep.push_back((long long)B.nz * B.ny * B.hp);
    it_cells.push_back((long long)(B.nx + 2) * (B.ny + 2) * (B.nz + 2));
    geom[b] = LevelGeom{B.nx, B.ny, B.nz};
    base[b] = cell_base;
    cell_base += geom[b].cells();
    L.ngg = std::max(L.ngg, std::max(B.nx, std::max(B.ny, B.nz)) + 2);
  }
  cudaStream_t s = C->stream;
  int st;
  if ((st = L.phi.alloc(phi_off))) return st;
  if ((st = L.rhs.alloc(phi_off))) return st;
  CK(cudaMemsetAsync(L.phi.p, 0, phi_off * sizeof(T), s));
  CK(cudaMemsetAsync(L.rhs.p, 0, phi_off * sizeof(T), s));
  if ((st = L.coef.upload(coef, s))) return st;
  if ((st = L.geo.upload(geo, s))) return st;
  if ((st = L.db.upload(L.hb, s))) return st;
  auto ts = make_tiles(it_sweep), tc = make_tiles(it_cells);
  L.n_sweep = (int)ts.size();
  L.n_cells = (int)tc.size();
  if ((st = L.t_sweep.upload(ts, s))) return st;
  if ((st = L.t_cells.upload(tc, s))) return st;
  // halo copy map -> element addresses in the colour-split pool
  std::vector<HaloPair> pairs = build_halo_map(C->blocks, geom, base);
  std::unordered_set<long long> dsts;
  for (auto &pr : pairs) dsts.insert(pr.dst);
  auto addr = [&](long long id) -> long long {
    int b = (int)(std::upper_bound(base.begin(), base.end(), id) - base.begin()) - 1;
    long long lin = id - base[b];
    const LevelGeom &G = geom[b];
    int i = (int)(lin % (G.nx + 2));
    long long r = lin / (G.nx + 2);
    int j = (int)(r % (G.ny + 2));
    int k = (int)(r / (G.ny + 2));
    const BlkLev &B = L.hb[b];
    int c = (i + j + k + 1) & 1;
    return B.phi0 + c * B.cstr + ((long long)k * (B.ny + 2) + j) * B.hp + (i >> 1);
  };
  std::vector<long long> hd, hs;
  for (int pass = 0; pass < 2; ++pass)
    for (auto &pr : pairs) {
      bool staged = dsts.count(pr.src) > 0;
      if ((pass == 0) != staged) continue;
      hd.push_back(addr(pr.dst));
      hs.push_back(addr(pr.src));
    }
  L.nstaged = 0;
  for (auto &pr : pairs) L.nstaged += dsts.count(pr.src) > 0;
  L.nhalo = (int)hd.size();
  if ((st = L.hdst.upload(hd, s))) return st;
  if ((st = L.hsrc.upload(hs, s))) return st;
  if ((st = L.hbuf.alloc(std::max(L.nstaged, 1)))) return st;
  if (C->prm.mg_itrsch == 2) {
    if ((st = L.tdma_work.alloc((size_t)nb * 128 * 2 * L.ngg))) return st;
  }
  return MF3D_OK;
}

// ---------------------------------------------------------------------------
// V-cycle building blocks.
// ---------------------------------------------------------------------------
template <typename T>
static void halo(mf3d_ctx *C, Level<T> &L) {
  if (L.nhalo == 0) return;
  if (L.nstaged) {
    k_halo_stage<T><<<grid_of(L.nstaged, 256), 256, 0, C->stream>>>(L.hsrc.p, L.nstaged, L.phi.p, L.hbuf.p);
    ++C->launches;
  }
  k_halo_apply<T><<<grid_of(L.nhalo, 256), 256, 0, C->stream>>>(L.hdst.p, L.hsrc.p, L.nhalo, L.nstaged, L.phi.p,
                                                                L.hbuf.p);
  ++C->launches;
}

// mgrelax(g, it) (mgsolver.for:371-617): `it` sweeps, each followed by
// mgbound + exchangepp (+ exchbc_mgpp), here one halo-map application.
template <typename T>
static void relax(mf3d_ctx *C, Level<T> &L, int it) {
  const int sch = C->prm.mg_itrsch;
  for (int itr = 0; itr < it; ++itr) {
    if (sch == 3) {
      const int pk = L.g == 1 ? MF3D_PROF_SMOOTH_L1 : 0;
      const double half = 0.5 * (double)C->n_l1 * sizeof(T);  // one colour of the finest level
      if (L.zero_interior) {
        prof_begin(C, pk, 2 * half);  // rhs in, colour out
        k_rbgs<T, true><<<L.n_sweep, kTile, 0, C->stream>>>(L.db.p, L.t_sweep.p, L.phi.p, L.rhs.p, L.coef.p, 0);
      } else {
        prof_begin(C, pk, 3 * half);  // other colour + rhs in, colour out
        k_rbgs<T, false><<<L.n_sweep, kTile, 0, C->stream>>>(L.db.p, L.t_sweep.p, L.phi.p, L.rhs.p, L.coef.p, 0);
      }
      prof_end(C, pk);
      prof_begin(C, pk, 3 * half);
      k_rbgs<T, false><<<L.n_sweep, kTile, 0, C->stream>>>(L.db.p, L.t_sweep.p, L.phi.p, L.rhs.p, L.coef.p, 1);
      prof_end(C, pk);
      C->launches += 2;
    } else if (sch == 1) {
      k_lexgs<T><<<C->nb, 1024, 0, C->stream>>>(L.db.p, L.phi.p, L.rhs.p, L.coef.p);
      ++C->launches;
    } else {
      k_tdma<T><<<C->nb, 128, 0, C->stream>>>(L.db.p, L.phi.p, L.rhs.p, L.coef.p, L.tdma_work.p, L.ngg);
      ++C->launches;
    }
    L.zero_interior = false;
    halo(C, L);
  }
}

// A level whose interior must read as zero but whose first use is not a
// red-black sweep gets real zeros.
template <typename T>
static void materialize_zero(mf3d_ctx *C, Level<T> &L) {
  if (L.zero_interior) {
    cudaMemsetAsync(L.phi.p, 0, L.phi.n * sizeof(T), C->stream);
    L.zero_interior = false;
  }
}

template <typename T>
static void restr(mf3d_ctx *C, Level<T> &F, Level<T> &Cl) {
  materialize_zero(C, F);
  const int pk = F.g == 1 ? MF3D_PROF_RESTRICT_L1 : 0;
  prof_begin(C, pk, (double)C->n_l1 * sizeof(T) * (2.0 + 2.0 / 8.0));  // fine phi, rhs in; coarse phi, rhs out
  k_restrict<T, T><<<Cl.n_cells, kTile, 0, C->stream>>>(F.db.p, Cl.db.p, Cl.t_cells.p, F.phi.p, F.rhs.p, F.coef.p,
                                                       Cl.phi.p, Cl.rhs.p, F.geo.p);
  prof_end(C, pk);
  ++C->launches;
  Cl.zero_interior = (C->prm.mg_itrsch == 3);  // k_restrict wrote real zeros too
  if (C->prm.mg_itrsch != 3) Cl.zero_interior = false;
}

template <typename T>
static void corr(mf3d_ctx *C, Level<T> &F, Level<T> &Cl) {
  materialize_zero(C, F);
  materialize_zero(C, Cl);
  const int pk = F.g == 1 ? MF3D_PROF_PROLONG_L1 : 0;
  prof_begin(C, pk, (double)C->n_l1 * sizeof(T) * (2.0 + 1.0 / 8.0));  // fine phi in/out, coarse phi in
  k_prolong<T, T><<<F.n_cells, kTile, 0, C->stream>>>(F.db.p, Cl.db.p, F.t_cells.p, F.phi.p, Cl.phi.p);
  prof_end(C, pk);
  ++C->launches;
}

// mgkcyc (mgsolver.for:224-369) with kcycle = 1: a V-cycle, irestr
// pre-sweeps and iproln post-sweeps, irestr + iproln sweeps on the coarsest
// level.  The level-1 rhs must hold su; level-1 phi starts at zero.
template <typename T>
static void vcycle(mf3d_ctx *C, std::vector<std::unique_ptr<Level<T>>> &Lv) {
  const int ngrd = C->prm.ngrid;
  Level<T> &L1 = *Lv[1];
  // pp = 0 including ghosts (newsolv_mg.for:19-21, 44)
  if (C->prm.mg_itrsch == 3) {
    k_zero_ghosts<T><<<L1.n_cells, kTile, 0, C->stream>>>(L1.db.p, L1.t_cells.p, L1.phi.p);
    ++C->launches;
    L1.zero_interior = true;
  } else {
    cudaMemsetAsync(L1.phi.p, 0, L1.phi.n * sizeof(T), C->stream);
    L1.zero_interior = false;
  }
  int glevel = 1, nrel;
  const int kcycle = 1;
  std::vector<int> kount(ngrd + 1, 0);
  relax(C, *Lv[1], C->prm.irestr);
  if (ngrd != 1) {
    restr(C, *Lv[1], *Lv[2]);
    glevel = 2;
    nrel = C->prm.irestr;
    for (;;) {
      if (glevel == 1) break;
      kount[glevel] += 1;
      relax(C, *Lv[glevel], nrel);
      if (kount[glevel] == kcycle + 1) {
        corr(C, *Lv[glevel - 1], *Lv[glevel]);
        kount[glevel] = 0;
        glevel -= 1;
        nrel = C->prm.iproln;
      } else if (glevel < ngrd) {
        restr(C, *Lv[glevel], *Lv[glevel + 1]);
        glevel += 1;
        nrel = C->prm.irestr;
      } else {
        relax(C, *Lv[glevel], C->prm.iproln);
        corr(C, *Lv[glevel - 1], *Lv[glevel]);
        nrel = C->prm.iproln;
        glevel = ngrd - 1;
      }
    }
  }
  relax(C, *Lv[1], C->prm.iproln);
  materialize_zero(C, L1);
}

template <typename T>
static T *level1_phi(mf3d_ctx *C);
template <>
double *level1_phi<double>(mf3d_ctx *C) { return C->L64[1]->phi.p; }
template <>
float *level1_phi<float>(mf3d_ctx *C) { return C->L32[1]->phi.p; }
template <typename T>
static T *level1_rhs(mf3d_ctx *C);
template <>
double *level1_rhs<double>(mf3d_ctx *C) { return C->L64[1]->rhs.p; }
template <>
float *level1_rhs<float>(mf3d_ctx *C) { return C->L32[1]->rhs.p; }
template <typename T>
static std::vector<std::unique_ptr<Level<T>>> &levels(mf3d_ctx *C);
template <>
std::vector<std::unique_ptr<Level<double>>> &levels<double>(mf3d_ctx *C) { return C->L64; }
template <>
std::vector<std::unique_ptr<Level<float>>> &levels<float>(mf3d_ctx *C) { return C->L32; }

// ---------------------------------------------------------------------------
// Fields: bind per-block pointers and upload the BlkFld table.
// ---------------------------------------------------------------------------
static int bind_fields(mf3d_ctx *C, const mf3d_fields *f) {
  for (int b = 0; b < C->nb; ++b) {
    BlkFld &F = C->hf[b];
    F.ustar = f[b].ustar; F.vstar = f[b].vstar; F.wstar = f[b].wstar;
    F.u = f[b].u; F.v = f[b].v; F.w = f[b].w; F.p = f[b].p; F.su = f[b].su;
    if (!F.ustar || !F.vstar || !F.wstar || !F.u || !F.v || !F.w || !F.p) {
      set_error("mf3d_fields: a required pointer is NULL");
      return MF3D_E_INVALID;
    }
  }
  CK(cudaMemcpyAsync(C->df.p, C->hf.data(), C->hf.size() * sizeof(BlkFld), cudaMemcpyHostToDevice, C->stream));
  return MF3D_OK;
}

// One outer iteration of newsolv_mg (newsolv_mg.for:25-58): V-cycle,
// p += pp, p halo + pbound, calvel + calmas, iteration bookkeeping.
template <typename T>
static void iteration_body(mf3d_ctx *C, bool in_graph) {
  cudaStream_t s = C->stream;
  vcycle<T>(C, levels<T>(C));
  k_add_correction<T><<<C->n_l1cells, kTile, 0, s>>>(C->df.p, C->t_l1cells.p, level1_phi<T>(C));
  k_p_faces<<<C->n_faces, kTile, 0, s>>>(C->df.p, C->t_faces.p);
  prof_begin(C, MF3D_PROF_CALMAS, (double)C->n_l1 * (4 * sizeof(double) + sizeof(T)));  // p, u*, v*, w* in; su out
  k_calvel_calmas<T><<<C->n_int, kTile, 0, s>>>(C->df.p, C->t_int.p, C->st.p, level1_rhs<T>(C), C->rmax_cur.p, 0);
  prof_end(C, MF3D_PROF_CALMAS);
  k_iter_end<<<1, 1, 0, s>>>(C->st.p, C->rmax_cur.p, C->hist_d.p, C->cond, in_graph ? 1 : 0);
  C->launches += 4;
}

// The whole outer loop as one graph: a conditional WHILE node whose body is
// one iteration; k_iter_end clears the condition when the loop must stop.
template <typename T>
static int build_solve_graph(mf3d_ctx *C) {
  if (C->graph_exec) return MF3D_OK;
  cudaGraph_t g;
  CK(cudaGraphCreate(&g, 0));
  C->graph = g;
  CK(cudaGraphConditionalHandleCreate(&C->cond, g, 1u, cudaGraphCondAssignDefault));
  cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
  np.conditional.handle = C->cond;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, g, nullptr, 0, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  CK(cudaStreamBeginCaptureToGraph(C->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  const long long before = C->launches;
  const int saved_prof = C->prof_kind;
  C->prof_kind = 0;  // no event records inside the graph
  iteration_body<T>(C, true);
  C->prof_kind = saved_prof;
  C->launches_per_iter = C->launches - before;
  cudaGraph_t captured;
  CK(cudaStreamEndCapture(C->stream, &captured));
  CK(cudaGraphInstantiate(&C->graph_exec, g, 0));
  return MF3D_OK;
}

template <typename T>
static int solve_device(mf3d_ctx *C, double dt, double alfapr, mf3d_solve_info *info, double *hist, int cap) {
  cudaStream_t s = C->stream;
  C->launches = 0;
  const int maxcy = std::max(C->prm.maxcy, 0);
  SolveState hs;
  std::memset(&hs, 0, sizeof hs);
  hs.dt = dt; hs.alfapr = alfapr; hs.eps = 0.0; hs.maxcy = maxcy;
  CK(cudaMemcpyAsync(C->st.p, &hs, sizeof hs, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(C->rmax_cur.p, 0, sizeof(unsigned long long), s));
  CK(cudaEventRecord(C->ev0, s));
  k_face_planes<<<C->n_planes, kTile, 0, s>>>(C->df.p, C->t_planes.p);
  // calvel; calmas (newsolv_mg.for:16-17): p's ghosts are used as given
  k_calvel_calmas<T><<<C->n_int, kTile, 0, s>>>(C->df.p, C->t_int.p, C->st.p, level1_rhs<T>(C), C->rmax_cur.p, 0);
  C->launches += 2;
  CK(cudaMemcpyAsync(C->rmax_host, C->rmax_cur.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  CK(cudaMemsetAsync(C->rmax_cur.p, 0, sizeof(unsigned long long), s));
  CK(cudaStreamSynchronize(s));
  double rmax0;
  std::memcpy(&rmax0, C->rmax_host, sizeof(double));
  hs.eps = C->prm.eps_relative ? C->prm.eps * rmax0 : C->prm.eps;
  CK(cudaMemcpyAsync(&C->st.p->eps, &hs.eps, sizeof(double), cudaMemcpyHostToDevice, s));
  const bool nonfinite0 = !std::isfinite(rmax0);
  if (maxcy > 0 && !nonfinite0) {
    if (C->use_graph && C->prof_kind == 0) {
      int st = build_solve_graph<T>(C);
      if (st) return st;
      CK(cudaGraphLaunch(C->graph_exec, s));
    } else {
      for (int it = 1; it <= maxcy; ++it) {
        iteration_body<T>(C, false);
        CK(cudaMemcpyAsync(&hs, C->st.p, sizeof hs, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        prof_collect(C);
        if (hs.done) break;
      }
    }
  }
  // final su (optional) and u, v, w (calvel with the final p)
  bool want_su = false;
  for (auto &F : C->hf) want_su |= F.su != nullptr;
  if (want_su) {
    k_calvel_calmas<T><<<C->n_int, kTile, 0, s>>>(C->df.p, C->t_int.p, C->st.p, level1_rhs<T>(C), C->rmax_scratch.p, 1);
    ++C->launches;
  }
  k_calvel<<<C->n_int, kTile, 0, s>>>(C->df.p, C->t_int.p, C->st.p);
  ++C->launches;
  CK(cudaEventRecord(C->ev1, s));
  CK(cudaMemcpyAsync(&hs, C->st.p, sizeof hs, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  prof_collect(C);
  const int iters = hs.iter;
  if (C->use_graph && C->prof_kind == 0) C->launches += (long long)iters * C->launches_per_iter;
  if (hist && iters > 0) {
    CK(cudaMemcpy(hist, C->hist_d.p, std::min(iters, cap) * sizeof(double), cudaMemcpyDeviceToHost));
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, C->ev0, C->ev1);
  const double rmax = iters > 0 ? hs.rmax : rmax0;
  int status = MF3D_OK;
  if (nonfinite0 || hs.done == 2) status = MF3D_E_NONFINITE;
  else if (hs.done != 1) status = MF3D_NOT_CONVERGED;
  if (status >= 0 && rmax > 100.0) status = MF3D_DIVERGED;  // newsolv_mg.for:64
  if (info) {
    info->rmax = rmax; info->rmax0 = rmax0; info->iter = iters; info->status = status; info->ms_device = ms;
  }
  if (status == MF3D_E_NONFINITE) set_error("non-finite rmax");
  return status;
}

template <typename T>
static int mgkcyc_device(mf3d_ctx *C, double *const *su, double *const *pp) {
  cudaStream_t s = C->stream;
  C->launches = 0;
  CK(cudaMemcpyAsync(C->ptrs.p, su, C->nb * sizeof(double *), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(C->ptrs.p + C->nb, pp, C->nb * sizeof(double *), cudaMemcpyHostToDevice, s));
  k_load_rhs<T><<<C->n_int, kTile, 0, s>>>(C->df.p, C->t_int.p, C->ptrs.p, level1_rhs<T>(C));
  vcycle<T>(C, levels<T>(C));
  k_store_pp<T><<<C->n_l1cells, kTile, 0, s>>>(C->df.p, C->t_l1cells.p, C->ptrs.p + C->nb, level1_phi<T>(C));
  C->launches += 2;
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  return MF3D_OK;
}

static size_t ttc_elems(const mf3d_ctx *C, int b) {
  const auto &d = C->blocks[b];
  const int pl = C->prm.pl;
  return (size_t)(d.nx + 2 * pl) * (d.ny + 2 * pl) * (d.nz + 2 * pl);
}

static int create(const mf3d_block_desc *blocks, int nb, const mf3d_params *prm, mf3d_ctx **out) {
  if (!blocks || nb <= 0 || !prm || !out) { set_error("mf3d_create: bad arguments"); return MF3D_E_INVALID; }
  if (prm->ngrid < 1 || prm->ngrid > 16) { set_error("ngrid out of range"); return MF3D_E_INVALID; }
  if (prm->mg_itrsch < 1 || prm->mg_itrsch > 3) { set_error("error about mg iteration selection (mg_itrsch)"); return MF3D_E_INVALID; }
  if (prm->irestr < 0 || prm->iproln < 0 || prm->maxcy < 0) { set_error("negative sweep/cycle count"); return MF3D_E_INVALID; }
  if (prm->pl < 1) { set_error("pl must be >= 1"); return MF3D_E_INVALID; }
  if (prm->differencing != 1) { set_error("differencing != 1 (4th-order calmas) is not supported"); return MF3D_E_UNSUPPORTED; }
  if (prm->precision < 0 || prm->precision > 1) { set_error("precision mode not supported"); return MF3D_E_UNSUPPORTED; }
  const int pow2 = 1 << (prm->ngrid - 1);
  for (int b = 0; b < nb; ++b) {
    const auto &d = blocks[b];
    if (d.nx < 1 || d.ny < 1 || d.nz < 1 || d.nx % pow2 || d.ny % pow2 || d.nz % pow2) {  // localparameters.for:201-206
      set_error("2:the given number not correct for mgsolver! (block " + std::to_string(d.id) +
                " not divisible by 2^(ngrid-1))");
      return MF3D_E_INVALID;
    }
  }
  auto C = std::make_unique<mf3d_ctx>();
  C->prm = *prm;
  C->blocks.assign(blocks, blocks + nb);
  C->nb = nb;
  C->device = prm->device;
  // widths arrays are borrowed at create time only
  int st = face_rules(C->blocks, C->rules);
  if (st) return st;
  CK(cudaSetDevice(C->device));
  // A blocking stream: it orders after work the caller queued on the legacy
  // default stream (e.g. the copies that produced the device inputs).
  CK(cudaStreamCreateWithFlags(&C->stream, cudaStreamDefault));
  CK(cudaEventCreate(&C->ev0));
  CK(cudaEventCreate(&C->ev1));
  CK(cudaMallocHost(&C->rmax_host, sizeof(unsigned long long) * 2));
  if ((st = C->rmax_cur.alloc(1))) return st;
  if ((st = C->rmax_scratch.alloc(1))) return st;
  if ((st = C->st.alloc(1))) return st;
  if ((st = C->hist_d.alloc(std::max(prm->maxcy, 0) + 1))) return st;
  {
    const char *e = getenv("MF3D_NO_GRAPH");
    C->use_graph = !(e && e[0] == '1');
  }
  if ((st = C->ptrs.alloc(2 * nb))) return st;
  const int ngrid = prm->ngrid;
  if (prm->precision == MF3D_PREC_FP64) {
    C->L64.resize(ngrid + 1);
    for (int g = 1; g <= ngrid; ++g) {
      C->L64[g].reset(new Level<double>());
      if ((st = build_level<double>(C.get(), *C->L64[g], g))) return st;
    }
  } else {
    C->L32.resize(ngrid + 1);
    for (int g = 1; g <= ngrid; ++g) {
      C->L32[g].reset(new Level<float>());
      if ((st = build_level<float>(C.get(), *C->L32[g], g))) return st;
    }
  }
  // field geometry: widths, face distances, face planes
  std::vector<double> geo;
  std::vector<size_t> off_h(3 * nb), off_df(3 * nb);
  size_t plane_total = 0;
  std::vector<size_t> plane_off(nb);
  for (int b = 0; b < nb; ++b) {
    const auto &d = C->blocks[b];
    const double *ext[3] = {d.hx, d.hy, d.hz};
    const double hh[3] = {d.dx, d.dy, d.dz};
    const int n[3] = {d.nx, d.ny, d.nz};
    for (int a = 0; a < 3; ++a) {
      std::vector<double> w = level_widths(ext[a], n[a], hh[a], ngrid, 1);
      off_h[3 * b + a] = geo.size();
      for (int c = 0; c < n[a] + 2; ++c) geo.push_back(ext[a] ? w[c] : hh[a]);
      off_df[3 * b + a] = geo.size();
      for (int c = 0; c <= n[a]; ++c) geo.push_back(ext[a] ? 0.5 * (w[c] + w[c + 1]) : hh[a]);
    }
    plane_off[b] = plane_total;
    plane_total += 2 * ((size_t)d.ny * d.nz + (size_t)d.nx * d.nz + (size_t)d.nx * d.ny);
  }
  if ((st = C->widths.upload(geo, C->stream))) return st;
  if ((st = C->planes.alloc(plane_total))) return st;
  CK(cudaMemsetAsync(C->planes.p, 0, plane_total * sizeof(double), C->stream));
  C->hf.resize(nb);
  std::vector<long long> it_int, it_l1, it_faces, it_planes;
  for (int b = 0; b < nb; ++b) {
    const auto &d = C->blocks[b];
    BlkFld &F = C->hf[b];
    std::memset(&F, 0, sizeof F);
    F.nx = d.nx; F.ny = d.ny; F.nz = d.nz; F.pl = prm->pl;
    F.ti = d.nx + 2 * prm->pl; F.tj = d.ny + 2 * prm->pl;
    for (int f = 0; f < 6; ++f) {
      F.wall[f] = C->rules[6 * b + f].kind == FACE_WALL;
      F.src[f] = C->rules[6 * b + f].src;
    }
    for (int a = 0; a < 3; ++a) {
      F.h[a] = C->widths.p + off_h[3 * b + a];
      F.df[a] = C->widths.p + off_df[3 * b + a];
    }
    double *pp = C->planes.p + plane_off[b];
    const size_t pyz = (size_t)d.ny * d.nz, pxz = (size_t)d.nx * d.nz, pxy = (size_t)d.nx * d.ny;
    F.lo[0] = pp; F.hi[0] = pp + pyz; pp += 2 * pyz;
    F.lo[1] = pp; F.hi[1] = pp + pxz; pp += 2 * pxz;
    F.lo[2] = pp; F.hi[2] = pp + pxy;
    F.L1 = prm->precision == MF3D_PREC_FP64 ? C->L64[1]->hb[b] : C->L32[1]->hb[b];
    it_int.push_back((long long)d.nx * d.ny * d.nz);
    C->n_l1 += (long long)d.nx * d.ny * d.nz;
    it_l1.push_back((long long)(d.nx + 2) * (d.ny + 2) * (d.nz + 2));
    it_faces.push_back(2 * ((long long)d.ny * d.nz + (long long)d.nx * d.nz + (long long)d.nx * d.ny));
    it_planes.push_back((long long)d.ny * d.nz + (long long)d.nx * d.nz + (long long)d.nx * d.ny);
  }
  if ((st = C->df.alloc(nb))) return st;
  auto t1 = make_tiles(it_int), t2 = make_tiles(it_l1), t3 = make_tiles(it_faces), t4 = make_tiles(it_planes);
  C->n_int = (int)t1.size(); C->n_l1cells = (int)t2.size(); C->n_faces = (int)t3.size(); C->n_planes = (int)t4.size();
  if ((st = C->t_int.upload(t1, C->stream))) return st;
  if ((st = C->t_l1cells.upload(t2, C->stream))) return st;
  if ((st = C->t_faces.upload(t3, C->stream))) return st;
  if ((st = C->t_planes.upload(t4, C->stream))) return st;
  CK(cudaStreamSynchronize(C->stream));
  // host-field mirrors are allocated lazily by the host entry point
  for (auto &d : C->blocks) d.hx = d.hy = d.hz = nullptr;
  *out = C.release();
  return MF3D_OK;
}

static int run_solve(mf3d_ctx *C, double dt, double alfapr, mf3d_solve_info *info, double *hist, int cap) {
  if (C->prm.precision == MF3D_PREC_FP64) return solve_device<double>(C, dt, alfapr, info, hist, cap);
  return solve_device<float>(C, dt, alfapr, info, hist, cap);
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

int mf3d_destroy(mf3d_ctx *ctx) {
  if (!ctx) return MF3D_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->rmax_host) cudaFreeHost(ctx->rmax_host);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  for (auto e : ctx->prof_ev) cudaEventDestroy(e);
  if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  cudaStream_t s = ctx->stream;
  delete ctx;
  if (s) cudaStreamDestroy(s);
  return MF3D_OK;
}

int mf3d_newsolv_mg_device(mf3d_ctx *C, const mf3d_fields *fields, double dt, double alfapr, mf3d_solve_info *info,
                           double *hist, int cap) {
  if (!C || !fields) { mf3d::set_error("mf3d_newsolv_mg_device: bad arguments"); return MF3D_E_INVALID; }
  if (cudaSetDevice(C->device) != cudaSuccess) { mf3d::set_error("cudaSetDevice failed"); return MF3D_E_CUDA; }
  int st = mf3d::bind_fields(C, fields);
  if (st) return st;
  return mf3d::run_solve(C, dt, alfapr, info, hist, cap);
}

int mf3d_newsolv_mg(mf3d_ctx *C, const mf3d_fields *fields, double dt, double alfapr, mf3d_solve_info *info,
                    double *hist, int cap) {
  if (!C || !fields) { mf3d::set_error("mf3d_newsolv_mg: bad arguments"); return MF3D_E_INVALID; }
  if (cudaSetDevice(C->device) != cudaSuccess) { mf3d::set_error("cudaSetDevice failed"); return MF3D_E_CUDA; }
  cudaStream_t s = C->stream;
  // device mirrors: 8 arrays per block (ustar, vstar, wstar, u, v, w, p, su)
  if (!C->mirror.p) {
    size_t tot = 0;
    C->mirror_off.resize(C->nb);
    for (int b = 0; b < C->nb; ++b) { C->mirror_off[b] = tot; tot += 8 * mf3d::ttc_elems(C, b); }
    int st = C->mirror.alloc(tot);
    if (st) return st;
  }
  std::vector<mf3d_fields> dev(C->nb);
  for (int b = 0; b < C->nb; ++b) {
    const size_t n = mf3d::ttc_elems(C, b);
    double *m = C->mirror.p + C->mirror_off[b];
    double *const hsrc[7] = {fields[b].ustar, fields[b].vstar, fields[b].wstar, fields[b].u, fields[b].v, fields[b].w, fields[b].p};
    for (int q = 0; q < 7; ++q) {
      if (!hsrc[q]) { mf3d::set_error("mf3d_fields: a required pointer is NULL"); return MF3D_E_INVALID; }
      if (cudaMemcpyAsync(m + q * n, hsrc[q], n * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess) {
        mf3d::set_error("host-to-device copy failed"); return MF3D_E_CUDA;
      }
    }
    dev[b] = mf3d_fields{m, m + n, m + 2 * n, m + 3 * n, m + 4 * n, m + 5 * n, m + 6 * n,
                         fields[b].su ? m + 7 * n : nullptr};
  }
  int st = mf3d::bind_fields(C, dev.data());
  if (st) return st;
  st = mf3d::run_solve(C, dt, alfapr, info, hist, cap);
  if (st < 0 && st != MF3D_E_NONFINITE) return st;
  for (int b = 0; b < C->nb; ++b) {
    const size_t n = mf3d::ttc_elems(C, b);
    double *m = C->mirror.p + C->mirror_off[b];
    double *const hdst[5] = {fields[b].u, fields[b].v, fields[b].w, fields[b].p, fields[b].su};
    const int q_of[5] = {3, 4, 5, 6, 7};
    for (int q = 0; q < 5; ++q) {
      if (!hdst[q]) continue;
      if (cudaMemcpyAsync(hdst[q], m + q_of[q] * n, n * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess) {
        mf3d::set_error("device-to-host copy failed"); return MF3D_E_CUDA;
      }
    }
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) { mf3d::set_error("stream sync failed"); return MF3D_E_CUDA; }
  return st;
}

int mf3d_mgkcyc_device(mf3d_ctx *C, double *const *su, double *const *pp) {
  if (!C || !su || !pp) { mf3d::set_error("mf3d_mgkcyc_device: bad arguments"); return MF3D_E_INVALID; }
  if (cudaSetDevice(C->device) != cudaSuccess) { mf3d::set_error("cudaSetDevice failed"); return MF3D_E_CUDA; }
  // the V-cycle needs the block geometry of the field table, not the fields
  cudaMemcpyAsync(C->df.p, C->hf.data(), C->hf.size() * sizeof(mf3d::BlkFld), cudaMemcpyHostToDevice, C->stream);
  if (C->prm.precision == MF3D_PREC_FP64) return mf3d::mgkcyc_device<double>(C, su, pp);
  return mf3d::mgkcyc_device<float>(C, su, pp);
}

long long mf3d_last_launch_count(const mf3d_ctx *C) { return C ? C->launches : 0; }

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

}  // extern "C"
