// solver = 1: pressure_1sweep (press.for:274-420) with Stone's strongly
// implicit procedure, sipsol(44) (sipsol.for:2-206), on the device.
//
// The ILU factorisation and the two substitutions are recurrences over the
// previous cell along j, i and k (the reference's ijk-1, ijk-nj, ijk-nij).
// A cell depends only on cells of a smaller i+j+k, so every cell of one
// hyperplane i+j+k = h can be formed at once with exactly the reference's
// operands and operation order: one launch per hyperplane and block set,
// the whole sweep captured once in a CUDA graph.  The factors and the
// residual live in per-block arrays over the ghost-inclusive box, i fastest,
// zero outside the interior (the reference zeroes its arrays and only ever
// writes interior cells).  The correction pp is the level-1 phi of the
// multigrid storage, so the pressure update, the halo refresh of pp
// (exchange(44): its face values are the multigrid halo's) and
// calvel/calmas are the multigrid path's own kernels.
//
// The summed |residual| of a sweep, which only steers the stopping test, is
// reduced in a fixed order (deterministic, but not the reference's serial
// order: the test can differ only when a ratio lies within rounding of
// 0.001 or 1e-5).
#pragma once

namespace mf3d {

constexpr double kSipAlfa = 0.92;  // sipsol.for:31
constexpr double kSipSmall = 1e-20;

struct SipBlk {
  double *lb, *lw, *ls, *lpr, *un, *ue, *ut, *res;  // (nx+2)(ny+2)(nz+2) each, i fastest
  int nx, ny, nz;
};
__device__ __forceinline__ long long sip_idx(const SipBlk &S, int i, int j, int k) {
  return ((long long)k * (S.ny + 2) + j) * (S.nx + 2) + i;
}

// One hyperplane i+j+k = h of the ILU factors (sipsol.for:79-101).
// Thread per (i, j) of every block.
__global__ void k_sip_factor(const SipBlk *__restrict__ sb, const BlkLev *__restrict__ bl,
                             const Tile *__restrict__ tiles, int h) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const SipBlk S = sb[t.blk];
  const int q = t.i0 + threadIdx.x;
  if (q >= S.nx * S.ny) return;
  const int i = q % S.nx + 1, j = q / S.nx + 1, k = h - i - j;
  if (k < 1 || k > S.nz) return;
  const BlkLev &B = bl[t.blk];
  const Coef<double> cf(B);
  const double aw = cf.aw[i], ae = cf.ae[i], as = cf.as[j], an = cf.an[j], ab = cf.ab[k], at = cf.at[k];
  const double ap = -1.0 * (aw + ae + as + an + ab + at);
  const long long c = sip_idx(S, i, j, k), cb = sip_idx(S, i, j, k - 1), cw = sip_idx(S, i - 1, j, k),
                  cs = sip_idx(S, i, j - 1, k);
  const double lb = ab / (1. + kSipAlfa * (S.un[cb] + S.ue[cb]));
  const double lw = aw / (1. + kSipAlfa * (S.un[cw] + S.ut[cw]));
  const double ls = as / (1. + kSipAlfa * (S.ue[cs] + S.ut[cs]));
  const double p1 = kSipAlfa * (lb * S.un[cb] + lw * S.un[cw]);
  const double p2 = kSipAlfa * (lb * S.ue[cb] + ls * S.ue[cs]);
  const double p3 = kSipAlfa * (lw * S.ut[cw] + ls * S.ut[cs]);
  const double lpr = 1. / (ap + p1 + p2 + p3 - lb * S.ut[cb] - lw * S.ue[cw] - ls * S.un[cs] + kSipSmall);
  S.lb[c] = lb; S.lw[c] = lw; S.ls[c] = ls; S.lpr[c] = lpr;
  S.un[c] = (an - p1) * lpr;
  S.ue[c] = (ae - p2) * lpr;
  S.ut[c] = (at - p3) * lpr;
}

// The residual of pp (sipsol.for:137-147) over every interior cell, and
// each CTA's sum of |res| (a fixed tree) into part[blockIdx.x].
__global__ void __launch_bounds__(RW_TX *RW_RJ) k_sip_residual(const SipBlk *__restrict__ sb,
                                                               const BlkLev *__restrict__ bl,
                                                               const Tile *__restrict__ tiles,
                                                               double *__restrict__ part) {
  pdl_wait();
  __shared__ double red[RW_RJ];
  const Tile t = tiles[blockIdx.x];
  const SipBlk S = sb[t.blk];
  const BlkLev &B = bl[t.blk];
  const Coef<double> cf(B);
  const double *__restrict__ fi = phi_of<double>(B);
  const double *__restrict__ su = rhs_of<double>(B);
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  double acc = 0.0;
  if (i <= S.nx && j <= S.ny) {
    const int k1 = min(t.k0 + RW_KCH - 1, S.nz);
    for (int k = t.k0; k <= k1; ++k) {
      const double aw = cf.aw[i], ae = cf.ae[i], as = cf.as[j], an = cf.an[j], ab = cf.ab[k], at = cf.at[k];
      const double ap = -1.0 * (aw + ae + as + an + ab + at);
      const double r = (su[cell_off(B, i, j, k)] - ap * fi[cell_off(B, i, j, k)] - an * fi[cell_off(B, i, j + 1, k)] -
                        as * fi[cell_off(B, i, j - 1, k)] - ae * fi[cell_off(B, i + 1, j, k)] -
                        aw * fi[cell_off(B, i - 1, j, k)] - ab * fi[cell_off(B, i, j, k - 1)] -
                        at * fi[cell_off(B, i, j, k + 1)]);
      S.res[sip_idx(S, i, j, k)] = r;
      acc = acc + fabs(r);
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc = acc + __shfl_xor_sync(0xffffffffu, acc, o);
  if (threadIdx.x == 0) red[threadIdx.y] = acc;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    double v = 0.0;
    for (int r = 0; r < RW_RJ; ++r) v = v + red[r];
    part[blockIdx.x] = v;
  }
}

// The per-CTA sums added in index order by one CTA: a fixed tree.
__global__ void k_sip_sum(const double *__restrict__ part, int n, double *__restrict__ out) {
  pdl_wait();
  __shared__ double s[1024];
  double v = 0.0;
  for (int q = threadIdx.x; q < n; q += blockDim.x) v = v + part[q];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] = s[threadIdx.x] + s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = s[0];
}

// Forward substitution on hyperplane h (sipsol.for:149-157).
__global__ void k_sip_forward(const SipBlk *__restrict__ sb, const Tile *__restrict__ tiles, int h) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const SipBlk S = sb[t.blk];
  const int q = t.i0 + threadIdx.x;
  if (q >= S.nx * S.ny) return;
  const int i = q % S.nx + 1, j = q / S.nx + 1, k = h - i - j;
  if (k < 1 || k > S.nz) return;
  const long long c = sip_idx(S, i, j, k);
  S.res[c] = (S.res[c] - S.lb[c] * S.res[sip_idx(S, i, j, k - 1)] - S.lw[c] * S.res[sip_idx(S, i - 1, j, k)] -
              S.ls[c] * S.res[sip_idx(S, i, j - 1, k)]) *
             S.lpr[c];
}

// Backward substitution on hyperplane h and the correction of pp
// (sipsol.for:159-170).
__global__ void k_sip_backward(const SipBlk *__restrict__ sb, const BlkLev *__restrict__ bl,
                               const Tile *__restrict__ tiles, int h) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const SipBlk S = sb[t.blk];
  const int q = t.i0 + threadIdx.x;
  if (q >= S.nx * S.ny) return;
  const int i = q % S.nx + 1, j = q / S.nx + 1, k = h - i - j;
  if (k < 1 || k > S.nz) return;
  const long long c = sip_idx(S, i, j, k);
  const double r = S.res[c] - S.un[c] * S.res[sip_idx(S, i, j + 1, k)] - S.ue[c] * S.res[sip_idx(S, i + 1, j, k)] -
                   S.ut[c] * S.res[sip_idx(S, i, j, k + 1)];
  S.res[c] = r;
  double *fi = phi_of<double>(bl[t.blk]);
  const long long e = cell_off(bl[t.blk], i, j, k);
  fi[e] = fi[e] + r;
}

// Both substitutions of a block in one CTA: its hyperplanes one after
// another, a CTA barrier between them (a block's recurrences never reach
// into another block).  For small blocks, where a hyperplane holds a few
// thousand cells at most, this replaces 2*(nx+ny+nz-2) launches per sweep
// by one; the per-cell arithmetic is k_sip_forward's and k_sip_backward's.
__global__ void __launch_bounds__(1024) k_sip_subst_block(const SipBlk *__restrict__ sb,
                                                          const BlkLev *__restrict__ bl) {
  pdl_wait();
  const SipBlk S = sb[blockIdx.x];
  const BlkLev &B = bl[blockIdx.x];
  double *fi = phi_of<double>(B);
  const int hmax = S.nx + S.ny + S.nz, pairs = S.nx * S.ny;
  for (int h = 3; h <= hmax; ++h) {
    for (int q = threadIdx.x; q < pairs; q += blockDim.x) {
      const int i = q % S.nx + 1, j = q / S.nx + 1, k = h - i - j;
      if (k < 1 || k > S.nz) continue;
      const long long c = sip_idx(S, i, j, k);
      S.res[c] = (S.res[c] - S.lb[c] * S.res[sip_idx(S, i, j, k - 1)] - S.lw[c] * S.res[sip_idx(S, i - 1, j, k)] -
                  S.ls[c] * S.res[sip_idx(S, i, j - 1, k)]) *
                 S.lpr[c];
    }
    __syncthreads();
  }
  for (int h = hmax; h >= 3; --h) {
    for (int q = threadIdx.x; q < pairs; q += blockDim.x) {
      const int i = q % S.nx + 1, j = q / S.nx + 1, k = h - i - j;
      if (k < 1 || k > S.nz) continue;
      const long long c = sip_idx(S, i, j, k);
      const double r = S.res[c] - S.un[c] * S.res[sip_idx(S, i, j + 1, k)] -
                       S.ue[c] * S.res[sip_idx(S, i + 1, j, k)] - S.ut[c] * S.res[sip_idx(S, i, j, k + 1)];
      S.res[c] = r;
      const long long e = cell_off(B, i, j, k);
      fi[e] = fi[e] + r;
    }
    __syncthreads();
  }
}

// Blocks whose (i, j) plane holds at most this many cells take the one-CTA
// substitution kernel; larger ones the hyperplane launches.
constexpr int kSipBlockCells = 4096;

// The same two substitutions with one thread per (i, j) column, for blocks
// of at most 1024 columns.  At hyperplane h column (i, j) holds cell
// k = h-i-j: the cell below is its own previous value (a register), and
// the cells west and south (forward) or east and north (backward) at the
// same k were formed by those columns one hyperplane earlier and wait in a
// shared-memory plane.  Each hyperplane is then two CTA barriers and no
// dependent global load; the operands of the next cell are loaded one step
// ahead.  The arithmetic is the reference's, operand for operand.
__global__ void __launch_bounds__(1024) k_sip_subst_col(const SipBlk *__restrict__ sb,
                                                        const BlkLev *__restrict__ bl) {
  pdl_wait();
  extern __shared__ double plane[];  // (ny+2) x (nx+2), zero border
  const SipBlk S = sb[blockIdx.x];
  const BlkLev &B = bl[blockIdx.x];
  double *fi = phi_of<double>(B);
  const int nx = S.nx, ny = S.ny, nz = S.nz, px = nx + 2;
  const int tid = threadIdx.x;
  for (int q = tid; q < (ny + 2) * px; q += blockDim.x) plane[q] = 0.0;
  const bool col = tid < nx * ny;
  const int i = tid % nx + 1, j = tid / nx + 1;
  const int hmax = nx + ny + nz;
  __syncthreads();
  // forward: res = (res - lb*res(k-1) - lw*res(i-1) - ls*res(j-1)) * lpr
  double below = 0.0;
  int kn = 3 - i - j;  // k at the next step
  double nres = 0.0, nlb = 0.0, nlw = 0.0, nls = 0.0, nlpr = 0.0;
  auto fetch_f = [&](int k) {
    if (col && k >= 1 && k <= nz) {
      const long long c = sip_idx(S, i, j, k);
      nres = S.res[c]; nlb = S.lb[c]; nlw = S.lw[c]; nls = S.ls[c]; nlpr = S.lpr[c];
    }
  };
  fetch_f(kn);
  for (int h = 3; h <= hmax; ++h) {
    const int k = h - i - j;
    const bool act = col && k >= 1 && k <= nz;
    double v = 0.0;
    if (act) {
      const double w = plane[j * px + i - 1], so = plane[(j - 1) * px + i];
      v = (nres - nlb * below - nlw * w - nls * so) * nlpr;
    }
    fetch_f(k + 1);
    __syncthreads();
    if (act) {
      plane[j * px + i] = v;
      S.res[sip_idx(S, i, j, k)] = v;
      below = v;
    }
    __syncthreads();
  }
  // backward: res = res - un*res(j+1) - ue*res(i+1) - ut*res(k+1); fi += res
  for (int q = tid; q < (ny + 2) * px; q += blockDim.x) plane[q] = 0.0;
  __syncthreads();
  double above = 0.0;
  double bres = 0.0, bun = 0.0, bue = 0.0, but = 0.0;
  auto fetch_b = [&](int k) {
    if (col && k >= 1 && k <= nz) {
      const long long c = sip_idx(S, i, j, k);
      bres = S.res[c]; bun = S.un[c]; bue = S.ue[c]; but = S.ut[c];
    }
  };
  fetch_b(hmax - i - j);
  for (int h = hmax; h >= 3; --h) {
    const int k = h - i - j;
    const bool act = col && k >= 1 && k <= nz;
    double r = 0.0;
    if (act) {
      const double no = plane[(j + 1) * px + i], ea = plane[j * px + i + 1];
      r = bres - bun * no - bue * ea - but * above;
    }
    fetch_b(k - 1);
    __syncthreads();
    if (act) {
      plane[j * px + i] = r;
      S.res[sip_idx(S, i, j, k)] = r;
      const long long e = cell_off(B, i, j, k);
      fi[e] = fi[e] + r;
      above = r;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
struct SipState {
  std::vector<DevBuf<double>> arrays;  // per block: 8 arrays
  DevBuf<SipBlk> sb;
  DevBuf<Tile> t_ij;                   // (i, j) pairs of every block
  int n_ij = 0, hmax = 0;
  DevBuf<double> part, resab;
  cudaGraphExec_t sweep = nullptr;     // forward + backward substitutions
  int subst_launches = 0;              // kernels in that graph
  ~SipState() {
    if (sweep) cudaGraphExecDestroy(sweep);
  }
};

static int sip_prepare(mf3d_ctx *C, View &V) {
  if (C->sip) return MF3D_OK;
  cudaStream_t s = C->stream;
  auto S = std::make_unique<SipState>();
  const int nb = (int)V.blk.size();
  std::vector<SipBlk> hb(nb);
  std::vector<long long> items;
  int st;
  S->arrays.resize((size_t)8 * nb);
  for (int b = 0; b < nb; ++b) {
    const mf3d_block_desc &d = V.blk[b]->d;
    const size_t n = (size_t)(d.nx + 2) * (d.ny + 2) * (d.nz + 2);
    double *p[8];
    for (int a = 0; a < 8; ++a) {
      DevBuf<double> &A = S->arrays[(size_t)8 * b + a];
      if ((st = A.alloc(n))) return st;
      CK(cudaMemsetAsync(A.p, 0, n * sizeof(double), s));
      p[a] = A.p;
    }
    hb[b] = SipBlk{p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], d.nx, d.ny, d.nz};
    items.push_back((long long)d.nx * d.ny);
    S->hmax = std::max(S->hmax, d.nx + d.ny + d.nz);
  }
  if ((st = S->sb.upload(hb, s))) return st;
  auto t = make_tiles(items);
  S->n_ij = (int)t.size();
  if ((st = S->t_ij.upload(t, s))) return st;
  if ((st = S->part.alloc(std::max(V.n_int, 1)))) return st;
  if ((st = S->resab.alloc(1))) return st;
  // the factors, hyperplane by hyperplane (the coefficients never change)
  const BlkLev *L1 = V.lv[1].tab.p;
  for (int h = 3; h <= S->hmax; ++h)
    launch(k_sip_factor, S->n_ij, kTile, 0, s, S->sb.p, L1, S->t_ij.p, h);
  // one graph per context for the two substitutions of a sweep: one CTA
  // per block when every block is small, else a launch per hyperplane
  int maxpairs = 0;
  for (const auto &b : hb) maxpairs = std::max(maxpairs, b.nx * b.ny);
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int maxplane = 0;
  for (const auto &b : hb) maxplane = std::max(maxplane, (b.nx + 2) * (b.ny + 2));
  if (maxpairs <= 1024 && maxplane * 8 <= 48 * 1024) {
    launch(k_sip_subst_col, nb, 1024, (size_t)maxplane * 8, s, S->sb.p, L1);
  } else if (maxpairs <= kSipBlockCells) {
    launch(k_sip_subst_block, nb, 1024, 0, s, S->sb.p, L1);
  } else {
    for (int h = 3; h <= S->hmax; ++h) launch(k_sip_forward, S->n_ij, kTile, 0, s, S->sb.p, S->t_ij.p, h);
    for (int h = S->hmax; h >= 3; --h) launch(k_sip_backward, S->n_ij, kTile, 0, s, S->sb.p, L1, S->t_ij.p, h);
  }
  CK(cudaStreamEndCapture(s, &g));
  const cudaError_t e = cudaGraphInstantiate(&S->sweep, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { set_error(std::string("SIP graph: ") + cudaGetErrorString(e)); return MF3D_E_CUDA; }
  CK(cudaStreamSynchronize(s));
  S->subst_launches = maxpairs <= kSipBlockCells ? 1 : 2 * (S->hmax - 2);
  C->launches += S->hmax - 2;
  C->sip = std::move(S);
  return MF3D_OK;
}

// sipsol(44): pp := 0, then up to nswp sweeps; returns the sweeps run.
static int sip_solve(mf3d_ctx *C, View &V, int *sweeps) {
  cudaStream_t s = C->stream;
  SipState &S = *C->sip;
  const ViewLevel &L1 = V.lv[1];
  for (size_t b = 0; b < V.blk.size(); ++b) {
    const BlkLev &B = V.blk[b]->lv[1].desc;
    CK(cudaMemsetAsync(B.phi, 0, (size_t)2 * B.cstr * sizeof(double), s));
  }
  double relast = 0.0, res1 = 0.0;
  int n = 0;
  for (int sweep = 1; sweep <= C->prm.nswp; ++sweep) {
    launch(k_sip_residual, V.n_int, dim3(RW_TX, RW_RJ), 0, s, S.sb.p, L1.tab.p, V.t_int.p, S.part.p);
    launch(k_sip_sum, 1, 1024, 0, s, S.part.p, V.n_int, S.resab.p);
    CK(cudaGraphLaunch(S.sweep, s));
    halo<double>(C, V, 1, SUB_A);
    double resab = 0.0;
    CK(cudaMemcpyAsync(&resab, S.resab.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    C->launches += 2 + S.subst_launches;
    n = sweep;
    if (sweep == 1) res1 = resab;
    const double rsm = resab / (res1 + kSipSmall);
    const double reldif = std::fabs(rsm - relast);
    relast = rsm;
    if (rsm <= 0.001 || reldif <= 0.00001) break;
  }
  *sweeps = n;
  return MF3D_OK;
}

// pressure_1sweep: the outer loop on the host, one domain.
static int solve_view_sip(mf3d_ctx *C, View &V, const double *dt, const double *alfapr, mf3d_solve_info *infos,
                          double *hist, int hcap) {
  cudaStream_t s = C->stream;
  C->launches = 0;
  CK(cudaEventRecord(C->ev0, s));
  int st = solve_begin<double>(C, V, dt, alfapr);
  if (st) return st;
  if ((st = sip_prepare(C, V))) return st;
  DomState D;
  CK(cudaMemcpyAsync(&D, V.ds.p, sizeof D, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  const int maxcy = std::min(std::max(C->prm.maxcy, 0), V.hcap);
  double rmax = D.rmax0;
  int calls = 0, done = D.done == 2 ? 2 : 0;
  long long sweeps = 0;
  std::vector<double> hh;
  for (int iter = 1; iter <= maxcy && done == 0; ++iter) {
    if (iter > 1 && rmax < D.eps) { done = 1; break; }
    int n = 0;
    if ((st = sip_solve(C, V, &n))) return st;
    sweeps += n;
    ++calls;
    launch(k_add_correction<double>, V.n_pairs, kTile, 0, s, V.df.p, V.t_pairs.p, V.act.p, V.pairs_kch);
    p_exchange(C, V, V.act.p);
    CK(cudaMemsetAsync(V.rmax.p, 0, sizeof(unsigned long long), s));
    calvel_calmas<double>(C, V, V.act.p, V.rmax.p, 0);
    field_evolve(C, V, V.act.p);
    C->launches += 2;
    if (iter == maxcy) break;  // the reference runs no calmas after its last round
    unsigned long long bits = 0;
    CK(cudaMemcpyAsync(&bits, V.rmax.p, sizeof bits, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    std::memcpy(&rmax, &bits, sizeof rmax);
    hh.push_back(rmax);
    if (!(rmax <= 1.7976931348623157e308)) done = 2;
  }
  D.rmax = rmax;
  D.iter = calls;
  D.done = done == 0 ? 3 : done;
  C->sip_sweeps = sweeps;
  CK(cudaMemcpyAsync(V.ds.p, &D, sizeof D, cudaMemcpyHostToDevice, s));
  if (!hh.empty()) CK(cudaMemcpyAsync(V.hist.p, hh.data(), std::min<size_t>(hh.size(), V.hcap) * sizeof(double),
                                      cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  if ((st = solve_end<double>(C, V))) return st;
  CK(cudaEventRecord(C->ev1, s));
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  float ms = 0.f;
  cudaEventElapsedTime(&ms, C->ev0, C->ev1);
  // collect() reports D.iter entries of the history; ours holds one per
  // completed round that was followed by a calmas
  const int res = collect(C, V, infos, nullptr, 0, ms);
  if (hist && hcap > 0)
    for (int q = 0; q < (int)hh.size() && q < hcap; ++q) hist[q] = hh[q];
  return res;
}

}  // namespace mf3d
