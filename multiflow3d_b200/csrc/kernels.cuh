// Device kernels of libmf3d (sm_100a).
//
// Storage of a multigrid level (the reference keeps it in `cof`,
// mgsolver.for:20-38): every block's correction phi and right-hand side,
// each with a one-cell ghost shell, split by red/black colour.  Cell (i,j,k)
// (0-based, ghost-inclusive, 0..n+1) has colour c = (i+j+k+1)&1 - colour 0
// is the reference's even MOD(i+j+k,2) on its 1-based indices, updated first
// (mgsolver.for:552) - and lives at
//     base + c*cstr + (k*(ny+2) + j)*hp + (i>>1),   hp = (nx+3)/2.
// A red-black half-sweep then streams exactly one colour in and the other
// out: 12 B/cell/half-sweep in FP64, contiguous and coalesced along i.
//
// The 7-point coefficients are not stored per cell (the reference streams 7
// arrays, ~80 B/cell/sweep): per level and block, six 1-D arrays
// (aw, ae along x; as, an along y; ab, at along z) with the Neumann faces
// zeroed (mgsolver.for:184-203); ap = -(aw+ae+as+an+ab+at) is re-formed per
// cell in the reference's order (mgsolver.for:205-208), so every value is
// bit-identical to the reference's `cof` entries.
//
// Every FP64 expression keeps the reference's evaluation order; the file is
// built with -fmad=false so no multiply-add is contracted.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace mf3d {

constexpr int kTile = 256;  // threads (= work items) per CTA for the 1-D tiled kernels

// Per-block, per-level descriptor (device side).
struct BlkLev {
  long long phi0;   // offset of colour 0 in the level's phi pool
  long long rhs0;   // offset of colour 0 in the level's rhs pool
  long long cstr;   // elements per colour array = (nz+2)*(ny+2)*hp
  int nx, ny, nz, hp;
  int coef;         // offset of aw in the level coefficient pool (6 arrays, see coef_*)
  int geo;          // offset of the restriction ratio arrays (rx, ry, rz) of this level
  int nmask;        // Neumann faces: bit f set for f = W,E,S,N,B,T
  int pos;          // block position
};

__host__ __device__ inline int hp_of(int nx) { return (nx + 3) / 2; }
__device__ inline int colour_of(int i, int j, int k) { return (i + j + k + 1) & 1; }
__device__ inline long long cell_addr(const BlkLev &B, long long base, int i, int j, int k) {
  int c = colour_of(i, j, k);
  return base + c * B.cstr + ((long long)k * (B.ny + 2) + j) * B.hp + (i >> 1);
}
// Coefficient layout: aw[nx+2], ae[nx+2], as[ny+2], an[ny+2], ab[nz+2], at[nz+2].
__device__ inline int coef_aw(const BlkLev &B) { return B.coef; }
__device__ inline int coef_ae(const BlkLev &B) { return B.coef + (B.nx + 2); }
__device__ inline int coef_as(const BlkLev &B) { return B.coef + 2 * (B.nx + 2); }
__device__ inline int coef_an(const BlkLev &B) { return B.coef + 2 * (B.nx + 2) + (B.ny + 2); }
__device__ inline int coef_ab(const BlkLev &B) { return B.coef + 2 * (B.nx + 2) + 2 * (B.ny + 2); }
__device__ inline int coef_at(const BlkLev &B) { return B.coef + 2 * (B.nx + 2) + 2 * (B.ny + 2) + (B.nz + 2); }

// A CTA's work: block position and first item.
struct Tile {
  int blk;
  int item0;
};

// ---------------------------------------------------------------------------
// Red-black Gauss-Seidel half-sweep (mgsolver.for:547-601) of one colour over
// all blocks of a level: phi = (rhs - (aw*w + ae*e + as*s + an*n + ab*b +
// at*t)) / ap, neighbours of the other colour.  Ghost cells are read as they
// are: the reference refreshes them only after the whole sweep.  Items: the
// compact (h, j, k) positions of the interior rows, hp per row.
// FROM_ZERO: the level was just zeroed (pp = 0 at the start of a V-cycle,
// coarse phi = 0 after mgrestr), so the other colour is read as 0 without a
// load; the result is bit-identical.
// ---------------------------------------------------------------------------
template <typename T, bool FROM_ZERO>
__global__ void __launch_bounds__(kTile) k_rbgs(const BlkLev *__restrict__ bl, const Tile *__restrict__ tiles,
                                                T *__restrict__ phi, const T *__restrict__ rhs,
                                                const T *__restrict__ coef, int colour) {
  const Tile t = tiles[blockIdx.x];
  const BlkLev B = bl[t.blk];
  const int hp = B.hp;
  const long long plane = (long long)B.ny * hp;
  const long long q = (long long)t.item0 + threadIdx.x;
  if (q >= plane * B.nz) return;
  const int k = (int)(q / plane) + 1;
  const int rem = (int)(q - (long long)(k - 1) * plane);
  const int j = rem / hp + 1;
  const int h = rem - (j - 1) * hp;
  const int s = (colour + j + k + 1) & 1;
  const int i = 2 * h + s;
  if (i < 1 || i > B.nx) return;
  const long long rs = (long long)(B.ny + 2) * hp;  // plane stride
  const long long row = (long long)k * rs + (long long)j * hp;
  const T aw = coef[coef_aw(B) + i], ae = coef[coef_ae(B) + i];
  const T as = coef[coef_as(B) + j], an = coef[coef_an(B) + j];
  const T ab = coef[coef_ab(B) + k], at = coef[coef_at(B) + k];
  const T ap = (T)-1.0 * (aw + ae + as + an + ab + at);
  T w, e, so, no, bo, to;
  if (FROM_ZERO) {
    w = e = so = no = bo = to = (T)0;
  } else {
    const T *P = phi + B.phi0 + (1 - colour) * B.cstr + row;
    w = P[h - 1 + s];
    e = P[h + s];
    so = P[h - hp];
    no = P[h + hp];
    bo = P[h - rs];
    to = P[h + rs];
  }
  const T r = rhs[B.rhs0 + colour * B.cstr + row + h];
  phi[B.phi0 + colour * B.cstr + row + h] = ((r - (aw * w + ae * e + as * so + an * no + ab * bo + at * to)) / ap);
}

// ---------------------------------------------------------------------------
// Lexicographic Gauss-Seidel (mgsolver.for:403-428), loop order k, j, i:
// cell (i,j,k) reads new values at i-1, j-1, k-1 and old ones at i+1, j+1,
// k+1, so every hyperplane i+j+k = const is independent.  One CTA per block
// walks the hyperplanes in order (a parity kernel for small blocks).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_lexgs(const BlkLev *__restrict__ bl, T *__restrict__ phi, const T *__restrict__ rhs,
                        const T *__restrict__ coef) {
  const BlkLev B = bl[blockIdx.x];
  const int nx = B.nx, ny = B.ny, nz = B.nz;
  const long long rs = (long long)(ny + 2) * B.hp;
  for (int sum = 3; sum <= nx + ny + nz; ++sum) {
    // cells with i+j+k = sum, 1<=i<=nx, 1<=j<=ny, 1<=k<=nz; enumerate (j,k)
    for (int idx = threadIdx.x; idx < ny * nz; idx += blockDim.x) {
      const int j = idx % ny + 1, k = idx / ny + 1;
      const int i = sum - j - k;
      if (i < 1 || i > nx) continue;
      const T aw = coef[coef_aw(B) + i], ae = coef[coef_ae(B) + i];
      const T as = coef[coef_as(B) + j], an = coef[coef_an(B) + j];
      const T ab = coef[coef_ab(B) + k], at = coef[coef_at(B) + k];
      const T ap = (T)-1.0 * (aw + ae + as + an + ab + at);
      const T w = phi[cell_addr(B, B.phi0, i - 1, j, k)], e = phi[cell_addr(B, B.phi0, i + 1, j, k)];
      const T so = phi[cell_addr(B, B.phi0, i, j - 1, k)], no = phi[cell_addr(B, B.phi0, i, j + 1, k)];
      const T bo = phi[cell_addr(B, B.phi0, i, j, k - 1)], to = phi[cell_addr(B, B.phi0, i, j, k + 1)];
      const T r = rhs[cell_addr(B, B.rhs0, i, j, k)];
      phi[cell_addr(B, B.phi0, i, j, k)] = ((r - (aw * w + ae * e + as * so + an * no + ab * bo + at * to)) / ap);
      (void)rs;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Line TDMA relaxation (mgsolver.for:430-545): Thomas solves along j-lines
// (line order k, i), then i-lines (k, j), then k-lines (i, j), each pass a
// Gauss-Seidel over lines.  Lines whose two transverse indices have the same
// sum are independent, so one CTA per block sweeps those diagonals in order,
// one thread per line.  `work` gives each thread two scratch vectors (a, c)
// of length `ngg`.  a(1) = 0 and c(1) = the line's first ghost value.
// ---------------------------------------------------------------------------
template <typename T>
__device__ void tdma_line(const BlkLev &B, T *__restrict__ phi, const T *__restrict__ rhs,
                          const T *__restrict__ coef, int dir, int u, int v, T *a, T *c) {
  // dir 0: j-line at (i=u, k=v); dir 1: i-line at (j=u, k=v); dir 2: k-line at (i=u, j=v)
  const int n = dir == 0 ? B.ny : dir == 1 ? B.nx : B.nz;
  auto addr = [&](int m) -> long long {
    if (dir == 0) return cell_addr(B, B.phi0, u, m, v);
    if (dir == 1) return cell_addr(B, B.phi0, m, u, v);
    return cell_addr(B, B.phi0, u, v, m);
  };
  auto raddr = [&](int m) -> long long {
    if (dir == 0) return cell_addr(B, B.rhs0, u, m, v);
    if (dir == 1) return cell_addr(B, B.rhs0, m, u, v);
    return cell_addr(B, B.rhs0, u, v, m);
  };
  a[0] = (T)0;
  c[0] = phi[addr(0)];
  for (int m = 1; m <= n; ++m) {
    int i, j, k;
    if (dir == 0) { i = u; j = m; k = v; }
    else if (dir == 1) { i = m; j = u; k = v; }
    else { i = u; j = v; k = m; }
    const T aw = coef[coef_aw(B) + i], ae = coef[coef_ae(B) + i];
    const T as = coef[coef_as(B) + j], an = coef[coef_an(B) + j];
    const T ab = coef[coef_ab(B) + k], at = coef[coef_at(B) + k];
    const T ap = (T)-1.0 * (aw + ae + as + an + ab + at);
    const T su = rhs[raddr(m)];
    if (dir == 0) {
      const T apr = (T)1.0 / (ap - as * a[m - 1]);
      a[m] = an * apr;
      c[m] = (su - ae * phi[cell_addr(B, B.phi0, i + 1, j, k)] - aw * phi[cell_addr(B, B.phi0, i - 1, j, k)] -
              at * phi[cell_addr(B, B.phi0, i, j, k + 1)] - ab * phi[cell_addr(B, B.phi0, i, j, k - 1)] -
              as * c[m - 1]) * apr;
    } else if (dir == 1) {
      const T apr = (T)1.0 / (ap - aw * a[m - 1]);
      a[m] = ae * apr;
      c[m] = (su - an * phi[cell_addr(B, B.phi0, i, j + 1, k)] - as * phi[cell_addr(B, B.phi0, i, j - 1, k)] -
              at * phi[cell_addr(B, B.phi0, i, j, k + 1)] - ab * phi[cell_addr(B, B.phi0, i, j, k - 1)] -
              aw * c[m - 1]) * apr;
    } else {
      const T apr = (T)1.0 / (ap - ab * a[m - 1]);
      a[m] = at * apr;
      c[m] = (su - an * phi[cell_addr(B, B.phi0, i, j + 1, k)] - as * phi[cell_addr(B, B.phi0, i, j - 1, k)] -
              ae * phi[cell_addr(B, B.phi0, i + 1, j, k)] - aw * phi[cell_addr(B, B.phi0, i - 1, j, k)] -
              ab * c[m - 1]) * apr;
    }
  }
  for (int m = n; m >= 1; --m) phi[addr(m)] = (c[m] - a[m] * phi[addr(m + 1)]);
}

template <typename T>
__global__ void k_tdma(const BlkLev *__restrict__ bl, T *__restrict__ phi, const T *__restrict__ rhs,
                       const T *__restrict__ coef, T *__restrict__ work, int ngg) {
  const BlkLev B = bl[blockIdx.x];
  T *a = work + ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 2 * ngg;
  T *c = a + ngg;
  for (int dir = 0; dir < 3; ++dir) {
    // transverse extents (u, v) and the line order of the reference
    const int nu = dir == 0 ? B.nx : dir == 1 ? B.ny : B.nx;
    const int nv = dir == 0 ? B.nz : dir == 1 ? B.nz : B.ny;
    for (int sum = 2; sum <= nu + nv; ++sum) {
      for (int u = 1 + threadIdx.x; u <= nu; u += blockDim.x) {
        const int v = sum - u;
        if (v < 1 || v > nv) continue;
        tdma_line(B, phi, rhs, coef, dir, u, v, a, c);
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// Residual + restriction (mgrestr, mgsolver.for:619-761), one thread per
// coarse cell including its ghost shell: coarse phi := 0 everywhere
// (:650-657); interior coarse rhs := 0.125 * sum over the 8 children of
// s * (rhs - (aw*w + ae*e + as*s + an*n + ab*b + at*t + ap*p)) in the
// reference's child order (:743-747).  s = 8*rx*ry*rz is the volume weight
// of the non-uniform-grid extension and is exactly 1.0 on a uniform grid.
// ---------------------------------------------------------------------------
template <typename T>
__device__ inline T residual_at(const BlkLev &F, const T *__restrict__ phi, const T *__restrict__ rhs,
                                const T *__restrict__ coef, int i, int j, int k) {
  const T aw = coef[coef_aw(F) + i], ae = coef[coef_ae(F) + i];
  const T as = coef[coef_as(F) + j], an = coef[coef_an(F) + j];
  const T ab = coef[coef_ab(F) + k], at = coef[coef_at(F) + k];
  const T ap = (T)-1.0 * (aw + ae + as + an + ab + at);
  const T pw = phi[cell_addr(F, F.phi0, i - 1, j, k)], pe = phi[cell_addr(F, F.phi0, i + 1, j, k)];
  const T ps = phi[cell_addr(F, F.phi0, i, j - 1, k)], pn = phi[cell_addr(F, F.phi0, i, j + 1, k)];
  const T pb = phi[cell_addr(F, F.phi0, i, j, k - 1)], pt = phi[cell_addr(F, F.phi0, i, j, k + 1)];
  const T pp = phi[cell_addr(F, F.phi0, i, j, k)];
  const T r = rhs[cell_addr(F, F.rhs0, i, j, k)];
  return r - (aw * pw + ae * pe + as * ps + an * pn + ab * pb + at * pt + ap * pp);
}

template <typename TF, typename TC>
__global__ void __launch_bounds__(kTile) k_restrict(const BlkLev *__restrict__ fl, const BlkLev *__restrict__ cl,
                                                    const Tile *__restrict__ tiles, const TF *__restrict__ phif,
                                                    const TF *__restrict__ rhsf, const TF *__restrict__ coeff,
                                                    TC *__restrict__ phic, TC *__restrict__ rhsc,
                                                    const TF *__restrict__ geo) {
  const Tile t = tiles[blockIdx.x];
  const BlkLev Cb = cl[t.blk];
  const BlkLev Fb = fl[t.blk];
  const int W = Cb.nx + 2, H = Cb.ny + 2;
  const long long q = (long long)t.item0 + threadIdx.x;
  if (q >= (long long)W * H * (Cb.nz + 2)) return;
  const int k = (int)(q / ((long long)W * H));
  const int rem = (int)(q - (long long)k * W * H);
  const int j = rem / W, i = rem - j * W;
  phic[cell_addr(Cb, Cb.phi0, i, j, k)] = (TC)0;
  if (i < 1 || i > Cb.nx || j < 1 || j > Cb.ny || k < 1 || k > Cb.nz) return;
  // restriction ratios of the fine level: rx[nxf+2], ry[nyf+2], rz[nzf+2]
  const TF *rx = geo + Fb.geo, *ry = rx + (Fb.nx + 2), *rz = ry + (Fb.ny + 2);
  TF acc[8];
  int n = 0;
  for (int dk = 0; dk < 2; ++dk)
    for (int dj = 0; dj < 2; ++dj)
      for (int di = 0; di < 2; ++di) {
        const int fi = 2 * i - 1 + di, fj = 2 * j - 1 + dj, fk = 2 * k - 1 + dk;
        const TF s = (TF)8.0 * rx[fi] * ry[fj] * rz[fk];
        acc[n++] = residual_at(Fb, phif, rhsf, coeff, fi, fj, fk) * s;
      }
  const TF v = (TF)0.125 * (acc[0] + acc[1] + acc[2] + acc[3] + acc[4] + acc[5] + acc[6] + acc[7]);
  rhsc[cell_addr(Cb, Cb.rhs0, i, j, k)] = (TC)v;
}

// ---------------------------------------------------------------------------
// Prolongation + correction + Neumann ghosts (mgcorr, mgsolver.for:763-905,
// then mgbound :902).  Every fine cell, ghosts included, adds the trilinear
// (27,9,3,1)/64 interpolant of the coarse correction, summed in the
// reference's term order (:833-887).  A fine cell on a Neumann face of the
// block then also writes its corrected value into the ghost cells that
// mgbound copies it to, so no cell is read after another thread wrote it.
// ---------------------------------------------------------------------------
template <typename TF, typename TC>
__global__ void __launch_bounds__(kTile) k_prolong(const BlkLev *__restrict__ fl, const BlkLev *__restrict__ cl,
                                                   const Tile *__restrict__ tiles, TF *__restrict__ phif,
                                                   const TC *__restrict__ phic) {
  const Tile t = tiles[blockIdx.x];
  const BlkLev Fb = fl[t.blk];
  const BlkLev Cb = cl[t.blk];
  const int W = Fb.nx + 2, H = Fb.ny + 2;
  const long long q = (long long)t.item0 + threadIdx.x;
  if (q >= (long long)W * H * (Fb.nz + 2)) return;
  const int k = (int)(q / ((long long)W * H));
  const int rem = (int)(q - (long long)k * W * H);
  const int j = rem / W, i = rem - j * W;
  const int m = Fb.nmask;
  // Neumann ghost cells are written by their owners below
  if ((i == 0 && (m & 1)) || (i == Fb.nx + 1 && (m & 2)) || (j == 0 && (m & 4)) || (j == Fb.ny + 1 && (m & 8)) ||
      (k == 0 && (m & 16)) || (k == Fb.nz + 1 && (m & 32)))
    return;
  const int ic = i >> 1, jc = j >> 1, kc = k >> 1;        // lower coarse cell
  const int wi0 = (i & 1) ? 1 : 3, wj0 = (j & 1) ? 1 : 3, wk0 = (k & 1) ? 1 : 3;
  const int wi1 = 4 - wi0, wj1 = 4 - wj0, wk1 = 4 - wk0;
  const TF c000 = (TF)phic[cell_addr(Cb, Cb.phi0, ic, jc, kc)];
  const TF c010 = (TF)phic[cell_addr(Cb, Cb.phi0, ic, jc + 1, kc)];
  const TF c001 = (TF)phic[cell_addr(Cb, Cb.phi0, ic, jc, kc + 1)];
  const TF c011 = (TF)phic[cell_addr(Cb, Cb.phi0, ic, jc + 1, kc + 1)];
  const TF c100 = (TF)phic[cell_addr(Cb, Cb.phi0, ic + 1, jc, kc)];
  const TF c110 = (TF)phic[cell_addr(Cb, Cb.phi0, ic + 1, jc + 1, kc)];
  const TF c101 = (TF)phic[cell_addr(Cb, Cb.phi0, ic + 1, jc, kc + 1)];
  const TF c111 = (TF)phic[cell_addr(Cb, Cb.phi0, ic + 1, jc + 1, kc + 1)];
  const TF corr = ((TF)(wi0 * wj0 * wk0) * c000 + (TF)(wi0 * wj1 * wk0) * c010 + (TF)(wi0 * wj0 * wk1) * c001 +
                   (TF)(wi0 * wj1 * wk1) * c011 + (TF)(wi1 * wj0 * wk0) * c100 + (TF)(wi1 * wj1 * wk0) * c110 +
                   (TF)(wi1 * wj0 * wk1) * c101 + (TF)(wi1 * wj1 * wk1) * c111) /
                  (TF)64.0;
  const long long a = cell_addr(Fb, Fb.phi0, i, j, k);
  const TF v = phif[a] + corr;
  phif[a] = v;
  // mirror targets on Neumann faces (mgbound order W,E,S,N,B,T composes to a clamp)
  int xs[3] = {i, i, i}, ys[3] = {j, j, j}, zs[3] = {k, k, k};
  int nxo = 1, nyo = 1, nzo = 1;
  if (i == 1 && (m & 1)) xs[nxo++] = 0;
  if (i == Fb.nx && (m & 2)) xs[nxo++] = Fb.nx + 1;
  if (j == 1 && (m & 4)) ys[nyo++] = 0;
  if (j == Fb.ny && (m & 8)) ys[nyo++] = Fb.ny + 1;
  if (k == 1 && (m & 16)) zs[nzo++] = 0;
  if (k == Fb.nz && (m & 32)) zs[nzo++] = Fb.nz + 1;
  if (nxo == 1 && nyo == 1 && nzo == 1) return;
  for (int a3 = 0; a3 < nzo; ++a3)
    for (int a2 = 0; a2 < nyo; ++a2)
      for (int a1 = 0; a1 < nxo; ++a1) {
        if (a1 == 0 && a2 == 0 && a3 == 0) continue;
        phif[cell_addr(Fb, Fb.phi0, xs[a1], ys[a2], zs[a3])] = v;
      }
}

// ---------------------------------------------------------------------------
// Halo copies of one level: the composition of exchangepp + mgbound +
// exchbc_mgpp as (dst, src) element pairs against the state before the
// exchange.  Pairs [0, nstaged) have a source that is itself overwritten:
// k_halo_stage reads those first, k_halo_apply writes everything.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_halo_stage(const long long *__restrict__ src, int nstaged, const T *__restrict__ phi,
                             T *__restrict__ buf) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nstaged) buf[t] = phi[src[t]];
}
template <typename T>
__global__ void k_halo_apply(const long long *__restrict__ dst, const long long *__restrict__ src, int n,
                             int nstaged, T *__restrict__ phi, const T *__restrict__ buf) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  T v = t < nstaged ? buf[t] : phi[src[t]];
  phi[dst[t]] = v;
}

// Zero the ghost shell of every block of a level (pp = 0 before a V-cycle).
template <typename T>
__global__ void k_zero_ghosts(const BlkLev *__restrict__ bl, const Tile *__restrict__ tiles, T *__restrict__ phi) {
  const Tile t = tiles[blockIdx.x];
  const BlkLev B = bl[t.blk];
  const int W = B.nx + 2, H = B.ny + 2;
  const long long q = (long long)t.item0 + threadIdx.x;
  if (q >= (long long)W * H * (B.nz + 2)) return;
  const int k = (int)(q / ((long long)W * H));
  const int rem = (int)(q - (long long)k * W * H);
  const int j = rem / W, i = rem - j * W;
  if (i >= 1 && i <= B.nx && j >= 1 && j <= B.ny && k >= 1 && k <= B.nz) return;
  phi[cell_addr(B, B.phi0, i, j, k)] = (T)0;
}

}  // namespace mf3d
