// FP64 outer-loop kernels of newsolv_mg (newsolv_mg.for:2-102) on the
// reference's field layout: Fortran (ttc_i, ttc_j, ttc_k), i fastest, pl
// ghost layers.  Level-1 index i (0..nx+1, ghost-inclusive) is field index
// i + pl - 1 (0-based), so local index 1 is isp (mgsolver.for:245).
#pragma once

#include "kernels.cuh"

namespace mf3d {

// Device-resident control state of one solve (newsolv_mg's module variables
// dt, alfapr, eps, maxcy, iter, rmax), so the outer loop can run as a CUDA
// graph with no host round trip per iteration.
struct SolveState {
  double dt, alfapr;
  double eps;      // absolute threshold on rmax (eps * rmax0 in relative mode)
  double rmax;     // rmax after the last outer iteration
  int maxcy;
  int iter;        // outer iterations done
  int done;        // 0 running, 1 converged, 2 non-finite rmax, 3 maxcy reached
};

// Per-block view of the fields and of the level-1 multigrid arrays.
struct BlkFld {
  double *ustar, *vstar, *wstar, *u, *v, *w, *p, *su;
  int nx, ny, nz, pl, ti, tj;        // interior, ghost layers, ttc_i, ttc_j
  int wall[6];                       // 1 = physical (Neumann) face, W,E,S,N,B,T
  int src[6];                        // block supplying a non-wall face ghost
  double *lo[3], *hi[3];             // face planes: u,v,w at the low / high block face
  const double *h[3];                // cell widths, n+2 entries (ghost-inclusive)
  const double *df[3];               // centre distances of faces 0..n (face a: cells a|a+1)
  BlkLev L1;                         // level-1 descriptor
};

__device__ inline long long fidx(const BlkFld &F, int i, int j, int k) {
  // level-1 ghost-inclusive (i,j,k) -> 0-based ttc element
  return (long long)(i + F.pl - 1) + (long long)F.ti * ((long long)(j + F.pl - 1) + (long long)F.tj * (k + F.pl - 1));
}

// p := p + (pp - ppref) over isp-1..iep+1 (newsolv_mg.for:38-48), ppref = 0
// (the reference-pressure code is commented out, :28-36); pp is the level-1
// correction of the V-cycle.  One thread per ghost-inclusive level-1 cell.
template <typename T>
__global__ void __launch_bounds__(kTile) k_add_correction(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles,
                                                          const T *__restrict__ phi1) {
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  const BlkLev &B = F.L1;
  const int W = B.nx + 2, H = B.ny + 2;
  const long long q = (long long)t.item0 + threadIdx.x;
  if (q >= (long long)W * H * (B.nz + 2)) return;
  const int k = (int)(q / ((long long)W * H));
  const int rem = (int)(q - (long long)k * W * H);
  const int j = rem / W, i = rem - j * W;
  const double pp = (double)phi1[cell_addr(B, B.phi0, i, j, k)];
  const double ppref = 0.0;
  double *p = F.p + fidx(F, i, j, k);
  *p = (*p + (pp - ppref));
}

// exchange(4) + pbound on the face ghosts of p (exchange.for:2402-2490,
// exchange_bc.for, press.for:77-137): inter-block and periodic faces take
// the source block's adjacent interior value, wall faces mirror the first
// interior cell.  Only the interior tangential range: the path reads no
// other ghost of p.  Items per block: 2*(ny*nz + nx*nz + nx*ny).
__global__ void k_p_faces(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles) {
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  int q = t.item0 + threadIdx.x;
  const int nx = F.nx, ny = F.ny, nz = F.nz;
  const int nyz = ny * nz, nxz = nx * nz, nxy = nx * ny;
  int f, a, b;
  if (q < 2 * nyz) { f = q / nyz; q -= f * nyz; a = q % ny + 1; b = q / ny + 1; }
  else if ((q -= 2 * nyz) < 2 * nxz) { f = 2 + q / nxz; q -= (f - 2) * nxz; a = q % nx + 1; b = q / nx + 1; }
  else if ((q -= 2 * nxz) < 2 * nxy) { f = 4 + q / nxy; q -= (f - 4) * nxy; a = q % nx + 1; b = q / nx + 1; }
  else return;
  int gi, gj, gk, si, sj, sk;  // ghost cell; source cell (in the source block)
  const bool wall = F.wall[f];
  const BlkFld &S = wall ? F : fl[F.src[f]];
  switch (f) {
    case 0: gi = 0; gj = a; gk = b; si = wall ? 1 : S.nx; sj = a; sk = b; break;
    case 1: gi = nx + 1; gj = a; gk = b; si = wall ? nx : 1; sj = a; sk = b; break;
    case 2: gi = a; gj = 0; gk = b; si = a; sj = wall ? 1 : S.ny; sk = b; break;
    case 3: gi = a; gj = ny + 1; gk = b; si = a; sj = wall ? ny : 1; sk = b; break;
    case 4: gi = a; gj = b; gk = 0; si = a; sj = b; sk = wall ? 1 : S.nz; break;
    default: gi = a; gj = b; gk = nz + 1; si = a; sj = b; sk = wall ? nz : 1; break;
  }
  F.p[fidx(F, gi, gj, gk)] = S.p[fidx(S, si, sj, sk)];
}

// Face planes used by the fused calvel/calmas kernel, filled once per solve:
// lo[a] = the velocity component normal to the block's low face on that face
// when it is a wall (the caller's boundary value, never rewritten by calvel),
// else the source block's ustar on its last face (exchange(1..3) hands over
// that block's u); hi[a] = the caller's velocity on a high wall face
// (localparameters.for:185-190 stops calvel one face short there).
__global__ void k_face_planes(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles) {
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  int q = t.item0 + threadIdx.x;
  const int nx = F.nx, ny = F.ny, nz = F.nz;
  const int nyz = ny * nz, nxz = nx * nz, nxy = nx * ny;
  int ax, a, b;
  if (q < nyz) { ax = 0; a = q % ny + 1; b = q / ny + 1; }
  else if ((q -= nyz) < nxz) { ax = 1; a = q % nx + 1; b = q / nx + 1; }
  else if ((q -= nxz) < nxy) { ax = 2; a = q % nx + 1; b = q / nx + 1; }
  else return;
  const int fl0 = 2 * ax, fh = 2 * ax + 1;
  double *vel = ax == 0 ? F.u : ax == 1 ? F.v : F.w;
  const int plane = ax == 0 ? ny : nx;
  const int o = (b - 1) * plane + (a - 1);
  // low face
  if (F.wall[fl0]) {
    long long e = ax == 0 ? fidx(F, 0, a, b) : ax == 1 ? fidx(F, a, 0, b) : fidx(F, a, b, 0);
    F.lo[ax][o] = vel[e];
  } else {
    const BlkFld &S = fl[F.src[fl0]];
    const double *st = ax == 0 ? S.ustar : ax == 1 ? S.vstar : S.wstar;
    long long e = ax == 0 ? fidx(S, S.nx, a, b) : ax == 1 ? fidx(S, a, S.ny, b) : fidx(S, a, b, S.nz);
    F.lo[ax][o] = st[e];
  }
  // high face
  long long e = ax == 0 ? fidx(F, nx, a, b) : ax == 1 ? fidx(F, a, ny, b) : fidx(F, a, b, nz);
  F.hi[ax][o] = F.wall[fh] ? vel[e] : 0.0;
}

__device__ inline void atomic_max_nonneg(unsigned long long *slot, double v) {
  // |x| >= 0: the IEEE bit pattern orders like the value
  atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}

// calvel (press.for:139-198) fused with calmas (press.for:38-73): each
// interior cell forms the six face velocities it needs -
//   u(i) = ustar(i) - dt*alfapr*(p(i+1)-p(i))/dx   (face between i and i+1)
// with the faces the reference never recomputes taken from the face planes -
// then fact = (u(i)-u(i-1))/dx + (v(j)-v(j-1))/dy + (w(k)-w(k-1))/dz,
// su = fact/dt (written into the level-1 multigrid rhs) and
// rmax = max |fact*dx*dy*dz| (MPI_MAX over one device: an order-free
// atomic max on the bit pattern, hence deterministic).
template <typename T>
__global__ void __launch_bounds__(kTile) k_calvel_calmas(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles,
                                                         const SolveState *__restrict__ st, T *__restrict__ rhs1,
                                                         unsigned long long *__restrict__ rmax_slot, int write_su) {
  const double dt = st->dt, alfapr = st->alfapr;
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  const int nx = F.nx, ny = F.ny;
  const long long q = (long long)t.item0 + threadIdx.x;
  double fact1 = 0.0;
  if (q < (long long)nx * ny * F.nz) {
    const int k = (int)(q / ((long long)nx * ny)) + 1;
    const int rem = (int)(q - (long long)(k - 1) * nx * ny);
    const int j = rem / nx + 1, i = rem - (j - 1) * nx + 1;
    const double dta = dt * alfapr;
    const long long c = fidx(F, i, j, k);
    const long long sx = 1, sy = F.ti, sz = (long long)F.ti * F.tj;
    const double *p = F.p;
    const double pc = p[c];
    // x faces
    double ue, uw;
    if (i == nx && F.wall[1]) ue = F.hi[0][(k - 1) * ny + (j - 1)];
    else ue = (F.ustar[c] - dta * (p[c + sx] - pc) / F.df[0][i]);
    if (i == 1) {
      const double lo = F.lo[0][(k - 1) * ny + (j - 1)];
      uw = F.wall[0] ? lo : (lo - dta * (pc - p[c - sx]) / F.df[0][0]);
    } else {
      uw = (F.ustar[c - sx] - dta * (pc - p[c - sx]) / F.df[0][i - 1]);
    }
    // y faces
    double vn, vs;
    if (j == ny && F.wall[3]) vn = F.hi[1][(k - 1) * nx + (i - 1)];
    else vn = (F.vstar[c] - dta * (p[c + sy] - pc) / F.df[1][j]);
    if (j == 1) {
      const double lo = F.lo[1][(k - 1) * nx + (i - 1)];
      vs = F.wall[2] ? lo : (lo - dta * (pc - p[c - sy]) / F.df[1][0]);
    } else {
      vs = (F.vstar[c - sy] - dta * (pc - p[c - sy]) / F.df[1][j - 1]);
    }
    // z faces
    double wt, wb;
    if (k == F.nz && F.wall[5]) wt = F.hi[2][(j - 1) * nx + (i - 1)];
    else wt = (F.wstar[c] - dta * (p[c + sz] - pc) / F.df[2][k]);
    if (k == 1) {
      const double lo = F.lo[2][(j - 1) * nx + (i - 1)];
      wb = F.wall[4] ? lo : (lo - dta * (pc - p[c - sz]) / F.df[2][0]);
    } else {
      wb = (F.wstar[c - sz] - dta * (pc - p[c - sz]) / F.df[2][k - 1]);
    }
    const double hx = F.h[0][i], hy = F.h[1][j], hz = F.h[2][k];
    const double fact = ((ue - uw) / hx + (vn - vs) / hy + (wt - wb) / hz);
    const double su = fact / dt;
    rhs1[cell_addr(F.L1, F.L1.rhs0, i, j, k)] = (T)su;
    if (write_su && F.su) F.su[c] = su;
    fact1 = fact * hx * hy * hz;
    fact1 = fabs(fact1);
    if (!(fact1 == fact1)) fact1 = __longlong_as_double(0x7ff0000000000000LL);  // NaN -> +Inf (flagged)
  }
  // CTA max: warp shuffles, then one atomic per warp
  for (int o = 16; o > 0; o >>= 1) fact1 = fmax(fact1, __shfl_xor_sync(0xffffffffu, fact1, o));
  if ((threadIdx.x & 31) == 0 && fact1 > 0.0) atomic_max_nonneg(rmax_slot, fact1);
}

// Final calvel (press.for:139-198): u, v, w on the faces calvel writes
// (isu..ieu etc., one face short at a high wall), from the final p.
__global__ void __launch_bounds__(kTile) k_calvel(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles,
                                                  const SolveState *__restrict__ st) {
  const double dt = st->dt, alfapr = st->alfapr;
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  const int nx = F.nx, ny = F.ny;
  const long long q = (long long)t.item0 + threadIdx.x;
  if (q >= (long long)nx * ny * F.nz) return;
  const int k = (int)(q / ((long long)nx * ny)) + 1;
  const int rem = (int)(q - (long long)(k - 1) * nx * ny);
  const int j = rem / nx + 1, i = rem - (j - 1) * nx + 1;
  const double dta = dt * alfapr;
  const long long c = fidx(F, i, j, k);
  const long long sy = F.ti, sz = (long long)F.ti * F.tj;
  const double *p = F.p;
  if (!(i == nx && F.wall[1])) F.u[c] = (F.ustar[c] - dta * (p[c + 1] - p[c]) / F.df[0][i]);
  if (!(j == ny && F.wall[3])) F.v[c] = (F.vstar[c] - dta * (p[c + sy] - p[c]) / F.df[1][j]);
  if (!(k == F.nz && F.wall[5])) F.w[c] = (F.wstar[c] - dta * (p[c + sz] - p[c]) / F.df[2][k]);
}

// End of one outer iteration (newsolv_mg.for:54-58): record rmax, count the
// iteration, test `rmax < eps .and. iter > 1`, and - inside the solve graph -
// set the WHILE condition that repeats the iteration body.
__global__ void k_iter_end(SolveState *st, unsigned long long *rmax_slot, double *hist,
                           cudaGraphConditionalHandle cond, int in_graph) {
  const double r = __longlong_as_double((long long)*rmax_slot);
  *rmax_slot = 0ull;
  const int it = st->iter + 1;
  st->iter = it;
  st->rmax = r;
  hist[it - 1] = r;
  int done = 0;
  if (!(r <= 1.7976931348623157e308)) done = 2;  // +Inf (a NaN is stored as +Inf)
  else if (r < st->eps && it > 1) done = 1;
  else if (it >= st->maxcy) done = 3;
  st->done = done;
  if (in_graph) cudaGraphSetConditional(cond, done ? 0u : 1u);
}

// Level-1 rhs := su (mgkcyc's copy-in, mgsolver.for:250-263) from a ttc array.
template <typename T>
__global__ void k_load_rhs(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles, double *const *__restrict__ su,
                           T *__restrict__ rhs1) {
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  const int nx = F.nx, ny = F.ny;
  const long long q = (long long)t.item0 + threadIdx.x;
  if (q >= (long long)nx * ny * F.nz) return;
  const int k = (int)(q / ((long long)nx * ny)) + 1;
  const int rem = (int)(q - (long long)(k - 1) * nx * ny);
  const int j = rem / nx + 1, i = rem - (j - 1) * nx + 1;
  rhs1[cell_addr(F.L1, F.L1.rhs0, i, j, k)] = (T)su[t.blk][fidx(F, i, j, k)];
}

// pp := level-1 phi including the first ghost layer (mgsolver.for:351-364).
template <typename T>
__global__ void k_store_pp(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles, double *const *__restrict__ pp,
                           const T *__restrict__ phi1) {
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  const BlkLev &B = F.L1;
  const int W = B.nx + 2, H = B.ny + 2;
  const long long q = (long long)t.item0 + threadIdx.x;
  if (q >= (long long)W * H * (B.nz + 2)) return;
  const int k = (int)(q / ((long long)W * H));
  const int rem = (int)(q - (long long)k * W * H);
  const int j = rem / W, i = rem - j * W;
  pp[t.blk][fidx(F, i, j, k)] = (double)phi1[cell_addr(B, B.phi0, i, j, k)];
}

}  // namespace mf3d
