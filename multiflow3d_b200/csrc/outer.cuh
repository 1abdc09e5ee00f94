// FP64 outer-loop kernels of newsolv_mg (newsolv_mg.for:2-102) on the
// reference's field layout: Fortran (ttc_i, ttc_j, ttc_k), i fastest, pl
// ghost layers.  Level-1 index i (0..nx+1, ghost-inclusive) is field index
// i + pl - 1 (0-based), so local index 1 is isp (mgsolver.for:245).
#pragma once

#include "kernels.cuh"

namespace mf3d {

// Device-resident control state of one domain's solve (newsolv_mg's module
// variables dt, alfapr, eps, maxcy, iter, rmax), so the outer loop runs as a
// CUDA graph with no host round trip per iteration; independent domains
// (a batch) each carry their own.
struct DomState {
  double dt, alfapr;
  double tol;      // eps as given
  double eps;      // absolute threshold on rmax (tol * rmax0 in relative mode)
  double rmax0;    // rmax after the initial calvel/calmas
  double rmax;     // rmax after the last outer iteration
  double dtinv;    // 1/dt when dt is a power of two, else 0 (see xdiv)
  double rdt;      // RN(1/dt) for div_rcp (0: divide)
  int maxcy;
  int eps_relative;
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
  int dom;                           // domain of the block
  double pinv[3];                    // 1/h when the axis is uniform with h a power of two, else 0
  const CUtensorMap *fm;             // TMA maps of p, ustar, vstar, wstar (CvShape boxes), or null
  const double *rh[3], *rdf[3];      // RN(1/h), RN(1/df) for div_rcp (0: divide)
  const double *dens;                // L_LSM: cell densities (ttc layout), else null
  double *dlo[3];                    // L_LSM: face density 0.5*(d(n)+d(n+1)) of the source block
                                     // at a non-wall low face (k_face_planes)
  int bcode[6];                      // boundary code of each face (control.cin), W,E,S,N,B,T
  int pface[6];                      // periodic face with no neighbour: 1 block alone along the
                                     // axis (copies onto itself), 2 partner block src[f]; else 0
  double *bcst;                      // exchange_bc receive planes: 3 components x 6 faces x bcplane
  long long bcplane;                 // elements per receive plane (the largest ttc plane)
  const double *oo[3];               // velocity predictor: u, v, w at the start of the time step
  const double *vis;                 // velocity predictor: cell viscosity (ttc layout)
  const double *inl;                 // west inlet (codes 7, 8, 12, 13): u, v, w planes of level-1
                                     // rows 0..ny+1 x planes 0..nz+1, row fastest; null = not set
  int inl_s1[3], inl_t1[3];          // per component the last row / plane the inlet writes (-1: none)
  double *wtau;                      // wall functions (codes 61-65): tau, tau2 of face f at
  long long wplane;                  // wtau + (2f or 2f+1)*wplane, ttc face planes; else null
};

// x / h.  When h is a power of two the multiplication by its reciprocal
// (exact) rounds the same exact quotient once, so the result is the IEEE
// quotient bit for bit; otherwise divide.
__device__ __forceinline__ double xdiv(double x, double h, double inv) { return inv != 0.0 ? x * inv : x / h; }

// x / b, bit for bit, from rb = RN(1/b) (the IEEE-rounded reciprocal,
// formed once per divisor) in five FP64 operations.  q0 = RN(x*rb) lies
// within 1.5 ulp of x/b; one correction q1 = RN(q0 + RN(x - b*q0)*rb) is a
// faithful quotient (error far below an ulp).  For faithful q1 the remainder
// x - b*q1 is exact (one FMA), and with rb within half an ulp of 1/b,
// RN(q1 + (x - b*q1)*rb) = RN(x/b) (Markstein's theorem: P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990).  The theorem needs no overflow
// or underflow: rb is 0 (plain division) unless 2^-100 <= b <= 2^100, and
// |x| outside [2^-700, 2^701) (zero, subnormal, huge, Inf, NaN) divides too.
// The range test reads the exponent field (integer pipe).
__device__ __forceinline__ bool rcp_range(double x) {
  const unsigned e = (unsigned)((unsigned long long)__double_as_longlong(x) >> 52) & 0x7ffu;
  return e - (1023u - 700u) <= 1400u;  // biased exponent in [323, 1723]
}
__device__ __forceinline__ double div_rcp(double x, double b, double rb) {
  if (rb == 0.0 || !rcp_range(x)) return x / b;
  const double q0 = x * rb;
  const double q1 = fma(fma(-b, q0, x), rb, q0);
  return fma(fma(-b, q1, x), rb, q1);
}
// div_rcp against the IEEE division, element by element (mf3d_selftest_divide).
__global__ void k_selftest_divide(const double *x, const double *b, const double *rb, long long n, double *q,
                                  double *qref) {
  pdl_wait();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  q[t] = div_rcp(x[t], b[t], rb[t]);
  qref[t] = x[t] / b[t];
}

// x / b on an axis: EXACT when b is a power of two and rb its exact inverse.
template <bool EXACT>
__device__ __forceinline__ double qdiv(double x, double b, double rb) {
  return EXACT ? x * rb : div_rcp(x, b, rb);
}

__device__ inline long long fidx(const BlkFld &F, int i, int j, int k) {
  // level-1 ghost-inclusive (i,j,k) -> 0-based ttc element
  return (long long)(i + F.pl - 1) + (long long)F.ti * ((long long)(j + F.pl - 1) + (long long)F.tj * (k + F.pl - 1));
}

// p := p + (pp - ppref) over isp-1..iep+1 (newsolv_mg.for:38-48), ppref = 0
// (the reference-pressure code is commented out, :28-36); pp is the level-1
// correction of the V-cycle.  Also zeroes the ghost shell of pp after
// reading it: the next V-cycle starts from pp = 0 (newsolv_mg.for:44) and its
// first red sweep never reads the interior, so the shell is all that must
// hold zeros.  One thread per pair of x-neighbours (i = 2h, 2h+1: compact
// index h in both colour arrays, so neighbouring lanes read neighbouring
// elements of each) and row j of the ghost-inclusive plane, marching up kch
// planes.
template <typename T>
__global__ void __launch_bounds__(kTile) k_add_correction(const BlkFld *__restrict__ fl,
                                                          const Tile *__restrict__ tiles,
                                                          const int *__restrict__ act, int kch) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  if (!act[fl[t.blk].dom]) return;
  const BlkFld F = fl[t.blk];
  const int nx = F.L1.nx, ny = F.L1.ny, nz = F.L1.nz, hp = F.L1.hp;
  const int HX = (nx + 3) / 2;  // pairs per ghost-inclusive row
  const int g = t.i0 + threadIdx.x;
  if (g >= HX * (ny + 2)) return;
  const int j = g / HX, h = g - j * HX;
  const int i0 = 2 * h, i1 = 2 * h + 1;
  const bool has1 = i1 <= nx + 1;
  T *__restrict__ phi = phi_of<T>(F.L1);
  double *__restrict__ P = F.p;
  const long long cs = F.L1.cstr, plane = (long long)(ny + 2) * hp;
  const long long fs = (long long)F.ti * F.tj;
  const bool jg = j == 0 || j == ny + 1;
  const int k1 = min(t.k0 + kch - 1, nz + 1);
  const long long e0 = (long long)j * hp + h;  // compact element of plane 0 without the colour term
  const long long f0 = fidx(F, i0, j, 0);
  const double ppref = 0.0;
  // batches of AC_U planes: every load of a batch is issued before its stores
  constexpr int AC_U = 4;
  for (int kb = t.k0; kb <= k1; kb += AC_U) {
    double q0[AC_U], q1[AC_U], v0[AC_U], v1[AC_U];
#pragma unroll
    for (int u = 0; u < AC_U; ++u) {
      const int k = kb + u;
      if (k > k1) break;
      const int c0 = (i0 + j + k + 1) & 1;
      const long long e = e0 + k * plane, f = f0 + k * fs;
      q0[u] = (double)phi[c0 * cs + e];
      v0[u] = P[f];
      if (has1) {
        q1[u] = (double)phi[(1 - c0) * cs + e];
        v1[u] = P[f + 1];
      }
    }
#pragma unroll
    for (int u = 0; u < AC_U; ++u) {
      const int k = kb + u;
      if (k > k1) break;
      const int c0 = (i0 + j + k + 1) & 1;
      const long long e = e0 + k * plane, f = f0 + k * fs;
      const bool kg = k == 0 || k == nz + 1;
      P[f] = (v0[u] + (q0[u] - ppref));
      if (i0 == 0 || i0 == nx + 1 || jg || kg) phi[c0 * cs + e] = (T)0;  // i0 = nx+1 when nx is odd
      if (has1) {
        P[f + 1] = (v1[u] + (q1[u] - ppref));
        if (i1 == nx + 1 || jg || kg) phi[(1 - c0) * cs + e] = (T)0;
      }
    }
  }
}

// exchange(4) + pbound on the face ghosts of p (exchange.for:2402-2490,
// exchange_bc.for, press.for:77-137): inter-block and periodic faces take
// the source block's adjacent interior value, wall faces mirror the first
// interior cell.  Only the interior tangential range: the path reads no
// other ghost of p.  Items per block: 2*(ny*nz + nx*nz + nx*ny).
__global__ void k_p_faces(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles, const int *__restrict__ act) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  if (!act[F.dom]) return;
  int q = t.i0 + threadIdx.x;
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

// exchange(1), (2), (3) after the final calvel (exchange.for:2-23 with
// nly = pl_ex; exchange_bc.for:16-320; the face unpack of exchange_smlvl,
// exchange.for:2402-2490): on every face that is not a physical wall, ghost
// layer ly = 0..nly of u, v and w over the interior tangential range takes
// the source block's value ly planes inside its facing boundary - low ghost
// (0-ly) from source plane n-ly, high ghost (n+1+ly) from source plane 1+ly.
// The velocity ranges of a face that has a source block are never cut short
// (localparameters.for:185-190 shortens them at walls only), so the same
// planes serve u, v and w.  Reads touch interior cells only (every edge
// exceeds nly), writes ghost cells only: one pass, no ordering.  Ghost edges
// and corners are not written.  Items per block: (nly+1) * 2*(ny*nz + nx*nz
// + nx*ny); `only` (may be null) as in k_calvel.
__global__ void k_vel_faces(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles,
                            const int *__restrict__ only, int nly) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  if (only && !only[F.dom]) return;
  int q = t.i0 + threadIdx.x;
  const int nx = F.nx, ny = F.ny, nz = F.nz;
  const int nyz = ny * nz, nxz = nx * nz, nxy = nx * ny;
  const int per_layer = 2 * (nyz + nxz + nxy);
  const int ly = q / per_layer;
  if (ly > nly) return;
  q -= ly * per_layer;
  int f, a, b;
  if (q < 2 * nyz) { f = q / nyz; q -= f * nyz; a = q % ny + 1; b = q / ny + 1; }
  else if ((q -= 2 * nyz) < 2 * nxz) { f = 2 + q / nxz; q -= (f - 2) * nxz; a = q % nx + 1; b = q / nx + 1; }
  else { q -= 2 * nxz; f = 4 + q / nxy; q -= (f - 4) * nxy; a = q % nx + 1; b = q / nx + 1; }
  if (F.wall[f]) return;
  const BlkFld &S = fl[F.src[f]];
  int gi, gj, gk, si, sj, sk;  // ghost cell; source cell (in the source block)
  switch (f) {
    case 0: gi = -ly; gj = a; gk = b; si = S.nx - ly; sj = a; sk = b; break;
    case 1: gi = nx + 1 + ly; gj = a; gk = b; si = 1 + ly; sj = a; sk = b; break;
    case 2: gi = a; gj = -ly; gk = b; si = a; sj = S.ny - ly; sk = b; break;
    case 3: gi = a; gj = ny + 1 + ly; gk = b; si = a; sj = 1 + ly; sk = b; break;
    case 4: gi = a; gj = b; gk = -ly; si = a; sj = b; sk = S.nz - ly; break;
    default: gi = a; gj = b; gk = nz + 1 + ly; si = a; sj = b; sk = 1 + ly; break;
  }
  const long long g = fidx(F, gi, gj, gk), s = fidx(S, si, sj, sk);
  F.u[g] = S.u[s];
  F.v[g] = S.v[s];
  F.w[g] = S.w[s];
}

// exchange(op) on the fields as a copy map (the host replays exchange_bc,
// exchange_smlvl's corners, edges and faces, and pbound for the pressure, on
// cell tokens: exchange.for:2-23, 343-2498; exchange_bc.for:2-841; press.for:
// 77-137).  Each pair sets a ghost cell of component comp (0 u, 1 v, 2 w, 3 p)
// of block dblk from the pre-exchange value of cell soff of block sblk.
// Pairs whose source is itself written come first; k_fx_stage reads their
// sources, then k_fx_apply writes every pair.  `only` (may be null) as in
// k_calvel.
struct FxCopy {
  unsigned doff, soff;
  unsigned short dblk, sblk;
  int comp;
};
__device__ __forceinline__ double *fx_field(const BlkFld &F, int comp) {
  return comp == 0 ? F.u : comp == 1 ? F.v : comp == 2 ? F.w : F.p;
}
// the pre-exchange value a pair copies: from `prev` (slot soff) when comp
// carries bit 8 (a chained source, saved by k_fx_evolve), else the field
__device__ __forceinline__ double fx_source(const BlkFld *fl, const FxCopy &x, const double *prev) {
  return (x.comp & 8) ? prev[x.soff] : fx_field(fl[x.sblk], x.comp & 7)[x.soff];
}
__global__ void k_fx_stage(const BlkFld *__restrict__ fl, const FxCopy *__restrict__ c, long long nstaged,
                           const int *__restrict__ only, double *__restrict__ buf, const double *__restrict__ prev) {
  pdl_wait();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nstaged) return;
  const FxCopy x = c[t];
  if (only && !only[fl[x.dblk].dom]) return;
  buf[t] = fx_source(fl, x, prev);
}
__global__ void k_fx_apply(const BlkFld *__restrict__ fl, const FxCopy *__restrict__ c, long long n,
                           long long nstaged, const int *__restrict__ only, const double *__restrict__ buf,
                           const double *__restrict__ prev) {
  pdl_wait();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const FxCopy x = c[t];
  if (only && !only[fl[x.dblk].dom]) return;
  const double v = t < nstaged ? buf[t] : fx_source(fl, x, prev);
  fx_field(fl[x.dblk], x.comp & 7)[x.doff] = v;
}

// Face planes used by the fused calvel/calmas kernel, filled once per solve:
// lo[a] = the velocity component normal to the block's low face on that face
// when it is a wall (the caller's boundary value, never rewritten by calvel),
// else the source block's ustar on its last face (exchange(1..3) hands over
// that block's u); hi[a] = the caller's velocity on a high wall face
// (localparameters.for:185-190 stops calvel one face short there).
// walls_given: the wall values are already in lo/hi (the host entry point
// copies them there straight from the caller's arrays) and are left alone.
__global__ void k_face_planes(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles, int walls_given) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  int q = t.i0 + threadIdx.x;
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
    if (!walls_given) F.lo[ax][o] = vel[e];
  } else {
    const BlkFld &S = fl[F.src[fl0]];
    const double *st = ax == 0 ? S.ustar : ax == 1 ? S.vstar : S.wstar;
    long long e = ax == 0 ? fidx(S, S.nx, a, b) : ax == 1 ? fidx(S, a, S.ny, b) : fidx(S, a, b, S.nz);
    F.lo[ax][o] = st[e];
    if (F.dens) {  // the density calvel divides by on that face, in the source block (press.for:152-190)
      const long long s1 = ax == 0 ? 1 : ax == 1 ? (long long)S.ti : (long long)S.ti * S.tj;
      F.dlo[ax][o] = 0.5 * (S.dens[e] + S.dens[e + s1]);
    }
  }
  // high face
  long long e = ax == 0 ? fidx(F, nx, a, b) : ax == 1 ? fidx(F, a, ny, b) : fidx(F, a, b, nz);
  if (!(F.wall[fh] && walls_given)) F.hi[ax][o] = F.wall[fh] ? vel[e] : 0.0;
}

// ---------------------------------------------------------------------------
// boundu / boundv / boundw after the loop (newsolv_mg.for:86-88), and the
// full periodic planes of exchange(1..3) they need.  All three velocity
// components in each launch (independent arrays).  Local indices: 1..n
// interior, 1-pl..n+pl ghost-inclusive.
// ---------------------------------------------------------------------------
// The component's range along an axis (localparameters.for:185-190): the
// normal component stops one face short at a high wall.
__device__ inline int comp_end(const BlkFld &F, int comp, int ax) {
  const int n = ax == 0 ? F.nx : ax == 1 ? F.ny : F.nz;
  return n - ((comp == ax && F.wall[2 * ax + 1]) ? 1 : 0);
}
__device__ inline double *comp_field(const BlkFld &F, int comp) { return comp == 0 ? F.u : comp == 1 ? F.v : F.w; }
__device__ inline long long fidx_ax(const BlkFld &F, int ax, int a, int s, int t) {
  return ax == 0 ? fidx(F, a, s, t) : ax == 1 ? fidx(F, s, a, t) : fidx(F, s, t, a);
}

// One walk of exchange_bc (exchange_bc.for:16-838, every block on one
// rank) over the two faces of axis `ax`, layer ly, full ghost-inclusive
// planes.  mode 0: the first walk's self-copies of a block alone along the
// axis, ghost(s0-1-ly) = plane(e0-ly), ghost(e0+1+ly) = plane(s0+ly) (its
// packs are overwritten by the second walk's); mode 1: the second walk -
// the self-copies again and the packs into the partner's receive planes;
// mode 2: the third walk, ghost planes from the receive planes.  Launched
// per layer as walk 1 for x, y, z, walk 2 for x, y, z, walk 3 for x, y, z:
// a block's faces in the reference's W, E, S, N, B, T order.  Reads and
// writes of one launch never meet (interior planes or receive planes
// against ghost planes).  Items per block: 3 * 2 * n1 * n2 (ttc extents of
// the other two axes).  Skipped after a diverged solve.
__global__ void k_bc_walk(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles,
                          const DomState *__restrict__ ds, int ax, int ly, int mode, int only) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  if (ds[F.dom].rmax > 100.0) return;
  const int pl = F.pl;
  const int m1 = (ax == 0 ? F.ny : F.nx) + 2 * pl, m2 = (ax == 2 ? F.ny : F.nz) + 2 * pl;
  int q = t.i0 + threadIdx.x;
  const int plane = m1 * m2;
  if (q >= 6 * plane) return;
  const int comp = q / (2 * plane);
  if (only >= 0 && comp != only) return;  // one component (boundu, boundv or boundw alone)
  q -= comp * 2 * plane;
  const int side = q / plane;
  q -= side * plane;
  const int sl = q % m1 + 1 - pl, tl = q / m1 + 1 - pl;  // local coordinates of the plane cell
  const int f = 2 * ax + side;
  const int pf = F.pface[f];
  if (!pf) return;
  double *fi = comp_field(F, comp);
  const int s0 = 1, e0 = comp_end(F, comp, ax);
  const long long g = fidx_ax(F, ax, side ? e0 + 1 + ly : s0 - 1 - ly, sl, tl);
  if (mode == 2) {
    if (pf == 2) fi[g] = F.bcst[((long long)comp * 6 + f) * F.bcplane + q];
    return;
  }
  if (pf == 1) {
    fi[g] = fi[fidx_ax(F, ax, side ? s0 + ly : e0 - ly, sl, tl)];
  } else if (mode == 1) {
    const BlkFld &P = fl[F.src[f]];
    P.bcst[((long long)comp * 6 + (f ^ 1)) * P.bcplane + q] = fi[fidx_ax(F, ax, side ? e0 - ly : s0 + ly, sl, tl)];
  }
}

// The faces of axis `ax` without a neighbour, layer ly, by their code
// (bounds.for:2-916): over the component's ranges widened by one cell,
//   normal component: wall -> 0; symmetry -> 0 on y and z faces;
//   tangential: wall -> -(the cell ly inside); symmetry -> + on y and z faces;
//   inflow (1) on the west: u = ubulk, v = w = 0; on the bottom: u = v = 0,
//     w = 1.1 (bounds.for:42-53, 374-377, 662-665; 226-229, 536-539, 873-876);
//   outflow (2) on the east with alfabc = 1: every layer copies the last
//     face ie (bounds.for:136-170, 444-470);
//   convective outflow (21) on the east with alfabc = 1, when the velocity
//     predictor has bound the start-of-step velocities: oo(ie+1+ly) -
//     dt*alfapr*(oo(ie+1+ly) - oo(ie))/dx (the same branches);
// x-face symmetry, periodic faces and codes without a branch write nothing.
// Launched per layer for x, y, z (the reference's W, E, S, N, B, T).
// Skipped after a diverged solve.
// log_law (log_law.for:2-310, codes 61 smooth and 62 rough) and
// wall_function (wall_function.for:2-250, the power laws of 63, 64, 65) of
// the two faces of axis `ax` with a wall-function code: per cell of the
// face's plane (the cell ranges widened by one) the tangential speed of the
// first cell layer,
//   vtan = sqrt(|uc*uc + vc*vc + wc*wc - vnor*vnor + 1e-30|),
// cell-centred uc, vc, wc and vnor along the inward normal, and the wall
// stress tau, tau2 = tau/vtan into the face's planes.  log_law keeps the old
// tau2 where y+ is below 11.067 (11.63 on the top face).  The smooth-wall
// iteration records ERR_WALL_LAW where it does not converge in 10 steps
// (the reference prints and stops).  Transcendentals (sqrt, log, pow) are
// CUDA's.  Launched over the bounds tiles of the axis (before the faces'
// k_bound_faces of the same layer and component).
__global__ void k_wall_law(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles,
                           const DomState *__restrict__ ds, int ax, double re, double fric, int *err) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  if (ds[F.dom].rmax > 100.0 || !F.wtau) return;
  const int pl = F.pl;
  const int m1 = (ax == 0 ? F.ny : F.nx) + 2 * pl, m2 = (ax == 2 ? F.ny : F.nz) + 2 * pl;
  int q = t.i0 + threadIdx.x;
  const int plane = m1 * m2;
  if (q >= 2 * plane) return;
  const int side = q / plane;
  q -= side * plane;
  const int sl = q % m1 + 1 - pl, tl = q / m1 + 1 - pl;
  const int f = 2 * ax + side;
  const int code = F.bcode[f];
  if (!F.wall[f] || code < 61) return;
  const int n1 = ax == 0 ? F.ny : F.nx, n2 = ax == 2 ? F.ny : F.nz;
  if (sl < 0 || sl > n1 + 1 || tl < 0 || tl > n2 + 1) return;
  const int fix = side ? (ax == 0 ? F.nx : ax == 1 ? F.ny : F.nz) : 1;
  const int i = ax == 0 ? fix : sl, j = ax == 0 ? sl : ax == 1 ? fix : tl, k = ax == 2 ? fix : tl;
  const double rrey = 1.0 / re, small = 1.e-30, kappa = 0.41, Ecte = 9.0;
  const double delta = F.h[ax][1];
  const double nx = ax == 0 ? (side ? -1.0 : 1.0) : 0.0, ny = ax == 1 ? (side ? -1.0 : 1.0) : 0.0,
               nz = ax == 2 ? (side ? -1.0 : 1.0) : 0.0;
  const long long c = fidx(F, i, j, k);
  const long long sy = F.ti, sz = (long long)F.ti * F.tj;
  const double uc = 0.5 * (F.u[c] + F.u[c - 1]);
  const double vc = 0.5 * (F.v[c] + F.v[c - sy]);
  const double wc = 0.5 * (F.w[c] + F.w[c - sz]);
  const double vnor = nx * uc + ny * vc + nz * wc;
  const double vtan = sqrt(fabs(uc * uc + vc * vc + wc * wc - vnor * vnor + small));
  const long long e = (long long)(tl + pl - 1) * m1 + (sl + pl - 1);
  double *tau = F.wtau + 2 * f * F.wplane, *tau2 = tau + F.wplane;
  if (code >= 63) {
    // the 1/6, 1/7 and 1/8 power laws (wall_function.for:34-49)
    const double aaa = 8.3, bbb = code == 63 ? 0.1666666666 : code == 64 ? 0.1428571429 : 0.125;
    const double const1 = 0.5 * (1. - bbb) * pow(aaa, (1. + bbb) / (1. - bbb));
    const double const2 = (1. + bbb) / aaa;
    const double const3 = pow(aaa, 2. / (1. - bbb));
    const double const4 = 2. / (1. + bbb);
    const double dycell = 2. * delta, rycell = 1. / dycell;
    const double vtankr = 0.5 * rrey * rycell * const3;
    const double dvtan = vtankr - vtan;
    const double sub = fmax(copysign(1., dvtan), 0.);
    const double tausub = rrey * vtan / delta;
    const double taupow = pow(const1 * pow(rrey * rycell, 1. + bbb) + (const2 * pow(rrey * rycell, bbb)) * vtan, const4);
    tau[e] = (sub * tausub + (1. - sub) * taupow);
    tau2[e] = tau[e] / vtan;
    return;
  }
  double ustar = 0.0, yplus = 0.0;
  if (code == 62) {
    ustar = kappa * vtan / log(30.0 * delta / fric);
    yplus = delta * ustar / rrey;
  } else if (code == 61) {
    double conv = 1., ustarold;
    int icont = 0;
    const int tkmax = 10;
    ustar = 1.;
    while (conv > 1.e-3 && icont < tkmax) {
      ++icont;
      ustarold = ustar;
      yplus = fmax(1.0000001, delta * ustar / rrey);
      ustar = vtan * kappa / log(Ecte * yplus);
      conv = fabs((ustar - ustarold) / ustar);
    }
    if (icont == tkmax) atomicExch(err, ERR_WALL_LAW);
  }
  if (yplus < (f == 5 ? 11.63 : 11.067)) {
    tau[e] = rrey * vtan / delta;
  } else {
    tau[e] = ustar * ustar;  // ustar**2.0
    tau2[e] = tau[e] / vtan;
  }
}

__global__ void k_bound_faces(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles,
                              const DomState *__restrict__ ds, int ax, int ly, double ubulk, int alfabc,
                              int only, double dt, double alfapr) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  if (ds[F.dom].rmax > 100.0) return;
  const int pl = F.pl;
  const int m1 = (ax == 0 ? F.ny : F.nx) + 2 * pl, m2 = (ax == 2 ? F.ny : F.nz) + 2 * pl;
  int q = t.i0 + threadIdx.x;
  const int plane = m1 * m2;
  if (q >= 6 * plane) return;
  const int comp = q / (2 * plane);
  if (only >= 0 && comp != only) return;  // one component (boundu, boundv or boundw alone)
  q -= comp * 2 * plane;
  const int side = q / plane;
  q -= side * plane;
  const int sl = q % m1 + 1 - pl, tl = q / m1 + 1 - pl;
  const int f = 2 * ax + side;
  if (!F.wall[f]) return;
  const int code = F.bcode[f];
  const bool normal = comp == ax;
  // 1 constant cv, 2 -mirror, 3 +mirror, 4 copy of the last face,
  // 5 convective outflow, 6 the inlet plane, 7 wall-function update of the
  // first cell (layer 0), 8 wall-function mirror (deeper layers)
  int mode = 0;
  double cv = 0.0;
  if (code >= 61 && F.wtau) mode = normal ? 1 : ly == 0 ? 7 : 8;
  else if (code == 4) mode = normal ? 1 : 2;
  else if (code == 3 && ax != 0) mode = normal ? 1 : 3;
  else if (code == 1 && side == 0 && ax != 1) {  // inflow: west u = ubulk, bottom w = 1.1, the rest 0
    mode = 1;
    cv = ax == 0 ? (comp == 0 ? ubulk : 0.0) : (comp == 2 ? 1.1 : 0.0);
  } else if (code == 2 && ax == 0 && side == 1 && alfabc == 1) mode = 4;  // outflow: u(ie+1+ly) = u(ie)
  else if (code == 21 && ax == 0 && side == 1 && alfabc == 1 && F.oo[comp]) mode = 5;  // convective outflow
  else if (f == 0 && (code == 7 || code == 8 || code == 12 || code == 13)) {
    // the inlets (bounds.for:55-135, 397-438, 686-730): each component from
    // its inlet plane where it has one; code 12 sets v = w = 0 (:374-377,
    // 662-665), 13 leaves them
    if (F.inl && F.inl_s1[comp] >= 0) mode = 6;
    else if (comp != 0 && code == 12) mode = 1;
  }
  if (!mode) return;
  // the widened ranges of the other two axes: 0 .. end+1
  const int as = ax == 0 ? 1 : 0, at = ax == 2 ? 1 : 2;
  if (sl < 0 || sl > comp_end(F, comp, as) + 1 || tl < 0 || tl > comp_end(F, comp, at) + 1) return;
  double *fi = comp_field(F, comp);
  const int s0 = 1, e0 = comp_end(F, comp, ax);
  const long long g = fidx_ax(F, ax, side ? e0 + 1 + ly : s0 - 1 - ly, sl, tl);
  if (mode == 6) {
    const long long pn = (long long)(F.ny + 2) * (F.nz + 2);
    if (sl <= F.inl_s1[comp] && tl <= F.inl_t1[comp]) fi[g] = F.inl[comp * pn + (long long)tl * (F.ny + 2) + sl];
    return;
  }
  if (dt < 0.0) {  // the solve's own dt and alfapr
    dt = ds[F.dom].dt;
    alfapr = ds[F.dom].alfapr;
  }
  if (mode == 7) {
    // F = sign(tau2*c(first)/h, -c(first)), h along the component's own
    // axis; c(first) += F*alfapr*dt; c(ghost 0) = -c(first)
    const long long first = fidx_ax(F, ax, side ? e0 : s0, sl, tl);
    const double t2 = F.wtau[(2 * f + 1) * F.wplane + (long long)(tl + pl - 1) * m1 + (sl + pl - 1)];
    double c = fi[first];
    double fw = t2 * c / F.h[comp][1];
    fw = copysign(fabs(fw), -c);
    c = c + fw * alfapr * dt;
    fi[first] = c;
    fi[g] = -c;
    return;
  }
  if (mode == 8) {  // deeper layers: minus the first cell (u on the S, N, B faces: the cell ly inside)
    const int src = (comp == 0 && f != 5) ? (side ? e0 - ly : s0 + ly) : (side ? e0 : s0);
    fi[g] = -fi[fidx_ax(F, ax, src, sl, tl)];
    return;
  }
  if (mode == 5) {  // oo(ie+1+ly) - dt*alfapr*(oo(ie+1+ly) - oo(ie))/dx, from the start-of-step velocity
    const double *oo = F.oo[comp];
    const double og = oo[g], oe = oo[fidx_ax(F, ax, e0, sl, tl)];
    fi[g] = og - dt * alfapr * (og - oe) / F.h[0][1];
    return;
  }
  const int src = mode == 4 ? e0 : side ? e0 - ly : s0 + ly;
  const double m = fi[fidx_ax(F, ax, src, sl, tl)];
  fi[g] = mode == 1 ? cv : mode == 2 ? -m : m;
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
__global__ void __launch_bounds__(OZ_TX *OZ_RJ) k_calvel_calmas(const BlkFld *__restrict__ fl,
                                                               const Tile *__restrict__ tiles,
                                                               const DomState *__restrict__ ds,
                                                               const int *__restrict__ act,
                                                               unsigned long long *__restrict__ rmax_slot,
                                                               int write_su) {
  pdl_wait();
  __shared__ double red[OZ_RJ];
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  if (!act[F.dom]) return;
  const double dt = ds[F.dom].dt, alfapr = ds[F.dom].alfapr, dtinv = ds[F.dom].dtinv;
  const double dta = dt * alfapr;
  T *__restrict__ rhs1 = rhs_of<T>(F.L1);
  double *__restrict__ SU = write_su ? F.su : nullptr;
  const int nx = F.nx, ny = F.ny, nz = F.nz;
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  const bool in = i <= nx && j <= ny;
  const int ic = in ? i : 1, jc = in ? j : 1;  // clamped indices keep every load in bounds
  const long long sy = F.ti, sz = (long long)F.ti * F.tj;
  const double *__restrict__ p = F.p;
  const double *__restrict__ US = F.ustar;
  const double *__restrict__ VS = F.vstar;
  const double *__restrict__ WS = F.wstar;
  const double *__restrict__ DZ = F.df[2];
  const double *__restrict__ HZ = F.h[2];
  const double ix = F.pinv[0], iy = F.pinv[1], iz = F.pinv[2];
  const double hx = F.h[0][ic], hy = F.h[1][jc];
  const double dxe = F.df[0][ic], dxw = F.df[0][ic - 1];
  const double dyn = F.df[1][jc], dys = F.df[1][jc - 1];
  const bool ewall = F.wall[1], nwall = F.wall[3], twall = F.wall[5];
  const bool wwall = F.wall[0], swall = F.wall[2], bwall = F.wall[4];
  const int k1 = min(t.k0 + OZ_KCH - 1, nz);
  double vmax = 0.0;
  // w on the face below plane k0, carried up the march
  double wb;
  {
    const int k = t.k0;
    const long long c = fidx(F, ic, jc, k);
    if (k == 1) {
      const double lo = F.lo[2][(jc - 1) * nx + (ic - 1)];
      wb = bwall ? lo : (lo - xdiv(dta * (p[c] - p[c - sz]), F.df[2][0], iz));
    } else {
      wb = (WS[c - sz] - xdiv(dta * (p[c] - p[c - sz]), DZ[k - 1], iz));
    }
  }
  for (int k = t.k0; k <= k1; ++k) {
    const long long c = fidx(F, ic, jc, k);
    const double pc = p[c];
    // east face of this cell; the west face is the east face of the cell to the
    // left (the lane before), formed from the same operands
    double ue;
    if (ic == nx && ewall) ue = F.hi[0][(k - 1) * ny + (jc - 1)];
    else ue = (US[c] - xdiv(dta * (p[c + 1] - pc), dxe, ix));
    const double ul = __shfl_up_sync(0xffffffffu, ue, 1);
    double uw;
    if (ic == 1) {
      const double lo = F.lo[0][(k - 1) * ny + (jc - 1)];
      uw = wwall ? lo : (lo - xdiv(dta * (pc - p[c - 1]), dxw, ix));
    } else if (threadIdx.x > 0) {
      uw = ul;
    } else {
      uw = (US[c - 1] - xdiv(dta * (pc - p[c - 1]), dxw, ix));
    }
    double vn, vs, wt;
    if (jc == ny && nwall) vn = F.hi[1][(k - 1) * nx + (ic - 1)];
    else vn = (VS[c] - xdiv(dta * (p[c + sy] - pc), dyn, iy));
    if (jc == 1) {
      const double lo = F.lo[1][(k - 1) * nx + (ic - 1)];
      vs = swall ? lo : (lo - xdiv(dta * (pc - p[c - sy]), dys, iy));
    } else {
      vs = (VS[c - sy] - xdiv(dta * (pc - p[c - sy]), dys, iy));
    }
    if (k == nz && twall) wt = F.hi[2][(jc - 1) * nx + (ic - 1)];
    else wt = (WS[c] - xdiv(dta * (p[c + sz] - pc), DZ[k], iz));
    const double hz = HZ[k];
    const double fact = (xdiv(ue - uw, hx, ix) + xdiv(vn - vs, hy, iy) + xdiv(wt - wb, hz, iz));
    wb = wt;  // the top face of plane k is the bottom face of plane k+1
    if (!in) continue;
    const double su = xdiv(fact, dt, dtinv);
    rhs1[cell_off(F.L1, i, j, k)] = (T)su;
    if (SU) SU[c] = su;
    double f1 = fabs(fact * hx * hy * hz);
    if (!(f1 == f1)) f1 = __longlong_as_double(0x7ff0000000000000LL);  // NaN -> +Inf (flagged)
    vmax = vmax > f1 ? vmax : f1;
  }
  // CTA max: warp shuffles, shared memory, one atomic per CTA
  for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
  if (threadIdx.x == 0) red[threadIdx.y] = vmax;
  __syncthreads();
  if (threadIdx.y == 0) {
    double v = threadIdx.x < OZ_RJ ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0 && v > 0.0) atomic_max_nonneg(rmax_slot + F.dom, v);
  }
}

// Fused calvel + calmas under L_LSM (variable density; uniform spacing):
// every face velocity divides by its face density last,
//   u(i) = ustar(i) - ((dt*alfapr*(p(i+1)-p(i)))/dx)/(0.5*(dens(i)+dens(i+1)))
// (press.for:152-190), and the level-1 rhs is sup = fact*dx*dy*dz/dt
// (press.for:51-53, copied by mgkcyc at mgsolver.for:256-261).  A block
// face that is not a wall takes the source block's ustar and face density
// (k_face_planes).  One thread per (i, j) column, marching up OZ_KCH planes;
// the west face comes from the lane to the left and the bottom face from
// the plane below (formed from the same operands), so a cell forms four
// face velocities, not six.  rmax as in k_calvel_calmas.
__global__ void __launch_bounds__(OZ_TX *OZ_RJ) k_calvel_calmas_lsm(const BlkFld *__restrict__ fl,
                                                                   const Tile *__restrict__ tiles,
                                                                   const DomState *__restrict__ ds,
                                                                   const int *__restrict__ act,
                                                                   unsigned long long *__restrict__ rmax_slot,
                                                                   int write_su) {
  pdl_wait();
  __shared__ double red[OZ_RJ];
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  if (!act[F.dom]) return;
  const double dt = ds[F.dom].dt, alfapr = ds[F.dom].alfapr;
  const double dta = dt * alfapr;
  double *__restrict__ rhs1 = rhs_of<double>(F.L1);
  double *__restrict__ SU = write_su ? F.su : nullptr;
  const int nx = F.nx, ny = F.ny, nz = F.nz;
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  const bool in = i <= nx && j <= ny;
  const int ic = in ? i : 1, jc = in ? j : 1;
  const long long sy = F.ti, sz = (long long)F.ti * F.tj;
  const double *__restrict__ p = F.p;
  const double *__restrict__ D = F.dens;
  const double ix = F.pinv[0], iy = F.pinv[1], iz = F.pinv[2];
  const double hx = F.h[0][ic], hy = F.h[1][jc];
  const double dx = F.df[0][ic], dy = F.df[1][jc];
  const bool ewall = F.wall[1], nwall = F.wall[3], twall = F.wall[5];
  const bool wwall = F.wall[0], swall = F.wall[2], bwall = F.wall[4];
  const int k1 = min(t.k0 + OZ_KCH - 1, nz);
  double vmax = 0.0;
  double wcarry = 0.0;  // the top face of the previous plane: this plane's bottom face
  for (int k = t.k0; k <= k1; ++k) {
    const long long c = fidx(F, ic, jc, k);
    const double pc = p[c], dc = D[c];
    const double dz = F.df[2][k], hz = F.h[2][k];
    double ue, uw, vn, vs, wt, wb;
    if (ic == nx && ewall) ue = F.hi[0][(k - 1) * ny + (jc - 1)];
    else ue = (F.ustar[c] - xdiv(dta * (p[c + 1] - pc), dx, ix) / (0.5 * (dc + D[c + 1])));
    // the west face is the east face of the lane to the left (same operands)
    const double ul = __shfl_up_sync(0xffffffffu, ue, 1);
    if (ic == 1) {
      const int o = (k - 1) * ny + (jc - 1);
      uw = wwall ? F.lo[0][o] : (F.lo[0][o] - xdiv(dta * (pc - p[c - 1]), dx, ix) / F.dlo[0][o]);
    } else if (threadIdx.x > 0) {
      uw = ul;
    } else {
      uw = (F.ustar[c - 1] - xdiv(dta * (pc - p[c - 1]), dx, ix) / (0.5 * (D[c - 1] + dc)));
    }
    if (jc == ny && nwall) vn = F.hi[1][(k - 1) * nx + (ic - 1)];
    else vn = (F.vstar[c] - xdiv(dta * (p[c + sy] - pc), dy, iy) / (0.5 * (dc + D[c + sy])));
    if (jc == 1) {
      const int o = (k - 1) * nx + (ic - 1);
      vs = swall ? F.lo[1][o] : (F.lo[1][o] - xdiv(dta * (pc - p[c - sy]), dy, iy) / F.dlo[1][o]);
    } else {
      vs = (F.vstar[c - sy] - xdiv(dta * (pc - p[c - sy]), dy, iy) / (0.5 * (D[c - sy] + dc)));
    }
    if (k == nz && twall) wt = F.hi[2][(jc - 1) * nx + (ic - 1)];
    else wt = (F.wstar[c] - xdiv(dta * (p[c + sz] - pc), dz, iz) / (0.5 * (dc + D[c + sz])));
    if (k == 1) {
      const int o = (jc - 1) * nx + (ic - 1);
      wb = bwall ? F.lo[2][o] : (F.lo[2][o] - xdiv(dta * (pc - p[c - sz]), dz, iz) / F.dlo[2][o]);
    } else if (k > t.k0) {
      wb = wcarry;
    } else {
      wb = (F.wstar[c - sz] - xdiv(dta * (pc - p[c - sz]), dz, iz) / (0.5 * (D[c - sz] + dc)));
    }
    wcarry = wt;
    const double fact = (xdiv(ue - uw, hx, ix) + xdiv(vn - vs, hy, iy) + xdiv(wt - wb, hz, iz));
    if (!in) continue;
    const double sup = fact * hx * hy * hz / dt;
    rhs1[cell_off(F.L1, i, j, k)] = sup;
    if (SU) SU[c] = sup;
    double f1 = fabs(fact * hx * hy * hz);
    if (!(f1 == f1)) f1 = __longlong_as_double(0x7ff0000000000000LL);  // NaN -> +Inf (flagged)
    vmax = vmax > f1 ? vmax : f1;
  }
  for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
  if (threadIdx.x == 0) red[threadIdx.y] = vmax;
  __syncthreads();
  if (threadIdx.y == 0) {
    double v = threadIdx.x < OZ_RJ ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0 && v > 0.0) atomic_max_nonneg(rmax_slot + F.dom, v);
  }
}

// The same fused calvel + calmas with its operands staged by TMA.  Per
// plane a CTA (32 x OZ_RJ cells) needs p over its cells and a one-cell ring
// (plane k, and plane k+1 for the top faces), ustar over its cells and the
// column to the west, vstar over its cells and the row to the south, and
// wstar over its cells; one thread issues the four box loads of a plane
// CV_PD planes ahead into a ring of CV_NS slots.  Boxes start at the even
// field column X = (first cell's column - 1) rounded down, so their x origin
// is 16-byte aligned whatever the ghost width; CV_W = 36 columns cover the
// tile and its ring for either parity.  Each plane's p box is loaded once
// and serves as the upper plane of the plane below.  Arithmetic, operand
// order and the face planes are those of k_calvel_calmas.
constexpr int CV_PD = 2;           // planes in flight ahead of the computed one
constexpr int CV_NS = CV_PD + 1;   // slots: planes k .. k+CV_PD
constexpr int CV_MINB = 6;         // resident CTAs per SM the kernel is built for
constexpr int CV_W = 36;
struct CvShape {
  static constexpr int PR = OZ_RJ + 2, UR = OZ_RJ, VR = OZ_RJ + 1, WR = OZ_RJ;  // box rows
  static constexpr int PB = (PR * CV_W * 8 + 127) / 128 * 128, UB = (UR * CV_W * 8 + 127) / 128 * 128;
  static constexpr int VB = (VR * CV_W * 8 + 127) / 128 * 128, WB = (WR * CV_W * 8 + 127) / 128 * 128;
  static constexpr int STAGE = PB + UB + VB + WB;
};

constexpr int CV_TY = 4, CV_CR = OZ_RJ / CV_TY;  // 32 x CV_TY threads, CV_CR consecutive rows each

// x / b for k_calvel_calmas_tma's march: on an EXACT axis the product with
// the exact inverse; otherwise Markstein's correction of div_rcp without its
// branch - `bad` records an x outside the range where the correction is the
// IEEE quotient (zero, subnormal, huge, non-finite), and the tile then
// divides again (cv_cells_divide).
template <bool EXACT>
__device__ __forceinline__ double qdv(double x, double b, double rb, bool &bad) {
  if (EXACT) return x * rb;
  bad |= !rcp_range(x);
  const double q0 = x * rb;
  const double q1 = fma(fma(-b, q0, x), rb, q0);
  return fma(fma(-b, q1, x), rb, q1);
}

// The cells of one thread of k_calvel_calmas_tma (column i, rows j0 ..
// j0+CV_CR-1, planes k0..k1) from global memory with IEEE division
// throughout - calvel's six face velocities, calmas' divergence in the
// reference's order (press.for:38-67, 139-198) - writing su and returning
// the rmax contribution.  The tile's fallback where the march met an operand
// outside Markstein's range, or a divisor without its reciprocal.
template <typename T>
__device__ double cv_cells_divide(const BlkFld &F, int i, int j0, int k0, int k1, double dt, double dta, T *rhs1,
                                  double *SU) {
  const int nx = F.nx, ny = F.ny, nz = F.nz;
  const long long sy = F.ti, sz = (long long)F.ti * F.tj;
  const long long ps1 = (long long)(F.L1.ny + 2) * F.L1.hp;
  const double *p = F.p;
  double vmax = 0.0;
  if (i > nx) return vmax;
  for (int m = 0; m < CV_CR; ++m) {
    const int j = j0 + m;
    if (j > ny) break;
    for (int k = k0; k <= k1; ++k) {
      const long long c = fidx(F, i, j, k);
      const double pc = p[c];
      double ue, uw, vn, vs, wt, wb;
      if (i == nx && F.wall[1]) ue = F.hi[0][(k - 1) * ny + (j - 1)];
      else ue = (F.ustar[c] - dta * (p[c + 1] - pc) / F.df[0][i]);
      if (i == 1) {
        const double lo = F.lo[0][(k - 1) * ny + (j - 1)];
        uw = F.wall[0] ? lo : (lo - dta * (pc - p[c - 1]) / F.df[0][0]);
      } else {
        uw = (F.ustar[c - 1] - dta * (pc - p[c - 1]) / F.df[0][i - 1]);
      }
      if (j == ny && F.wall[3]) vn = F.hi[1][(k - 1) * nx + (i - 1)];
      else vn = (F.vstar[c] - dta * (p[c + sy] - pc) / F.df[1][j]);
      if (j == 1) {
        const double lo = F.lo[1][(k - 1) * nx + (i - 1)];
        vs = F.wall[2] ? lo : (lo - dta * (pc - p[c - sy]) / F.df[1][0]);
      } else {
        vs = (F.vstar[c - sy] - dta * (pc - p[c - sy]) / F.df[1][j - 1]);
      }
      if (k == nz && F.wall[5]) wt = F.hi[2][(j - 1) * nx + (i - 1)];
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
      rhs1[(((i + j + k + 1) & 1) ? F.L1.cstr : 0) + k * ps1 + (long long)j * F.L1.hp + (i >> 1)] = (T)su;
      if (SU) SU[c] = su;
      double f1 = fabs(fact * hx * hy * hz);
      if (!(f1 == f1)) f1 = __longlong_as_double(0x7ff0000000000000LL);  // NaN -> +Inf (flagged)
      vmax = vmax > f1 ? vmax : f1;
    }
  }
  return vmax;
}

// UMASK bit a: axis a of every block is uniform with a power-of-two spacing
// (x/h is x*(1/h) there); other axes divide through div_rcp.
template <typename T, int UMASK>
__global__ void __launch_bounds__(OZ_TX *CV_TY, CV_MINB) k_calvel_calmas_tma(const BlkFld *__restrict__ fl,
                                                                   const Tile *__restrict__ tiles,
                                                                   const DomState *__restrict__ ds,
                                                                   const int *__restrict__ act,
                                                                   unsigned long long *__restrict__ rmax_slot,
                                                                   int write_su, int kch, int *__restrict__ err) {
  pdl_wait();
  using S = CvShape;
  __shared__ __align__(128) unsigned char sbuf[CV_NS * S::STAGE];
  __shared__ __align__(8) uint64_t bar[CV_NS];
  __shared__ double red[CV_TY];
  const Tile t = tiles[blockIdx.x];
  if (!act[fl[t.blk].dom]) return;
  const BlkFld F = fl[t.blk];  // by value: read once, never reloaded after the stores below
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * OZ_TX + tx;
  constexpr bool UX = UMASK & 1, UY = (UMASK >> 1) & 1, UZ = (UMASK >> 2) & 1;
  const double dt = ds[F.dom].dt, alfapr = ds[F.dom].alfapr;
  const double dtinv = ds[F.dom].dtinv, rdt = ds[F.dom].rdt;
  const double dta = dt * alfapr;
  T *__restrict__ rhs1 = rhs_of<T>(F.L1);
  double *__restrict__ SU = write_su ? F.su : nullptr;
  const int nx = F.nx, ny = F.ny, nz = F.nz, pl = F.pl;
  const double ix = F.pinv[0], iy = F.pinv[1], iz = F.pinv[2];
  const bool ewall = F.wall[1], nwall = F.wall[3], twall = F.wall[5];
  const bool wwall = F.wall[0], swall = F.wall[2], bwall = F.wall[4];
  const int i = t.i0 + tx;
  const bool iin = i <= nx;
  const int ic = iin ? i : 1;  // clamped: every global load stays in bounds
  const double hx = F.h[0][ic], dxe = F.df[0][ic], dxw = F.df[0][ic - 1];
  // reciprocals of the x divisors (the exact inverse on a power-of-two axis)
  const double rhx = UX ? ix : F.rh[0][ic], rdxe = UX ? ix : F.rdf[0][ic], rdxw = UX ? ix : F.rdf[0][ic - 1];
  // rows of this thread
  int jc[CV_CR];
  bool in[CV_CR];
  double hy[CV_CR], dyn[CV_CR], dys[CV_CR], wb[CV_CR], rhy[CV_CR], rdyn[CV_CR], rdys[CV_CR];
  long long l1off[CV_CR];  // level-1 element of (i, j, 0) without the colour term
  int c0[CV_CR];           // colour of (i, j, 0)
  const long long ps1 = (long long)(F.L1.ny + 2) * F.L1.hp, sz = (long long)F.ti * F.tj;
  const int k0 = t.k0, k1 = min(t.k0 + kch - 1, nz);
#pragma unroll
  for (int m = 0; m < CV_CR; ++m) {
    const int j = t.j0 + CV_CR * ty + m;
    in[m] = iin && j <= ny;
    jc[m] = j <= ny ? j : 1;
    hy[m] = F.h[1][jc[m]];
    dyn[m] = F.df[1][jc[m]];
    dys[m] = F.df[1][jc[m] - 1];
    rhy[m] = UY ? iy : F.rh[1][jc[m]];
    rdyn[m] = UY ? iy : F.rdf[1][jc[m]];
    rdys[m] = UY ? iy : F.rdf[1][jc[m] - 1];
    l1off[m] = (long long)j * F.L1.hp + (i >> 1);
    c0[m] = (i + j + 1) & 1;
    // w on the face below plane k0, carried up the march (plain loads)
    const long long c = fidx(F, ic, jc[m], k0);
    if (k0 == 1) {
      const double lo = F.lo[2][(jc[m] - 1) * nx + (ic - 1)];
      wb[m] = bwall ? lo : (lo - qdiv<UZ>(dta * (F.p[c] - F.p[c - sz]), F.df[2][0], UZ ? iz : F.rdf[2][0]));
    } else {
      wb[m] = (F.wstar[c - sz] -
               qdiv<UZ>(dta * (F.p[c] - F.p[c - sz]), F.df[2][k0 - 1], UZ ? iz : F.rdf[2][k0 - 1]));
    }
  }
  const int a0 = t.i0 + pl - 1;   // field column of cell i0
  const int X = (a0 - 1) & ~1;    // box origin: even, so 16-byte aligned
  const int cx = a0 + tx - X;     // box column of this lane's cell
  const int yb = t.j0 + pl - 1;   // field row of row j0
  const CUtensorMap *mp = F.fm, *mu = F.fm + 1, *mv = F.fm + 2, *mw = F.fm + 3;
  auto stage = [&](int kk) { return (kk - k0) % CV_NS; };
  auto parity = [&](int kk) { return (unsigned)(((kk - k0) / CV_NS) & 1); };
  auto issue = [&](int kk) {  // planes k0..k1 all four boxes; k1+1 p only
    const int st = stage(kk), z = kk + pl - 1;
    unsigned char *b = sbuf + st * S::STAGE;
    const bool all = kk <= k1;
    const unsigned bytes = S::PR * CV_W * 8 + (all ? (S::UR + S::VR + S::WR) * CV_W * 8 : 0);
    mbar_expect_tx(&bar[st], bytes);
    tma_load_3d(b, mp, &bar[st], X, yb - 1, z);
    if (all) {
      tma_load_3d(b + S::PB, mu, &bar[st], X, yb, z);
      tma_load_3d(b + S::PB + S::UB, mv, &bar[st], X, yb - 1, z);
      tma_load_3d(b + S::PB + S::UB + S::VB, mw, &bar[st], X, yb, z);
    }
  };
  // every divisor of the march has its reciprocal (Markstein's correction
  // needs RN(1/b)); else the tile divides throughout
  bool fast = dtinv != 0.0 || rdt != 0.0;
  if (!UX) fast = fast && rhx != 0.0 && rdxe != 0.0 && rdxw != 0.0;
  if (!UY)
#pragma unroll
    for (int m = 0; m < CV_CR; ++m) fast = fast && rhy[m] != 0.0 && rdyn[m] != 0.0 && rdys[m] != 0.0;
  if (!UZ)
    for (int kk = k0; kk <= k1; ++kk) fast = fast && F.rdf[2][kk] != 0.0 && F.rh[2][kk] != 0.0;
  double vmax = 0.0;
  bool bad = !__syncthreads_and(fast);
  if (!bad) {
  if (tid == 0) {
    for (int st = 0; st < CV_NS; ++st) mbar_init(&bar[st], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (tid == 0)
    for (int kk = k0; kk < k0 + CV_PD && kk <= k1 + 1; ++kk) issue(kk);
  bool ok = mbar_wait(&bar[stage(k0)], parity(k0), err);
  for (int k = k0; k <= k1; ++k) {
    if (tid == 0 && ok && k + CV_PD <= k1 + 1) issue(k + CV_PD);  // into the slot of plane k-1
    if (ok) ok = mbar_wait(&bar[stage(k + 1)], parity(k + 1), err);
    const unsigned char *b = sbuf + stage(k) * S::STAGE;
    const double *P = (const double *)b, *U = (const double *)(b + S::PB);
    const double *Vv = (const double *)(b + S::PB + S::UB), *Wv = (const double *)(b + S::PB + S::UB + S::VB);
    const double *PN = (const double *)(sbuf + stage(k + 1) * S::STAGE);
    const double dzk = F.df[2][k], hzk = F.h[2][k];
    const double rdzk = UZ ? iz : F.rdf[2][k], rhzk = UZ ? iz : F.rh[2][k];
    const bool top = k == nz && twall;
    double vprev = 0.0;
#pragma unroll
    for (int m = 0; m < CV_CR; ++m) {
      const int rr = CV_CR * ty + m;   // row within the tile
      bool cb = false;                 // an operand out of Markstein's range
      const int r = (rr + 1) * CV_W + cx;  // this cell in the p box
      const double pc = P[r];
      double ue;
      if (ic == nx && ewall) ue = F.hi[0][(k - 1) * ny + (jc[m] - 1)];
      else ue = (U[rr * CV_W + cx] - qdv<UX>(dta * (P[r + 1] - pc), dxe, rdxe, cb));
      const double ul = __shfl_up_sync(0xffffffffu, ue, 1);
      double uw;
      if (ic == 1) {
        const double lo = F.lo[0][(k - 1) * ny + (jc[m] - 1)];
        uw = wwall ? lo : (lo - qdv<UX>(dta * (pc - P[r - 1]), dxw, rdxw, cb));
      } else if (tx > 0) {
        uw = ul;
      } else {
        uw = (U[rr * CV_W + cx - 1] - qdv<UX>(dta * (pc - P[r - 1]), dxw, rdxw, cb));
      }
      double vn, vs;
      if (jc[m] == ny && nwall) vn = F.hi[1][(k - 1) * nx + (ic - 1)];
      else vn = (Vv[(rr + 1) * CV_W + cx] - qdv<UY>(dta * (P[r + CV_W] - pc), dyn[m], rdyn[m], cb));
      if (m > 0) {
        vs = vprev;  // the south face of row j is the north face of row j-1 (same operands)
      } else if (jc[m] == 1) {
        const double lo = F.lo[1][(k - 1) * nx + (ic - 1)];
        vs = swall ? lo : (lo - qdv<UY>(dta * (pc - P[r - CV_W]), dys[m], rdys[m], cb));
      } else {
        vs = (Vv[rr * CV_W + cx] - qdv<UY>(dta * (pc - P[r - CV_W]), dys[m], rdys[m], cb));
      }
      vprev = vn;
      double wt;
      if (top) wt = F.hi[2][(jc[m] - 1) * nx + (ic - 1)];
      else wt = (Wv[rr * CV_W + cx] - qdv<UZ>(dta * (PN[r] - pc), dzk, rdzk, cb));
      const double fact =
          (qdv<UX>(ue - uw, hx, rhx, cb) + qdv<UY>(vn - vs, hy[m], rhy[m], cb) + qdv<UZ>(wt - wb[m], hzk, rhzk, cb));
      wb[m] = wt;  // the top face of plane k is the bottom face of plane k+1
      const double su = dtinv != 0.0 ? fact * dtinv : qdv<false>(fact, dt, rdt, cb);
      bad |= cb && in[m];
      if (ok && in[m]) {
        rhs1[((c0[m] ^ (k & 1)) ? F.L1.cstr : 0) + k * ps1 + l1off[m]] = (T)su;
        if (SU) SU[fidx(F, i, jc[m], k)] = su;
        double f1 = fabs(fact * hx * hy[m] * hzk);
        if (!(f1 == f1)) f1 = __longlong_as_double(0x7ff0000000000000LL);  // NaN -> +Inf (flagged)
        vmax = vmax > f1 ? vmax : f1;
      }
    }
    if (__syncthreads_or(!ok)) return;  // plane k's slot is refilled next iteration
  }
  }
  // an operand out of range somewhere in the tile: divide it again
  if (__syncthreads_or(bad)) vmax = cv_cells_divide<T>(F, i, t.j0 + CV_CR * ty, k0, k1, dt, dta, rhs1, SU);
  // CTA max: warp shuffles, shared memory, one atomic per CTA
  for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
  if (tx == 0) red[ty] = vmax;
  __syncthreads();
  if (ty == 0) {
    double v = tx < CV_TY ? red[tx] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (tx == 0 && v > 0.0) atomic_max_nonneg(rmax_slot + F.dom, v);
  }
}

// calvel (press.for:139-198) of one face: component comp (0 u, 1 v, 2 w) at
// level-1 cell (i, j, k), when calvel writes it (isu..ieu etc.: one face short
// at a high wall).  Under L_LSM the face density divides last (:152-190).
__device__ __forceinline__ void calvel_face(const BlkFld &F, int comp, int i, int j, int k, double dta) {
  const long long c = fidx(F, i, j, k);
  const long long st = comp == 0 ? 1 : comp == 1 ? (long long)F.ti : (long long)F.ti * F.tj;
  const int a = comp == 0 ? i : comp == 1 ? j : k;
  const int n = comp == 0 ? F.nx : comp == 1 ? F.ny : F.nz;
  if (a == n && F.wall[2 * comp + 1]) return;
  const double *__restrict__ p = F.p;
  const double *S = comp == 0 ? F.ustar : comp == 1 ? F.vstar : F.wstar;
  double *O = comp == 0 ? F.u : comp == 1 ? F.v : F.w;
  const double *__restrict__ D = F.dens;
  if (D) O[c] = (S[c] - xdiv(dta * (p[c + st] - p[c]), F.df[comp][a], F.pinv[comp]) / (0.5 * (D[c] + D[c + st])));
  else O[c] = (S[c] - xdiv(dta * (p[c + st] - p[c]), F.df[comp][a], F.pinv[comp]));
}

// Final calvel (press.for:139-198): u, v, w on the faces calvel writes
// (isu..ieu etc., one face short at a high wall), from the final p.
// `only` (may be null): domains to update, others are left as they are.
__global__ void __launch_bounds__(RW_TX *RW_RJ) k_calvel(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles,
                                                         const DomState *__restrict__ ds, const int *__restrict__ only) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  if (only && !only[F.dom]) return;
  const double dt = ds[F.dom].dt, alfapr = ds[F.dom].alfapr;
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  if (i > F.nx || j > F.ny) return;
  const double dta = dt * alfapr;
  const int k1 = min(t.k0 + RW_KCH - 1, F.nz);
  for (int k = t.k0; k <= k1; ++k) {
    calvel_face(F, 0, i, j, k, dta);
    calvel_face(F, 1, i, j, k, dta);
    calvel_face(F, 2, i, j, k, dta);
  }
}

// exchange(1..3) across outer iterations.  The reference runs calvel and
// its exchange in every outer iteration; some ghost cells of an exchange
// take a ghost cell of the state before it (exchange_bc copies whole ghost-
// inclusive planes, corner cubes reach a neighbour's ghost layer), so their
// final values come from earlier iterations' exchanges.  The library
// evolves exactly those cells: the closure C of ghost cells such chains
// reach is re-exchanged at every calvel point (the initial calvel and each
// outer iteration).  k_fx_evolve (i) forms calvel at the interior faces the
// sub-map of C reads (`cells`: block, component, i, j, k; u, v, w written
// there as calvel writes them - the final calvel rewrites them with the same
// values), (ii) saves the pre-exchange value of every chained source into
// `prev`, and (iii) stages the sources of the sub-map's staged pairs; then
// k_fx_apply writes the sub-map.  The final exchange reads chained sources
// from `prev` (FxCopy comp bit 8).  Reads in k_fx_evolve touch ghost cells
// only, writes interior cells only, so the three parts do not race.
struct FxCell {
  int blk, comp, i, j, k;
};
__global__ void k_fx_evolve(const BlkFld *__restrict__ fl, const DomState *__restrict__ ds,
                            const int *__restrict__ only, const FxCell *__restrict__ cells, long long ncell,
                            const FxCopy *__restrict__ chain, long long nchain, double *__restrict__ prev,
                            const FxCopy *__restrict__ sub, long long nstaged, double *__restrict__ buf) {
  pdl_wait();
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < ncell) {
    const FxCell c = cells[t];
    const BlkFld &F = fl[c.blk];
    if (only && !only[F.dom]) return;
    calvel_face(F, c.comp, c.i, c.j, c.k, ds[F.dom].dt * ds[F.dom].alfapr);
    return;
  }
  t -= ncell;
  if (t < nchain) {  // chain[t]: src = the chained source cell, soff its prev slot
    const FxCopy x = chain[t];
    if (only && !only[fl[x.sblk].dom]) return;
    prev[t] = fx_field(fl[x.sblk], x.comp & 7)[x.doff];
    return;
  }
  t -= nchain;
  if (t < nstaged) {
    const FxCopy x = sub[t];
    if (only && !only[fl[x.dblk].dom]) return;
    buf[t] = fx_field(fl[x.sblk], x.comp & 7)[x.soff];
  }
}

// calmas, 4th-order branch (press.for:13-35, differencing = 2), on the
// velocities that calvel and exchange(1..3) left in u, v, w (k_calvel +
// k_vel_faces, the reference's order):
//   fact = (-u(i+1)+27.0*u(i)-27.0*u(i-1)+u(i-2))/(24.0*dx) + (the same in
//          v along j)/(24.0*dy) + (the same in w along k)/(24.0*dz),
// each numerator summed left to right; su = fact/dt into the level-1 rhs
// (and F.su when asked), rmax = max |((fact*dx)*dy)*dz| as in k_calvel_calmas.
// u(i+1) at i = nx and u(i-2) at i = 1 are ghost faces: the neighbour's
// values for the exchanged layers, else whatever the caller's arrays hold,
// as in the reference.  Uniform spacing (h[a][1] is the block's dx, dy, dz).
template <typename T>
__global__ void __launch_bounds__(RW_TX *RW_RJ) k_calmas4(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles,
                                                          const DomState *__restrict__ ds, const int *__restrict__ act,
                                                          unsigned long long *__restrict__ rmax_slot, int write_su) {
  pdl_wait();
  __shared__ double red[RW_RJ];
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  if (!act[F.dom]) return;
  const double dt = ds[F.dom].dt, dtinv = ds[F.dom].dtinv;
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  const bool in = i <= F.nx && j <= F.ny;
  const double dx = F.h[0][1], dy = F.h[1][1], dz = F.h[2][1];
  const double d24x = 24.0 * dx, d24y = 24.0 * dy, d24z = 24.0 * dz;
  const long long sy = F.ti, sz = (long long)F.ti * F.tj;
  const double *__restrict__ U = F.u;
  const double *__restrict__ Vv = F.v;
  const double *__restrict__ Wv = F.w;
  T *__restrict__ rhs1 = rhs_of<T>(F.L1);
  double *__restrict__ SU = write_su ? F.su : nullptr;
  double vmax = 0.0;
  if (in) {
    const int k1 = min(t.k0 + RW_KCH - 1, F.nz);
    for (int k = t.k0; k <= k1; ++k) {
      const long long c = fidx(F, i, j, k);
      const double fx = ((((-U[c + 1]) + 27.0 * U[c]) - 27.0 * U[c - 1]) + U[c - 2]) / d24x;
      const double fy = ((((-Vv[c + sy]) + 27.0 * Vv[c]) - 27.0 * Vv[c - sy]) + Vv[c - 2 * sy]) / d24y;
      const double fz = ((((-Wv[c + sz]) + 27.0 * Wv[c]) - 27.0 * Wv[c - sz]) + Wv[c - 2 * sz]) / d24z;
      const double fact = (fx + fy) + fz;
      const double su = xdiv(fact, dt, dtinv);
      rhs1[cell_off(F.L1, i, j, k)] = (T)su;
      if (SU) SU[c] = su;
      double f1 = fabs(fact * dx * dy * dz);
      if (!(f1 == f1)) f1 = __longlong_as_double(0x7ff0000000000000LL);  // NaN -> +Inf (flagged)
      vmax = vmax > f1 ? vmax : f1;
    }
  }
  for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
  if (threadIdx.x == 0) red[threadIdx.y] = vmax;
  __syncthreads();
  if (threadIdx.y == 0) {
    double v = threadIdx.x < RW_RJ ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0 && v > 0.0) atomic_max_nonneg(rmax_slot + F.dom, v);
  }
}

// One Runge-Kutta stage of the velocity predictor for component `comp`
// (rungek_conv2nd, rungek.for:314-412, then rungek_diff2nd, :584-779, the
// branch without L_LSM, immersed boundaries or wall functions), over the
// component's faces 1..comp_end:
//   star = (oo - dt*alfapr*(c1 + c2 + c3)), the 2nd-order conservative
//     convection terms as the reference writes them (x**2 is x*x);
//   star = (star + dt*alfapr*diff), diff = -(ap*c + an*c(j+1) + as*c(j-1)
//     + ae*c(i+1) + aw*c(i-1) + at*c(k+1) + ab*c(k-1)) with a* = -visc/d*d*
//     from the viscosity of the cell past the face, ap = -1.0*(aw+ae+as+an+
//     ab+at);
//   u under pressureforce: star = star + dt*alfapr*forcn.
// Fusing the two loops per cell keeps the reference's values: rungek_diff2nd
// reads only the component itself, which boundv/boundw do not touch.
__global__ void __launch_bounds__(RW_TX *RW_RJ) k_rk2nd(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles,
                                                        int comp, double dt, double alfapr, int pforce, double forcn) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  if (i > comp_end(F, comp, 0) || j > comp_end(F, comp, 1)) return;
  const int k1 = min(t.k0 + RW_KCH - 1, comp_end(F, comp, 2));
  const long long sy = F.ti, sz = (long long)F.ti * F.tj;
  const double dx = F.h[0][1], dy = F.h[1][1], dz = F.h[2][1];
  const double dxx = dx * dx, dyy = dy * dy, dzz = dz * dz;
  const double *__restrict__ U = F.u;
  const double *__restrict__ V = F.v;
  const double *__restrict__ W = F.w;
  const double *__restrict__ C = comp_field(F, comp);
  const double *__restrict__ OO = F.oo[comp];
  double *__restrict__ ST = comp == 0 ? F.ustar : comp == 1 ? F.vstar : F.wstar;
  const long long so = comp == 0 ? 1 : comp == 1 ? sy : sz;  // the cell past the face
  for (int k = t.k0; k <= k1; ++k) {
    const long long c = fidx(F, i, j, k);
    double c1, c2, c3;
    if (comp == 0) {
      const double up12 = 0.5 * (U[c] + U[c + 1]), um12 = 0.5 * (U[c] + U[c - 1]);
      c1 = (up12 * up12 - um12 * um12) / dx;
      c2 = 0.25 * ((V[c] + V[c + 1]) * (U[c] + U[c + sy]) - (V[c - sy] + V[c + 1 - sy]) * (U[c] + U[c - sy])) / dy;
      c3 = 0.25 * ((W[c] + W[c + 1]) * (U[c] + U[c + sz]) - (W[c - sz] + W[c + 1 - sz]) * (U[c] + U[c - sz])) / dz;
    } else if (comp == 1) {
      const double vp12 = 0.5 * (V[c] + V[c + sy]), vm12 = 0.5 * (V[c] + V[c - sy]);
      c2 = (vp12 * vp12 - vm12 * vm12) / dy;
      c1 = 0.25 * ((U[c] + U[c + sy]) * (V[c] + V[c + 1]) - (U[c - 1] + U[c - 1 + sy]) * (V[c] + V[c - 1])) / dx;
      c3 = 0.25 * ((W[c] + W[c + sy]) * (V[c] + V[c + sz]) - (W[c - sz] + W[c + sy - sz]) * (V[c] + V[c - sz])) / dz;
    } else {
      const double wp12 = 0.5 * (W[c] + W[c + sz]), wm12 = 0.5 * (W[c] + W[c - sz]);
      c3 = (wp12 * wp12 - wm12 * wm12) / dz;
      c1 = 0.25 * ((U[c] + U[c + sz]) * (W[c] + W[c + 1]) - (U[c - 1] + U[c - 1 + sz]) * (W[c] + W[c - 1])) / dx;
      c2 = 0.25 * ((V[c] + V[c + sz]) * (W[c] + W[c + sy]) - (V[c - sy] + V[c - sy + sz]) * (W[c] + W[c - sy])) / dy;
    }
    double st = (OO[c] - dt * alfapr * (c1 + c2 + c3));
    const double visc = F.vis[c + so];
    const double aw = -visc / dxx, ae = -visc / dxx, an = -visc / dyy, as = -visc / dyy;
    const double at = -visc / dzz, ab = -visc / dzz;
    const double ap = -1.0 * (aw + ae + as + an + ab + at);
    const double diff = -(ap * C[c] + an * C[c + sy] + as * C[c - sy] + ae * C[c + 1] + aw * C[c - 1] +
                          at * C[c + sz] + ab * C[c - sz]);
    st = (st + dt * alfapr * diff);
    if (comp == 0 && pforce) st = st + dt * alfapr * forcn;
    ST[c] = st;
  }
}

// The same stage with differencing = 2: rungek_conv4th (rungek.for:2-212)
// and rungek_diff4th (rungek.for:214-312) for component `comp` (axis a):
//   star = (oo - dt*alfapr*(t_x + t_y + t_z)), t_a = (-s(+2) + 27 s(+1) -
//     27 s(0) + s(-1))/(24 h_a) with s(m) the square of the component
//     interpolated to the cell centre m - 1/2 along a, and for b != a
//     t_b = (-P(+1) + 27 P(0) - 27 P(-1) + P(-2))/(24 h_b), P(m) = the
//     component interpolated along b times the b-velocity interpolated along
//     a, at b-offset m - each interpolant (-f(+1) + 9 f(0) + 9 f(-1) -
//     f(-2))/16 as the reference writes them;
//   star = (star + dt*alfapr*diff), diff = visc*(L_x + L_y + L_z),
//     L_b = (-c(+2) + 16 c(+1) - 30 c + 16 c(-1) - c(-2))/(12 h_b^2), visc
//     the viscosity of the face's own cell for u and of the cell past the
//     face for v and w (rungek.for:230, 262, 290);
//   u under pressureforce: star = star + dt*alfapr*forcn.
// The stencils reach three cells each way (pl >= 3).
__global__ void __launch_bounds__(RW_TX *RW_RJ) k_rk4th(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles,
                                                        int comp, double dt, double alfapr, int pforce, double forcn) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  if (i > comp_end(F, comp, 0) || j > comp_end(F, comp, 1)) return;
  const int k1 = min(t.k0 + RW_KCH - 1, comp_end(F, comp, 2));
  const long long st3[3] = {1, (long long)F.ti, (long long)F.ti * F.tj};
  const double h[3] = {F.h[0][1], F.h[1][1], F.h[2][1]};
  const double *vel[3] = {F.u, F.v, F.w};
  const double *__restrict__ Cf = vel[comp];
  const double *__restrict__ OO = F.oo[comp];
  double *__restrict__ ST = comp == 0 ? F.ustar : comp == 1 ? F.vstar : F.wstar;
  const long long sa = st3[comp];
  // (-f(+1) + 9 f(0) + 9 f(-1) - f(-2)) / 16 along stride s, around element e
  auto q4 = [](const double *f, long long e, long long s) {
    return (-f[e + s] + 9.0 * f[e] + 9.0 * f[e - s] - f[e - 2 * s]) / 16.0;
  };
  auto d4 = [](double p1, double p0, double m1, double m2, double hh) {
    return (-p1 + 27.0 * p0 - 27.0 * m1 + m2) / (24.0 * hh);
  };
  for (int k = t.k0; k <= k1; ++k) {
    const long long c = fidx(F, i, j, k);
    double term[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      if (b == comp) {
        double s4[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const double q = q4(Cf, c + (2 - m) * sa, sa);
          s4[m] = q * q;
        }
        term[b] = d4(s4[0], s4[1], s4[2], s4[3], h[b]);
      } else {
        const long long sb = st3[b];
        double p4[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          const long long e = c + (1 - m) * sb;  // b-offset 1, 0, -1, -2
          p4[m] = q4(Cf, e + sb, sb) * q4(vel[b], e + sa, sa);
        }
        term[b] = d4(p4[0], p4[1], p4[2], p4[3], h[b]);
      }
    }
    double st = (OO[c] - dt * alfapr * (term[0] + term[1] + term[2]));
    const double visc = F.vis[comp == 0 ? c : c + sa];
    double lap[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      const long long sb = st3[b];
      lap[b] = (-Cf[c + 2 * sb] + 16.0 * Cf[c + sb] - 30.0 * Cf[c] + 16.0 * Cf[c - sb] - Cf[c - 2 * sb]) /
               (12.0 * (h[b] * h[b]));
    }
    const double diff = visc * (lap[0] + lap[1] + lap[2]);
    st = (st + dt * alfapr * diff);
    if (comp == 0 && pforce) st = st + dt * alfapr * forcn;
    ST[c] = st;
  }
}

// HJ_WENO's fifth-order one-sided derivative from five divided differences
// (weno.for:56-78; REAL is double, x**2 is x*x, MAX of the five squares).
__device__ __forceinline__ double weno5(double v1, double v2, double v3, double v4, double v5) {
  const double v11 = v1 * v1, v22 = v2 * v2, v33 = v3 * v3, v44 = v4 * v4, v55 = v5 * v5;
  const double e = (1.0E-6) * fmax(fmax(fmax(fmax(v11, v22), v33), v44), v55) + 1.0E-99;
  const double t11 = v1 - 2.0 * v2 + v3, t12 = v1 - 4.0 * v2 + 3.0 * v3;
  const double t21 = v2 - 2.0 * v3 + v4, t22 = v2 - v4;
  const double t31 = v3 - 2.0 * v4 + v5, t32 = 3.0 * v3 - 4.0 * v4 + v5;
  const double S1 = (13.0 / 12.0) * (t11 * t11) + 0.25 * (t12 * t12);
  const double S2 = (13.0 / 12.0) * (t21 * t21) + 0.25 * (t22 * t22);
  const double S3 = (13.0 / 12.0) * (t31 * t31) + 0.25 * (t32 * t32);
  const double d1 = e + S1, d2 = e + S2, d3 = e + S3;
  const double a1 = 0.1 / (d1 * d1), a2 = 0.6 / (d2 * d2), a3 = 0.3 / (d3 * d3);
  const double w1 = a1 / (a1 + a2 + a3), w2 = a2 / (a1 + a2 + a3), w3 = a3 / (a1 + a2 + a3);
  return w1 * (v1 * (1.0 / 3.0) - v2 * (7.0 / 6.0) + v3 * (11.0 / 6.0)) +
         w2 * (-(v2 * (1.0 / 6.0)) + v3 * (5.0 / 6.0) + v4 * (1.0 / 3.0)) +
         w3 * (v3 * (1.0 / 3.0) + v4 * (5.0 / 6.0) - v5 * (1.0 / 6.0));
}

// The same stage with differencing = 3: rungek_convWENO (rungek.for:
// 414-582) then rungek_diff2nd, for component `comp`.  Each derivative is
// HJ_WENO's (weno.for:2-354) at this cell - the divided differences
// D1(m) = (f(m+1) - f(m))/h formed on the fly - upwinded by the sign of the
// advecting velocity (its own value along its axis, the 4-face average
// 0.25*(...) along the others), 0 where that is 0; HJ_WENO leaves 0 outside
// cells 4 .. end + pl_ex + 1 - 3 of each axis (1-based field indices; end
// the component's range end), and so does this.  Then rungek_diff2nd's
// terms as k_rk2nd forms them.
__global__ void __launch_bounds__(RW_TX *RW_RJ) k_rkweno(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles,
                                                         int comp, int pl_ex, double dt, double alfapr, int pforce,
                                                         double forcn) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  if (i > comp_end(F, comp, 0) || j > comp_end(F, comp, 1)) return;
  const int k1 = min(t.k0 + RW_KCH - 1, comp_end(F, comp, 2));
  const long long st3[3] = {1, (long long)F.ti, (long long)F.ti * F.tj};
  const double h[3] = {F.h[0][1], F.h[1][1], F.h[2][1]};
  const double *__restrict__ U = F.u;
  const double *__restrict__ V = F.v;
  const double *__restrict__ W = F.w;
  const double *__restrict__ Cf = comp_field(F, comp);
  const double *__restrict__ OO = F.oo[comp];
  double *__restrict__ ST = comp == 0 ? F.ustar : comp == 1 ? F.vstar : F.wstar;
  // HJ_WENO's range ends, 1-based field indices: the component's ends + pl_ex + 1
  int lim[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) lim[a] = comp_end(F, comp, a) + F.pl + pl_ex + 1;
  const long long sy = st3[1], sz = st3[2];
  for (int k = t.k0; k <= k1; ++k) {
    const long long c = fidx(F, i, j, k);
    const int fx[3] = {i + F.pl, j + F.pl, k + F.pl};  // 1-based field indices
    // the advecting velocity of each axis at this face
    double adv[3];
    if (comp == 0) {
      adv[0] = U[c];
      adv[1] = 0.25 * (V[c] + V[c + 1] + V[c - sy] + V[c + 1 - sy]);
      adv[2] = 0.25 * (W[c] + W[c + 1] + W[c - sz] + W[c + 1 - sz]);
    } else if (comp == 1) {
      adv[0] = 0.25 * (U[c] + U[c + sy] + U[c - 1] + U[c - 1 + sy]);
      adv[1] = V[c];
      adv[2] = 0.25 * (W[c] + W[c + sy] + W[c - sz] + W[c + sy - sz]);
    } else {
      adv[0] = 0.25 * (U[c] + U[c + sz] + U[c - 1] + U[c - 1 + sz]);
      adv[1] = 0.25 * (V[c] + V[c + sz] + V[c - sy] + V[c - sy + sz]);
      adv[2] = W[c];
    }
    double term[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double sgn = adv[a];
      double d = 0.0;
      // HJ_WENO writes cells 4 .. lim-3 along a, 1 .. lim of the others
      bool inside = fx[a] >= 4 && fx[a] <= lim[a] - 3;
#pragma unroll
      for (int b = 0; b < 3; ++b)
        if (b != a) inside = inside && fx[b] >= 1 && fx[b] <= lim[b];
      if (inside && sgn != 0.0) {
        const long long s = st3[a];
        auto D1 = [&](int m) { return (Cf[c + (m + 1) * s] - Cf[c + m * s]) / h[a]; };
        // plus (L = I = cell - 3): D1(+2) .. D1(-2); minus (L = I - 1): D1(-3) .. D1(+1)
        d = sgn > 0.0 ? weno5(D1(-3), D1(-2), D1(-1), D1(0), D1(1)) : weno5(D1(2), D1(1), D1(0), D1(-1), D1(-2));
      }
      term[a] = sgn * d;
    }
    double st = (OO[c] - dt * alfapr * (term[0] + term[1] + term[2]));
    const double dxx = h[0] * h[0], dyy = h[1] * h[1], dzz = h[2] * h[2];
    const double visc = F.vis[c + st3[comp]];
    const double aw = -visc / dxx, ae = -visc / dxx, an = -visc / dyy, as = -visc / dyy;
    const double at = -visc / dzz, ab = -visc / dzz;
    const double ap = -1.0 * (aw + ae + as + an + ab + at);
    const double diff = -(ap * Cf[c] + an * Cf[c + sy] + as * Cf[c - sy] + ae * Cf[c + 1] + aw * Cf[c - 1] +
                          at * Cf[c + sz] + ab * Cf[c - sz]);
    st = (st + dt * alfapr * diff);
    if (comp == 0 && pforce) st = st + dt * alfapr * forcn;
    ST[c] = st;
  }
}

// After the initial calvel/calmas (newsolv_mg.for:16-17): rmax0, the
// absolute threshold, and which domains iterate at all.
__global__ void k_dom_init(DomState *ds, int ndom, unsigned long long *rmax_slot, int *act) {
  pdl_wait();
  for (int d = threadIdx.x; d < ndom; d += blockDim.x) {
    const double r = __longlong_as_double((long long)rmax_slot[d]);
    rmax_slot[d] = 0ull;
    DomState &D = ds[d];
    D.rmax0 = r;
    D.rmax = r;
    D.eps = D.eps_relative ? D.tol * r : D.tol;
    D.iter = 0;
    D.done = !(r <= 1.7976931348623157e308) ? 2 : (D.maxcy <= 0 ? 3 : 0);
    act[d] = D.done ? 0 : 1;
  }
}

// End of one outer iteration (newsolv_mg.for:54-58), per active domain:
// record rmax, count the iteration, test `rmax < eps .and. iter > 1` (or
// maxcy); a domain that stops is switched off for every later launch.  In
// the solve graph, also sets the WHILE condition: any domain still running.
// in_graph 2 (the server's bounded loop): the WHILE condition also ends the
// loop when a domain stops in this iteration or when `budget` iterations
// have run, so the host can hand results back and admit new requests.
__global__ void k_iter_end(DomState *ds, int ndom, unsigned long long *rmax_slot, double *hist, int hcap, int *act,
                           cudaGraphConditionalHandle cond, int in_graph, int *budget) {
  pdl_wait();
  int any = 0, stopped = 0;
  for (int d = threadIdx.x; d < ndom; d += blockDim.x) {
    if (!act[d]) continue;
    DomState &D = ds[d];
    const double r = __longlong_as_double((long long)rmax_slot[d]);
    rmax_slot[d] = 0ull;
    const int it = D.iter + 1;
    D.iter = it;
    D.rmax = r;
    if (it - 1 < hcap) hist[(long long)d * hcap + it - 1] = r;
    int done = 0;
    if (!(r <= 1.7976931348623157e308)) done = 2;  // +Inf (a NaN is stored as +Inf)
    else if (r < D.eps && it > 1) done = 1;
    else if (it >= D.maxcy) done = 3;
    D.done = done;
    if (done) {
      act[d] = 0;
      stopped = 1;
    } else {
      any = 1;
    }
  }
  any = __syncthreads_or(any);
  stopped = __syncthreads_or(stopped);
  if (threadIdx.x == 0) {
    if (in_graph == 1) cudaGraphSetConditional(cond, any ? 1u : 0u);
    if (in_graph == 2) {
      const int left = --budget[0];
      cudaGraphSetConditional(cond, (any && !stopped && left > 0) ? 1u : 0u);
    }
  }
}

// Level-1 rhs := su (mgkcyc's copy-in, mgsolver.for:250-263) from a ttc array.
template <typename T>
__global__ void k_load_rhs(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles, double *const *__restrict__ su) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  if (i < 1 || i > F.nx || j < 1 || j > F.ny) return;
  for (int k = t.k0; k <= min(t.k0 + RW_KCH - 1, F.nz); ++k)
    rhs_of<T>(F.L1)[cell_off(F.L1, i, j, k)] = (T)su[t.blk][fidx(F, i, j, k)];
}

// pp := level-1 phi including the first ghost layer (mgsolver.for:351-364).
template <typename T>
__global__ void k_store_pp(const BlkFld *__restrict__ fl, const Tile *__restrict__ tiles, double *const *__restrict__ pp) {
  pdl_wait();
  const Tile t = tiles[blockIdx.x];
  const BlkFld &F = fl[t.blk];
  const BlkLev &B = F.L1;
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  if (i > B.nx + 1 || j > B.ny + 1) return;
  for (int k = t.k0; k <= min(t.k0 + RW_KCH - 1, B.nz + 1); ++k)
    pp[t.blk][fidx(F, i, j, k)] = (double)phi_of<T>(B)[cell_off(B, i, j, k)];
}

}  // namespace mf3d
