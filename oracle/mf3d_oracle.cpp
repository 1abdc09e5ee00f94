/*
 * TEST INFRASTRUCTURE ONLY - the oracle.
 *
 * A literal CPU restatement (C++17, -O2 -ffp-contract=off) of MultiFlow3D's
 * pressure-Poisson path, used by the tests, by __graft_entry__.smoke() and by
 * bench.py's CPU-baseline leg as the checker.  The shipped library never
 * links, loads or calls this file.
 *
 * Parity status: the reference is Fortran 90 + MPI and this container has no
 * Fortran compiler, so the reference cannot be run here ("parity pinned by
 * analytic known-answer tests, not by reference outputs"): the reference
 * ships no tests, golden vectors or fixtures.  This restatement is pinned by
 * the known-answer tests under tests/ (discrete eigenfunctions, an FFT/DCT
 * direct solve, nullspace and symmetry identities, decomposition invariance).
 *
 * Each routine follows the reference loop by loop, in the same evaluation
 * order, with the reference's own storage:
 *   - `cof` per block: level-g correction phi with a 1-cell ghost shell,
 *     j fastest then i then k, followed by the 8 interior arrays
 *     aw, ae, as, an, ab, at, ap, rhs (mgsolver.for:20-38, 112-210);
 *   - fields p, u, v, w, ustar, ... as Fortran (ttc_i,ttc_j,ttc_k) arrays,
 *     i fastest, pl ghost layers (initial.for:196-210).
 * The single-rank branches (one MPI rank owning every block, the
 * `dom_ad(a) .eq. dom_ad(b)` direct-buffer path) are restated, with the
 * L_LSM variable-density branches of coeff, calvel and calmas.  The LMR 2:1
 * branches are restated for the multigrid V-cycle (mgkcyc): the per-block
 * level clamping of localparameters.for:26-75 and mgsolver.for, and the
 * fine/coarse cases of exchangepp.  The outer loop's field exchanges at
 * refinement interfaces (exchangep.for, exchangeu/v/w.for) are not, so
 * orc_newsolv_mg refuses an LMR layout.  The LMR unpack of a fine block's
 * face reads entries of its receive buffer that the coarse sender never
 * writes (the ring s = 1, ns1 or t = 1, ns2; exchangepp.for:4036-4060):
 * the reference leaves there whatever an earlier exchange of any field put
 * in the shared buffer.  Here every pack starts from a buffer holding one
 * value, g_lmr_ring (0 by default, orc_set_lmr_ring), so that the cells
 * that depend on those entries can be found by changing it.
 *
 * Extension with no reference counterpart (marked EXT): non-uniform cell
 * widths.  With uniform widths every EXT formula reduces bit-for-bit to the
 * reference expression.
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <thread>

#include "../include/mf3d.h"

namespace {

struct Blk {
  mf3d_block_desc d;
  int ngrid;
  int rdiv = 1;                /* LMR refinement (localparameters.for:100-102) */
  std::vector<int> rdv;        /* rdv(dom, g), g = 1..ngrd_gl (localparameters.for:39-57) */
  int isp, iep, jsp, jep, ksp, kep;
  int isu, ieu, jsu, jeu, ksu, keu;
  int isv, iev, jsv, jev, ksv, kev;
  int isw, iew, jsw, jew, ksw, kew;
  int ttc_i, ttc_j, ttc_k;
  std::vector<long> faz;       /* faz[1..ngrd_gl] */
  std::vector<double> cof;     /* 1-based: cof[1..nwork] */
  double *ustar, *vstar, *wstar, *u, *v, *w, *p;
  double *dens = nullptr;      /* L_LSM: cell densities (ttc layout) */
  std::vector<std::vector<double>> dens_mg; /* L_LSM: per level, interior cells, j fastest */
  std::vector<double> su, pp;  /* su holds sup under L_LSM (mgsolver.for:256-261) */
  /* same-rank receive buffers of exchangepp / exchbc_mgpp (1-based) */
  std::vector<double> recvb_m1, recvb_p1;
  double rcm[5], rcp[5];
  std::vector<double> rem[7], rep[7];
  /* receive buffers of exchange_smlvl / exchange_bc (1-based) */
  std::vector<double> frm[4], frp[4];
  /* EXT: cell widths per level incl. ghost cells, index 0..n+1 */
  std::vector<std::vector<double>> hx, hy, hz;
  bool stretched;
  /* the velocity predictor: uoo, voo, woo (the convective outflow, code 21) */
  const double *oo[3] = {nullptr, nullptr, nullptr};
  /* west inlet of the codes 7, 8 (the file's values) and 12, 13 (the
   * power-law profile): u over j = js-1..je+1, k = ks-1..ke+1, j fastest */
  std::vector<double> inlet;
};

/* The reference runs one MPI rank per block; the restatement runs the
 * independent per-block loops of a phase on OpenMP threads (no effect on
 * the arithmetic: blocks never read each other inside a phase). */
int g_threads = 1;
double *g_tstamp = nullptr; /* optional wall-clock stamps, seconds */
int g_tcap = 0;
inline double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
inline void stamp(int q) { if (g_tstamp && q < g_tcap) g_tstamp[q] = now_s(); }
template <class Fn> void par_blocks(int n, Fn fn) {
  int nt = std::min(n, g_threads);
  if (nt <= 1) { for (int i = 0; i < n; ++i) fn(i); return; }
  std::atomic<int> next(0);
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t) th.emplace_back([&] { for (int i; (i = next++) < n;) fn(i); });
  for (auto &x : th) x.join();
}

struct Ctx {
  std::vector<Blk> b;
  std::map<int, int> indid; /* dom_indid: block id -> position */
  int ngrd_gl, mg_itrsch, irestr, iproln, maxcy, pl, pl_ex;
  bool lsm; /* L_LSM: variable-density coefficients, calvel and rhs */
  bool bounds; /* boundu/boundv/boundw after the loop (newsolv_mg.for:86-88) */
  int alfabc;   /* 1: outflow faces (code 2) copy the last face */
  double ubulk; /* inflow velocity of code-1 west faces */
  int solver;   /* 2: multigrid newsolv_mg; 1: pressure_1sweep with SIP */
  int nswp;     /* SIP inner sweeps per call (control.cin nswp(4)) */
  long long sip_sweeps; /* nsweeps: inner sweeps run over the solve */
  double eps;
  int eps_relative;
  int differencing; /* 2: calmas' 4th-order divergence (press.for:13-35) */
  bool periodic;
  double dt, alfapr, rmax;
  double yst, yen, zst, zen; /* extents of the whole domain (alloc_dom.for:427-439) */
  bool lmr = false;          /* blocks of different refinement */
};

/* The inlet files of the west codes 7 (Inlet/Inlet_<dom>_<n>.dat: u per
 * line) and 8 (inflow/Inlet_<dom>_<n>.dat: two header lines, then
 * "up dummy dummy" per line) stand here as value arrays registered per block
 * id, together with UPROF_SEM for code 8 (initial.for:37). */
struct InletFile {
  int code, uprof;
  std::vector<double> v;
};
std::map<int, InletFile> g_inlets;
/* uoo, voo, woo per block position for the convective outflow (code 21) of
 * the solve's boundu/v/w; empty = none */
std::vector<std::array<const double *, 3>> g_old;
/* Re and fric (control.cin) for the wall functions; Re = 0: not given */
double g_re = 0.0, g_fric = 0.0;
bool g_wall_fail = false; /* a smooth-wall law did not converge */
std::string g_err;        /* the last error (orc_last_error) */
double g_lmr_ring = 0.0;  /* LMR: the receive-buffer entries no sender writes */

inline double &F(Blk &B, double *a, int i, int j, int k) {
  return a[(size_t)(i - 1) + (size_t)B.ttc_i * ((size_t)(j - 1) + (size_t)B.ttc_j * (size_t)(k - 1))];
}
inline double F(Blk &B, const double *a, int i, int j, int k) {
  return a[(size_t)(i - 1) + (size_t)B.ttc_i * ((size_t)(j - 1) + (size_t)B.ttc_j * (size_t)(k - 1))];
}

int level_n(int n, int gl) { return n / (1 << (gl - 1)) + 2; }

/* EXT: widths of each level, ghost-inclusive (index 0 and n+1 are the
 * ghost cells).  `ext` holds the fine widths of the block with
 * W = 2^(ngrid-1) neighbour cells on each side (NULL = uniform h).  Level g
 * merges pairs of level g-1 cells, so uniform widths stay exact powers of
 * two times h and every EXT formula reduces to the reference's. */
std::vector<std::vector<double>> level_widths(const double *ext, int n, double h,
                                              int ngrid) {
  int W = 1 << (ngrid - 1);
  std::vector<std::vector<double>> out(ngrid + 1);
  std::vector<double> e(n + 2 * W);
  for (int q = 0; q < n + 2 * W; ++q) e[q] = ext ? ext[q] : h;
  int Wg = W;
  for (int g = 1; g <= ngrid; ++g) {
    if (g > 1) {
      std::vector<double> m(e.size() / 2);
      for (size_t q = 0; q < m.size(); ++q) m[q] = e[2 * q] + e[2 * q + 1];
      e.swap(m);
      Wg /= 2;
    }
    int nl = n >> (g - 1);
    std::vector<double> w(nl + 2);
    for (int c = 0; c < nl + 2; ++c) w[c] = e[Wg - 1 + c];
    out[g] = w;
  }
  return out;
}

/* ------------------------------------------------------------------ */
/* coeff (mgsolver.for:2-222), uniform and L_LSM branches + EXT widths. */
/* ------------------------------------------------------------------ */
/* L_LSM cell densities of level g, interior cells, reference layout
 * (j fastest, then i, then k; mgsolver.for:69-116): level 1 copies dens,
 * level g averages the 8 children of level g-1 in the reference's order
 * (j, j+1, i+1, i+1 j+1, then the same one plane up). */
void lsm_density(Blk &B, int ngrd, int pl) {
  int nx = B.iep - B.isp + 1, ny = B.jep - B.jsp + 1, nz = B.kep - B.ksp + 1;
  B.dens_mg.assign(ngrd + 1, {});
  for (int g = 1; g <= ngrd; ++g) {
    int gl = g > B.ngrid ? B.ngrid : g;
    int mi = level_n(nx, gl) - 2, mj = level_n(ny, gl) - 2, mk = level_n(nz, gl) - 2;
    std::vector<double> &d = B.dens_mg[g];
    d.assign((size_t)mi * mj * mk, 0.0);
    for (int k = 2; k <= mk + 1; ++k)
      for (int i = 2; i <= mi + 1; ++i)
        for (int j = 2; j <= mj + 1; ++j) {
          long q = (long)(k - 2) * mi * mj + (long)(i - 2) * mj + (j - 2);
          if (g == 1) {
            d[q] = F(B, B.dens, i + pl - 1, j + pl - 1, k + pl - 1);
          } else {
            const std::vector<double> &f = B.dens_mg[g - 1];
            int pi = 2 * mi, pj = 2 * mj;
            long ij1 = (long)(2 * k - 4) * pi * pj + (long)(2 * i - 4) * pj + (2 * j - 4);
            long ij2 = ij1 + 1, ij3 = ij1 + pj, ij4 = ij1 + pj + 1;
            long ij5 = ij1 + (long)pi * pj, ij6 = ij5 + 1, ij7 = ij5 + pj, ij8 = ij5 + pj + 1;
            d[q] = 0.125 * (f[ij1] + f[ij2] + f[ij3] + f[ij4] + f[ij5] + f[ij6] + f[ij7] + f[ij8]);
          }
        }
  }
}

void coeff(Ctx &C) {
  for (auto &B : C.b) {
    const bool lsm = C.lsm && B.dens;
    if (lsm) lsm_density(B, C.ngrd_gl, C.pl);
    int nx = B.iep - B.isp + 1, ny = B.jep - B.jsp + 1, nz = B.kep - B.ksp + 1;
    B.faz.assign(C.ngrd_gl + 1, 0);
    B.faz[1] = (long)(nx + 2) * (ny + 2) * (nz + 2);
    long pi = nx + 2, pj = ny + 2, pk = nz + 2;
    for (int g = 2; g <= C.ngrd_gl; ++g) {
      int gl = g > B.ngrid ? B.ngrid : g;
      long mi = level_n(nx, gl), mj = level_n(ny, gl), mk = level_n(nz, gl);
      B.faz[g] = B.faz[g - 1] + mi * mj * mk + 8 * (pi - 2) * (pj - 2) * (pk - 2);
      pi = mi; pj = mj; pk = mk;
    }
    long nwork = 0;
    for (int g = 1; g <= C.ngrd_gl; ++g) {
      int gl = g > B.ngrid ? B.ngrid : g;
      long mi = level_n(nx, gl), mj = level_n(ny, gl), mk = level_n(nz, gl);
      nwork += mi * mj * mk + 8 * (mi - 2) * (mj - 2) * (mk - 2);
    }
    B.cof.assign(nwork + 1, 0.0);
    for (int g = 1; g <= C.ngrd_gl; ++g) {
      int gl = g > B.ngrid ? B.ngrid : g;
      int mi = level_n(nx, gl), mj = level_n(ny, gl), mk = level_n(nz, gl);
      double ndx = B.d.dx * (double)(1 << (gl - 1));
      double ndy = B.d.dy * (double)(1 << (gl - 1));
      double ndz = B.d.dz * (double)(1 << (gl - 1));
      double dxx = ndx * ndx, dyy = ndy * ndy, dzz = ndz * ndz;
      long cnt = B.faz[g] - (long)mi * mj * mk;
      for (int k = 1; k <= mk; ++k)
        for (int i = 1; i <= mi; ++i)
          for (int j = 1; j <= mj; ++j)
            B.cof[cnt + (long)(k - 1) * mi * mj + (long)(i - 1) * mj + j] = 0.0;
      long incr = (long)(mi - 2) * (mj - 2) * (mk - 2);
      for (int k = 2; k <= mk - 1; ++k)
        for (int i = 2; i <= mi - 1; ++i)
          for (int j = 2; j <= mj - 1; ++j) {
            long ijk = B.faz[g] + (long)(k - 2) * (mi - 2) * (mj - 2) + (long)(i - 2) * (mj - 2) + (j - 1);
            double aw, ae, as, an, ab, at;
            if (lsm) {
              /* mgsolver.for:120-182: face densities within the block (a
               * boundary cell uses its own), coefficients scaled by the
               * block's fine spacings on every level */
              const std::vector<double> &d = B.dens_mg[g];
              long mi2 = mi - 2, mj2 = mj - 2;
              long q = (long)(k - 2) * mi2 * mj2 + (long)(i - 2) * mj2 + (j - 2);
              double dc = d[q];
              double densim12 = i == 2 ? dc : 0.5 * (dc + d[q - mj2]);
              double densip12 = i == mi - 1 ? dc : 0.5 * (dc + d[q + mj2]);
              double densjm12 = j == 2 ? dc : 0.5 * (dc + d[q - 1]);
              double densjp12 = j == mj - 1 ? dc : 0.5 * (dc + d[q + 1]);
              double denskm12 = k == 2 ? dc : 0.5 * (dc + d[q - mi2 * mj2]);
              double denskp12 = k == mk - 1 ? dc : 0.5 * (dc + d[q + mi2 * mj2]);
              aw = B.d.dy * B.d.dz / B.d.dx / densim12;
              ae = B.d.dy * B.d.dz / B.d.dx / densip12;
              as = B.d.dx * B.d.dz / B.d.dy / densjm12;
              an = B.d.dx * B.d.dz / B.d.dy / densjp12;
              ab = B.d.dx * B.d.dy / B.d.dz / denskm12;
              at = B.d.dx * B.d.dy / B.d.dz / denskp12;
            } else if (!B.stretched) {
              aw = 1.0 / dxx; ae = 1.0 / dxx;
              as = 1.0 / dyy; an = 1.0 / dyy;
              ab = 1.0 / dzz; at = 1.0 / dzz;
            } else {
              /* EXT: finite-volume coefficients 1/(h_c * d_face),
               * d_face = 0.5*(h_c + h_nb); equals 1/dxx when uniform. */
              const auto &wx = B.hx[gl]; const auto &wy = B.hy[gl]; const auto &wz = B.hz[gl];
              int ic = i - 1, jc = j - 1, kc = k - 1; /* 0-based ghost-inclusive */
              aw = 1.0 / (wx[ic] * (0.5 * (wx[ic] + wx[ic - 1])));
              ae = 1.0 / (wx[ic] * (0.5 * (wx[ic] + wx[ic + 1])));
              as = 1.0 / (wy[jc] * (0.5 * (wy[jc] + wy[jc - 1])));
              an = 1.0 / (wy[jc] * (0.5 * (wy[jc] + wy[jc + 1])));
              ab = 1.0 / (wz[kc] * (0.5 * (wz[kc] + wz[kc - 1])));
              at = 1.0 / (wz[kc] * (0.5 * (wz[kc] + wz[kc + 1])));
            }
            B.cof[ijk] = aw;
            B.cof[ijk + 1 * incr] = ae;
            B.cof[ijk + 2 * incr] = as;
            B.cof[ijk + 3 * incr] = an;
            B.cof[ijk + 4 * incr] = ab;
            B.cof[ijk + 5 * incr] = at;
            if (B.d.iprev < 0 && B.d.bc_west != 5 && i == 2) B.cof[ijk] = 0.0;
            if (B.d.inext < 0 && B.d.bc_east != 5 && i == mi - 1) B.cof[ijk + 1 * incr] = 0.0;
            if (B.d.jprev < 0 && B.d.bc_south != 5 && j == 2) B.cof[ijk + 2 * incr] = 0.0;
            if (B.d.jnext < 0 && B.d.bc_north != 5 && j == mj - 1) B.cof[ijk + 3 * incr] = 0.0;
            if (B.d.kprev < 0 && B.d.bc_bottom != 5 && k == 2) B.cof[ijk + 4 * incr] = 0.0;
            if (B.d.knext < 0 && B.d.bc_top != 5 && k == mk - 1) B.cof[ijk + 5 * incr] = 0.0;
            B.cof[ijk + 6 * incr] = -1.0 * (B.cof[ijk] + B.cof[ijk + 1 * incr] + B.cof[ijk + 2 * incr] +
                                            B.cof[ijk + 3 * incr] + B.cof[ijk + 4 * incr] + B.cof[ijk + 5 * incr]);
            B.cof[ijk + 7 * incr] = 0.0;
          }
    }
  }
}

struct Lev {
  int ni, nj, nk, nij;
  long nijk, base; /* base: faz(g)-ni*nj*nk, phi(i,j,k) = cof[base + (k-1)nij + (i-1)nj + j] */
};
Lev lev(Ctx &C, Blk &B, int g) {
  int gl = g > B.ngrid ? B.ngrid : g;
  Lev L;
  L.ni = level_n(B.iep - B.isp + 1, gl);
  L.nj = level_n(B.jep - B.jsp + 1, gl);
  L.nk = level_n(B.kep - B.ksp + 1, gl);
  L.nij = L.ni * L.nj;
  L.nijk = (long)L.ni * L.nj * L.nk;
  L.base = B.faz[g] - L.nijk;
  (void)C;
  return L;
}
inline long PH(const Lev &L, int i, int j, int k) {
  return L.base + (long)(k - 1) * L.nij + (long)(i - 1) * L.nj + j;
}

/* ------------------------------------------------------------------ */
/* mgbound (mgsolver.for:907-992)                                       */
/* ------------------------------------------------------------------ */
void mgbound(Ctx &C, int g) {
  for (auto &B : C.b) {
    Lev L = lev(C, B, g);
    double *c = B.cof.data();
    if (B.d.iprev < 0 && B.d.bc_west != 5)
      for (int k = 1; k <= L.nk; ++k) for (int j = 1; j <= L.nj; ++j) { long q = PH(L, 1, j, k); c[q] = c[q + L.nj]; }
    if (B.d.inext < 0 && B.d.bc_east != 5)
      for (int k = 1; k <= L.nk; ++k) for (int j = 1; j <= L.nj; ++j) { long q = PH(L, L.ni, j, k); c[q] = c[q - L.nj]; }
    if (B.d.jprev < 0 && B.d.bc_south != 5)
      for (int k = 1; k <= L.nk; ++k) for (int i = 1; i <= L.ni; ++i) { long q = PH(L, i, 1, k); c[q] = c[q + 1]; }
    if (B.d.jnext < 0 && B.d.bc_north != 5)
      for (int k = 1; k <= L.nk; ++k) for (int i = 1; i <= L.ni; ++i) { long q = PH(L, i, L.nj, k); c[q] = c[q - 1]; }
    if (B.d.kprev < 0 && B.d.bc_bottom != 5)
      for (int j = 1; j <= L.nj; ++j) for (int i = 1; i <= L.ni; ++i) { long q = PH(L, i, j, 1); c[q] = c[q + L.nij]; }
    if (B.d.knext < 0 && B.d.bc_top != 5)
      for (int j = 1; j <= L.nj; ++j) for (int i = 1; i <= L.ni; ++i) { long q = PH(L, i, j, L.nk); c[q] = c[q - L.nij]; }
  }
}

/* ------------------------------------------------------------------ */
/* exchbc_mgpp (exchangepp.for:4768-5383), same-rank branches.           */
/* ------------------------------------------------------------------ */
void exchbc_mgpp(Ctx &C, int g) {
  for (int ax = 0; ax < 3; ++ax) {
    /* pack (and the in-block copy of a block alone along the axis) */
    for (auto &B : C.b) {
      int bcp = ax == 0 ? B.d.bc_west : ax == 1 ? B.d.bc_south : B.d.bc_bottom;
      int bcn = ax == 0 ? B.d.bc_east : ax == 1 ? B.d.bc_north : B.d.bc_top;
      if (!(bcp == 5 || bcn == 5)) continue;
      int prev = ax == 0 ? B.d.iprev : ax == 1 ? B.d.jprev : B.d.kprev;
      int next = ax == 0 ? B.d.inext : ax == 1 ? B.d.jnext : B.d.knext;
      int perp = ax == 0 ? B.d.per_ip : ax == 1 ? B.d.per_jp : B.d.per_kp;
      int pern = ax == 0 ? B.d.per_in : ax == 1 ? B.d.per_jn : B.d.per_kn;
      Lev L = lev(C, B, g);
      double *c = B.cof.data();
      int n = ax == 0 ? L.ni : ax == 1 ? L.nj : L.nk;
      /* plane iterator over the two other axes, reference buffer order */
      auto cell = [&](int a, int s, int t) -> long {
        /* a: index along ax; (s,t) the other two axes in buffer order */
        if (ax == 0) return PH(L, a, s, t);        /* ijk=(k-1)*nj+j : s=j,t=k */
        if (ax == 1) return PH(L, s, a, t);        /* ijk=(k-1)*ni+i : s=i,t=k */
        return PH(L, t, s, a);                     /* ijk=(i-1)*nj+j : s=j,t=i */
      };
      int n1 = ax == 0 ? L.nj : ax == 1 ? L.ni : L.nj;
      int n2 = ax == 0 ? L.nk : ax == 1 ? L.nk : L.ni;
      if (prev < 0) {
        if (next < 0) {
          for (int t = 1; t <= n2; ++t) for (int s = 1; s <= n1; ++s) c[cell(1, s, t)] = c[cell(n - 1, s, t)];
        } else {
          Blk &P = C.b[C.indid.at(perp)];
          P.recvb_p1.assign((size_t)n1 * n2 + 1, 0.0);
          for (int t = 1; t <= n2; ++t) for (int s = 1; s <= n1; ++s) P.recvb_p1[(size_t)(t - 1) * n1 + s] = c[cell(2, s, t)];
        }
      }
      if (next < 0) {
        if (prev < 0) {
          for (int t = 1; t <= n2; ++t) for (int s = 1; s <= n1; ++s) c[cell(n, s, t)] = c[cell(2, s, t)];
        } else {
          Blk &P = C.b[C.indid.at(pern)];
          P.recvb_m1.assign((size_t)n1 * n2 + 1, 0.0);
          for (int t = 1; t <= n2; ++t) for (int s = 1; s <= n1; ++s) P.recvb_m1[(size_t)(t - 1) * n1 + s] = c[cell(n - 1, s, t)];
        }
      }
    }
    /* unpack */
    for (auto &B : C.b) {
      int bcp = ax == 0 ? B.d.bc_west : ax == 1 ? B.d.bc_south : B.d.bc_bottom;
      int bcn = ax == 0 ? B.d.bc_east : ax == 1 ? B.d.bc_north : B.d.bc_top;
      if (!(bcp == 5 || bcn == 5)) continue;
      int prev = ax == 0 ? B.d.iprev : ax == 1 ? B.d.jprev : B.d.kprev;
      int next = ax == 0 ? B.d.inext : ax == 1 ? B.d.jnext : B.d.knext;
      Lev L = lev(C, B, g);
      double *c = B.cof.data();
      int n = ax == 0 ? L.ni : ax == 1 ? L.nj : L.nk;
      auto cell = [&](int a, int s, int t) -> long {
        if (ax == 0) return PH(L, a, s, t);
        if (ax == 1) return PH(L, s, a, t);
        return PH(L, t, s, a);
      };
      int n1 = ax == 0 ? L.nj : ax == 1 ? L.ni : L.nj;
      int n2 = ax == 0 ? L.nk : ax == 1 ? L.nk : L.ni;
      if (prev < 0 && next >= 0)
        for (int t = 1; t <= n2; ++t) for (int s = 1; s <= n1; ++s) c[cell(1, s, t)] = B.recvb_m1[(size_t)(t - 1) * n1 + s];
      if (next < 0 && prev >= 0)
        for (int t = 1; t <= n2; ++t) for (int s = 1; s <= n1; ++s) c[cell(n, s, t)] = B.recvb_p1[(size_t)(t - 1) * n1 + s];
    }
  }
}

/* ------------------------------------------------------------------ */
/* exchangepp (exchangepp.for:2-4766), same-level same-rank branches.   */
/* Per sync_dir: every block packs (faces; in the z pass also corners   */
/* and edges) into its neighbours' receive buffers, then every block    */
/* unpacks: prev face, next face, then prev corners 1-4, prev edges    */
/* 1-6, next corners 1-4, next edges 1-6.  Then mgbound, exchbc_mgpp.   */
/* ------------------------------------------------------------------ */
/* ------------------------------------------------------------------ */
/* exchangepp with LMR (exchangepp.for:43-4763), single-rank branches:  */
/* per sync_dir every block packs into its neighbours' receive buffers  */
/* by the three cases of rdv(me, g) against rdv(neighbour, g), then     */
/* every block unpacks.  Equal: the copies above.  Sender finer: the    */
/* 8-cell average of the two layers next to the receiver (faces         */
/* 0.125*(...) with the tangential axes in buffer order before the      */
/* normal, exchangepp.for:163-172; corners and edges (...)/8.0 in j, i, */
/* k order, :448-452, :652-656).  Sender coarser: a face cell goes to   */
/* the four fine buffer entries as 2*phi (:174-187), a corner or edge   */
/* cell as the trilinear (27, 9, 9, 3, 9, 3, 3, 1)/64 blend toward the  */
/* receiver (:454-460, :658-669).  Unpack: a finer receiver takes       */
/* (recv + 3 phi(1 in) - phi(2 in))/4 on its whole face plane           */
/* (:4046-4056), a coarser one copies the interior of the plane         */
/* (:4057-4063), corners and edges are copies (:4433-4755).             */
/* ------------------------------------------------------------------ */
/* cell of the face plane of sync_dir sd: a along the normal, (s, t) the
 * buffer's axes (ijk = (t-1)*ns1 + s): sd 1 (j, k), sd 2 (i, k), sd 3 (j, i) */
inline long face_cell(const Lev &L, int sd, int a, int s, int t) {
  if (sd == 1) return PH(L, a, s, t);
  if (sd == 2) return PH(L, s, a, t);
  return PH(L, t, s, a);
}
/* the interior index along an axis next to a neighbour in direction e
 * (-1: the low side, 2; +1: the high side, n-1) and the first of the two
 * layers next to it (2 or n-2) */
inline int near_cell(int e, int n) { return e < 0 ? 2 : n - 1; }
inline int near_pair(int e, int n) { return e < 0 ? 2 : n - 2; }

void exchangepp_lmr(Ctx &C, int g) {
  for (int sd = 1; sd <= 3; ++sd) {
    /* pack */
    for (auto &B : C.b) {
      Lev L = lev(C, B, g);
      double *fi = B.cof.data();
      const int ni = L.ni, nj = L.nj, nk = L.nk, nij = L.nij;
      const int nn3[3] = {ni, nj, nk};
      const int cprev = sd == 1 ? B.d.iprev : sd == 2 ? B.d.jprev : B.d.kprev;
      const int cnext = sd == 1 ? B.d.inext : sd == 2 ? B.d.jnext : B.d.knext;
      const int ns1 = sd == 2 ? ni : nj, ns2 = sd == 1 ? nk : sd == 2 ? nk : ni;
      const int nd = sd == 1 ? ni : sd == 2 ? nj : nk;
      const int me = B.rdv[g];
      /* coarsened counts of a finer sender (exchangepp.for:63-72) */
      auto coarse_n = [&](int n) { return B.rdiv == 1 ? n : (n - 2) / 2 + 2; };
      const int nsc1 = coarse_n(ns1), nsc2 = coarse_n(ns2);
      const int nsr1 = 2 * (ns1 - 2) + 2, nsr2 = 2 * (ns2 - 2) + 2;
      auto pack_face = [&](Blk &N, std::vector<double> &R, bool prev) {
        const int nb_ = N.rdv[g];
        if (me == nb_) {
          R.assign((size_t)ns1 * ns2 + 1, g_lmr_ring);
          const int a = prev ? 2 : nd - 1;
          for (int t = 1; t <= ns2; ++t) for (int s = 1; s <= ns1; ++s)
            R[(size_t)(t - 1) * ns1 + s] = fi[face_cell(L, sd, a, s, t)];
        } else if (me > nb_) {
          R.assign((size_t)nsc1 * nsc2 + 1, g_lmr_ring);
          const int a = prev ? 2 : nd - 2;
          for (int t = 2; t <= nsc2 - 1; ++t) for (int s = 2; s <= nsc1 - 1; ++s) {
            const int s0 = 2 * s - 2, t0 = 2 * t - 2;
            R[(size_t)(t - 1) * nsc1 + s] =
                0.125 * (fi[face_cell(L, sd, a, s0, t0)] + fi[face_cell(L, sd, a, s0 + 1, t0)] +
                         fi[face_cell(L, sd, a, s0, t0 + 1)] + fi[face_cell(L, sd, a, s0 + 1, t0 + 1)] +
                         fi[face_cell(L, sd, a + 1, s0, t0)] + fi[face_cell(L, sd, a + 1, s0 + 1, t0)] +
                         fi[face_cell(L, sd, a + 1, s0, t0 + 1)] + fi[face_cell(L, sd, a + 1, s0 + 1, t0 + 1)]);
          }
        } else {
          R.assign((size_t)nsr1 * nsr2 + 1, g_lmr_ring);
          const int a = prev ? 2 : nd - 1;
          for (int tc = 2; tc <= ns2 - 1; ++tc) for (int sc = 2; sc <= ns1 - 1; ++sc) {
            const double v = 2.0 * fi[face_cell(L, sd, a, sc, tc)];
            for (int dt = 0; dt < 2; ++dt) for (int ds = 0; ds < 2; ++ds)
              R[(size_t)(2 * tc - 2 + dt - 1) * nsr1 + (2 * sc - 2 + ds)] = v;
          }
        }
      };
      if (cprev >= 0) { Blk &N = C.b[C.indid.at(cprev)]; pack_face(N, N.recvb_p1, true); }
      if (cnext >= 0) { Blk &N = C.b[C.indid.at(cnext)]; pack_face(N, N.recvb_m1, false); }
      if (sd != 3) continue;
      /* the value sent toward a corner or edge neighbour N in direction e
       * (e[a] = 0 along an edge's axis, where q is the index along it) */
      auto avg8 = [&](int i0, int j0, int k0) {
        const long l = PH(L, i0, j0, k0);
        return (fi[l] + fi[l + 1] + fi[l + nj] + fi[l + 1 + nj] + fi[l + nij] + fi[l + 1 + nij] + fi[l + nj + nij] +
                fi[l + 1 + nj + nij]) / 8.0;
      };
      auto tri = [&](int i, int j, int k, int ei, int ej, int ek) {
        const long l = PH(L, i, j, k);
        const long dj = ej, di = (long)ei * nj, dk = (long)ek * nij;
        return (27.0 * fi[l] + 9.0 * fi[l + dj] + 9.0 * fi[l + di] + 3.0 * fi[l + di + dj] + 9.0 * fi[l + dk] +
                3.0 * fi[l + dj + dk] + 3.0 * fi[l + di + dk] + 1.0 * fi[l + di + dj + dk]) / 64.0;
      };
      /* corners (exchangepp.for:439-633, 1387-1580): prev #1..4 at z-1,
       * next #1..4 at z+1 */
      const int cpx[4] = {-1, -1, +1, +1}, cpy[4] = {-1, +1, +1, -1};
      const int cnx[4] = {+1, +1, -1, -1}, cny[4] = {+1, -1, -1, +1};
      for (int side = 0; side < 2; ++side)
        for (int q = 0; q < 4; ++q) {
          const int id = side ? B.d.cornext[q] : B.d.corprev[q];
          if (id < 0) continue;
          Blk &N = C.b[C.indid.at(id)];
          const int e[3] = {side ? cnx[q] : cpx[q], side ? cny[q] : cpy[q], side ? +1 : -1};
          double v;
          if (me == N.rdv[g]) v = fi[PH(L, near_cell(e[0], ni), near_cell(e[1], nj), near_cell(e[2], nk))];
          else if (me > N.rdv[g]) v = avg8(near_pair(e[0], ni), near_pair(e[1], nj), near_pair(e[2], nk));
          else v = tri(near_cell(e[0], ni), near_cell(e[1], nj), near_cell(e[2], nk), e[0], e[1], e[2]);
          (side ? N.rcm : N.rcp)[q + 1] = v;
        }
      /* edges (exchangepp.for:640-1086, 1587-2036): prev #1..6, next #1..6 */
      const int epd[6][3] = {{-1, 0, -1}, {0, +1, -1}, {+1, 0, -1}, {0, -1, -1}, {-1, -1, 0}, {-1, +1, 0}};
      const int end_[6][3] = {{+1, 0, +1}, {0, -1, +1}, {-1, 0, +1}, {0, +1, +1}, {+1, +1, 0}, {+1, -1, 0}};
      for (int side = 0; side < 2; ++side)
        for (int q = 0; q < 6; ++q) {
          const int id = side ? B.d.edgnext[q] : B.d.edgprev[q];
          if (id < 0) continue;
          Blk &N = C.b[C.indid.at(id)];
          const int *e = side ? end_[q] : epd[q];
          const int ax = e[0] == 0 ? 0 : e[1] == 0 ? 1 : 2;  /* the edge's axis */
          const int n = nn3[ax];
          std::vector<double> &R = side ? N.rem[q + 1] : N.rep[q + 1];
          if (me == N.rdv[g]) {
            R.assign(n + 1, g_lmr_ring);
            for (int nn = 2; nn <= n - 1; ++nn) {
              int c[3] = {near_cell(e[0], ni), near_cell(e[1], nj), near_cell(e[2], nk)};
              c[ax] = nn;
              R[nn] = fi[PH(L, c[0], c[1], c[2])];
            }
          } else if (me > N.rdv[g]) {
            const int nc = coarse_n(n);
            R.assign(nc + 1, g_lmr_ring);
            for (int nn = 2; nn <= nc - 1; ++nn) {
              int c[3] = {near_pair(e[0], ni), near_pair(e[1], nj), near_pair(e[2], nk)};
              c[ax] = 2 * nn - 2;
              R[nn] = avg8(c[0], c[1], c[2]);
            }
          } else {
            const int nf = 2 * (n - 2) + 2;
            R.assign(nf + 1, g_lmr_ring);
            for (int nn = 2; nn <= n - 1; ++nn) {
              int c[3] = {near_cell(e[0], ni), near_cell(e[1], nj), near_cell(e[2], nk)};
              c[ax] = nn;
              for (int h = 0; h < 2; ++h) {
                int ee[3] = {e[0], e[1], e[2]};
                ee[ax] = h ? +1 : -1;
                R[2 * nn - 2 + h] = tri(c[0], c[1], c[2], ee[0], ee[1], ee[2]);
              }
            }
          }
        }
    }
    /* unpack */
    for (auto &B : C.b) {
      Lev L = lev(C, B, g);
      double *fi = B.cof.data();
      const int ni = L.ni, nj = L.nj, nk = L.nk;
      const int cprev = sd == 1 ? B.d.iprev : sd == 2 ? B.d.jprev : B.d.kprev;
      const int cnext = sd == 1 ? B.d.inext : sd == 2 ? B.d.jnext : B.d.knext;
      const int ns1 = sd == 2 ? ni : nj, ns2 = sd == 1 ? nk : sd == 2 ? nk : ni;
      const int nd = sd == 1 ? ni : sd == 2 ? nj : nk;
      const int me = B.rdv[g];
      auto unpack_face = [&](int nbr, const std::vector<double> &R, bool prev) {
        const int nb_ = C.b[C.indid.at(nbr)].rdv[g];
        const int a = prev ? 1 : nd, a1 = prev ? 2 : nd - 1, a2 = prev ? 3 : nd - 2;
        if (me == nb_) {
          for (int t = 1; t <= ns2; ++t) for (int s = 1; s <= ns1; ++s)
            fi[face_cell(L, sd, a, s, t)] = R[(size_t)(t - 1) * ns1 + s];
        } else if (me > nb_) {
          for (int t = 1; t <= ns2; ++t) for (int s = 1; s <= ns1; ++s)
            fi[face_cell(L, sd, a, s, t)] =
                (R[(size_t)(t - 1) * ns1 + s] + 3.0 * fi[face_cell(L, sd, a1, s, t)] - fi[face_cell(L, sd, a2, s, t)]) /
                4.0;
        } else {
          for (int t = 2; t <= ns2 - 1; ++t) for (int s = 2; s <= ns1 - 1; ++s)
            fi[face_cell(L, sd, a, s, t)] = R[(size_t)(t - 1) * ns1 + s];
        }
      };
      if (cprev >= 0) unpack_face(cprev, B.recvb_m1, true);
      if (cnext >= 0) unpack_face(cnext, B.recvb_p1, false);
      if (sd != 3) continue;
      const int upi[4] = {1, 1, ni, ni}, upj[4] = {1, nj, nj, 1};
      for (int q = 0; q < 4; ++q)
        if (B.d.corprev[q] >= 0) fi[PH(L, upi[q], upj[q], 1)] = B.rcm[q + 1];
      if (B.d.edgprev[0] >= 0) for (int nn = 2; nn <= nj - 1; ++nn) fi[PH(L, 1, nn, 1)] = B.rem[1][nn];
      if (B.d.edgprev[1] >= 0) for (int nn = 2; nn <= ni - 1; ++nn) fi[PH(L, nn, nj, 1)] = B.rem[2][nn];
      if (B.d.edgprev[2] >= 0) for (int nn = 2; nn <= nj - 1; ++nn) fi[PH(L, ni, nn, 1)] = B.rem[3][nn];
      if (B.d.edgprev[3] >= 0) for (int nn = 2; nn <= ni - 1; ++nn) fi[PH(L, nn, 1, 1)] = B.rem[4][nn];
      if (B.d.edgprev[4] >= 0) for (int nn = 2; nn <= nk - 1; ++nn) fi[PH(L, 1, 1, nn)] = B.rem[5][nn];
      if (B.d.edgprev[5] >= 0) for (int nn = 2; nn <= nk - 1; ++nn) fi[PH(L, 1, nj, nn)] = B.rem[6][nn];
      const int uni[4] = {ni, ni, 1, 1}, unj[4] = {nj, 1, 1, nj};
      for (int q = 0; q < 4; ++q)
        if (B.d.cornext[q] >= 0) fi[PH(L, uni[q], unj[q], nk)] = B.rcp[q + 1];
      if (B.d.edgnext[0] >= 0) for (int nn = 2; nn <= nj - 1; ++nn) fi[PH(L, ni, nn, nk)] = B.rep[1][nn];
      if (B.d.edgnext[1] >= 0) for (int nn = 2; nn <= ni - 1; ++nn) fi[PH(L, nn, 1, nk)] = B.rep[2][nn];
      if (B.d.edgnext[2] >= 0) for (int nn = 2; nn <= nj - 1; ++nn) fi[PH(L, 1, nn, nk)] = B.rep[3][nn];
      if (B.d.edgnext[3] >= 0) for (int nn = 2; nn <= ni - 1; ++nn) fi[PH(L, nn, nj, nk)] = B.rep[4][nn];
      if (B.d.edgnext[4] >= 0) for (int nn = 2; nn <= nk - 1; ++nn) fi[PH(L, ni, nj, nn)] = B.rep[5][nn];
      if (B.d.edgnext[5] >= 0) for (int nn = 2; nn <= nk - 1; ++nn) fi[PH(L, ni, 1, nn)] = B.rep[6][nn];
    }
  }
  mgbound(C, g);
  if (C.periodic) exchbc_mgpp(C, g);
}

void exchangepp(Ctx &C, int g) {
  if (C.lmr) { exchangepp_lmr(C, g); return; }
  for (int sd = 1; sd <= 3; ++sd) {
    for (auto &B : C.b) {
      Lev L = lev(C, B, g);
      double *fi = B.cof.data();
      int cprev = sd == 1 ? B.d.iprev : sd == 2 ? B.d.jprev : B.d.kprev;
      int cnext = sd == 1 ? B.d.inext : sd == 2 ? B.d.jnext : B.d.knext;
      int ns1 = sd == 1 ? L.nj : sd == 2 ? L.ni : L.nj;
      int ns2 = sd == 1 ? L.nk : sd == 2 ? L.nk : L.ni;
      auto face = [&](int a, int s, int t) -> long {
        if (sd == 1) return PH(L, a, s, t);
        if (sd == 2) return PH(L, s, a, t);
        return PH(L, t, s, a);
      };
      int nd = sd == 1 ? L.ni : sd == 2 ? L.nj : L.nk;
      if (cprev >= 0) {
        Blk &P = C.b[C.indid.at(cprev)];
        P.recvb_p1.assign((size_t)ns1 * ns2 + 1, 0.0);
        for (int t = 1; t <= ns2; ++t) for (int s = 1; s <= ns1; ++s)
          P.recvb_p1[(size_t)(t - 1) * ns1 + s] = fi[face(2, s, t)];
      }
      if (sd == 3) {
        /* previous corners (exchangepp.for:439-633) */
        const int cpi[4] = {2, 2, L.ni - 1, L.ni - 1}, cpj[4] = {2, L.nj - 1, L.nj - 1, 2};
        for (int q = 0; q < 4; ++q)
          if (B.d.corprev[q] >= 0) C.b[C.indid.at(B.d.corprev[q])].rcp[q + 1] = fi[PH(L, cpi[q], cpj[q], 2)];
        /* previous edges (exchangepp.for:640-1086) */
        if (B.d.edgprev[0] >= 0) { auto &R = C.b[C.indid.at(B.d.edgprev[0])].rep[1]; R.assign(L.nj + 1, 0.0); for (int nn = 2; nn <= L.nj - 1; ++nn) R[nn] = fi[PH(L, 2, nn, 2)]; }
        if (B.d.edgprev[1] >= 0) { auto &R = C.b[C.indid.at(B.d.edgprev[1])].rep[2]; R.assign(L.ni + 1, 0.0); for (int nn = 2; nn <= L.ni - 1; ++nn) R[nn] = fi[PH(L, nn, L.nj - 1, 2)]; }
        if (B.d.edgprev[2] >= 0) { auto &R = C.b[C.indid.at(B.d.edgprev[2])].rep[3]; R.assign(L.nj + 1, 0.0); for (int nn = 2; nn <= L.nj - 1; ++nn) R[nn] = fi[PH(L, L.ni - 1, nn, 2)]; }
        if (B.d.edgprev[3] >= 0) { auto &R = C.b[C.indid.at(B.d.edgprev[3])].rep[4]; R.assign(L.ni + 1, 0.0); for (int nn = 2; nn <= L.ni - 1; ++nn) R[nn] = fi[PH(L, nn, 2, 2)]; }
        if (B.d.edgprev[4] >= 0) { auto &R = C.b[C.indid.at(B.d.edgprev[4])].rep[5]; R.assign(L.nk + 1, 0.0); for (int nn = 2; nn <= L.nk - 1; ++nn) R[nn] = fi[PH(L, 2, 2, nn)]; }
        if (B.d.edgprev[5] >= 0) { auto &R = C.b[C.indid.at(B.d.edgprev[5])].rep[6]; R.assign(L.nk + 1, 0.0); for (int nn = 2; nn <= L.nk - 1; ++nn) R[nn] = fi[PH(L, 2, L.nj - 1, nn)]; }
      }
      if (cnext >= 0) {
        Blk &N = C.b[C.indid.at(cnext)];
        N.recvb_m1.assign((size_t)ns1 * ns2 + 1, 0.0);
        for (int t = 1; t <= ns2; ++t) for (int s = 1; s <= ns1; ++s)
          N.recvb_m1[(size_t)(t - 1) * ns1 + s] = fi[face(nd - 1, s, t)];
      }
      if (sd == 3) {
        /* next corners (exchangepp.for:1387-1580) */
        const int cni[4] = {L.ni - 1, L.ni - 1, 2, 2}, cnj[4] = {L.nj - 1, 2, 2, L.nj - 1};
        for (int q = 0; q < 4; ++q)
          if (B.d.cornext[q] >= 0) C.b[C.indid.at(B.d.cornext[q])].rcm[q + 1] = fi[PH(L, cni[q], cnj[q], L.nk - 1)];
        /* next edges (exchangepp.for:1587-2036) */
        if (B.d.edgnext[0] >= 0) { auto &R = C.b[C.indid.at(B.d.edgnext[0])].rem[1]; R.assign(L.nj + 1, 0.0); for (int nn = 2; nn <= L.nj - 1; ++nn) R[nn] = fi[PH(L, L.ni - 1, nn, L.nk - 1)]; }
        if (B.d.edgnext[1] >= 0) { auto &R = C.b[C.indid.at(B.d.edgnext[1])].rem[2]; R.assign(L.ni + 1, 0.0); for (int nn = 2; nn <= L.ni - 1; ++nn) R[nn] = fi[PH(L, nn, 2, L.nk - 1)]; }
        if (B.d.edgnext[2] >= 0) { auto &R = C.b[C.indid.at(B.d.edgnext[2])].rem[3]; R.assign(L.nj + 1, 0.0); for (int nn = 2; nn <= L.nj - 1; ++nn) R[nn] = fi[PH(L, 2, nn, L.nk - 1)]; }
        if (B.d.edgnext[3] >= 0) { auto &R = C.b[C.indid.at(B.d.edgnext[3])].rem[4]; R.assign(L.ni + 1, 0.0); for (int nn = 2; nn <= L.ni - 1; ++nn) R[nn] = fi[PH(L, nn, L.nj - 1, L.nk - 1)]; }
        if (B.d.edgnext[4] >= 0) { auto &R = C.b[C.indid.at(B.d.edgnext[4])].rem[5]; R.assign(L.nk + 1, 0.0); for (int nn = 2; nn <= L.nk - 1; ++nn) R[nn] = fi[PH(L, L.ni - 1, L.nj - 1, nn)]; }
        if (B.d.edgnext[5] >= 0) { auto &R = C.b[C.indid.at(B.d.edgnext[5])].rem[6]; R.assign(L.nk + 1, 0.0); for (int nn = 2; nn <= L.nk - 1; ++nn) R[nn] = fi[PH(L, L.ni - 1, 2, nn)]; }
      }
    }
    /* unpack (exchangepp.for:3996-4755) */
    for (auto &B : C.b) {
      Lev L = lev(C, B, g);
      double *fi = B.cof.data();
      int cprev = sd == 1 ? B.d.iprev : sd == 2 ? B.d.jprev : B.d.kprev;
      int cnext = sd == 1 ? B.d.inext : sd == 2 ? B.d.jnext : B.d.knext;
      int ns1 = sd == 1 ? L.nj : sd == 2 ? L.ni : L.nj;
      int ns2 = sd == 1 ? L.nk : sd == 2 ? L.nk : L.ni;
      auto face = [&](int a, int s, int t) -> long {
        if (sd == 1) return PH(L, a, s, t);
        if (sd == 2) return PH(L, s, a, t);
        return PH(L, t, s, a);
      };
      int nd = sd == 1 ? L.ni : sd == 2 ? L.nj : L.nk;
      if (cprev >= 0)
        for (int t = 1; t <= ns2; ++t) for (int s = 1; s <= ns1; ++s) fi[face(1, s, t)] = B.recvb_m1[(size_t)(t - 1) * ns1 + s];
      if (cnext >= 0)
        for (int t = 1; t <= ns2; ++t) for (int s = 1; s <= ns1; ++s) fi[face(nd, s, t)] = B.recvb_p1[(size_t)(t - 1) * ns1 + s];
      if (sd == 3) {
        const int upi[4] = {1, 1, L.ni, L.ni}, upj[4] = {1, L.nj, L.nj, 1};
        for (int q = 0; q < 4; ++q)
          if (B.d.corprev[q] >= 0) fi[PH(L, upi[q], upj[q], 1)] = B.rcm[q + 1];
        if (B.d.edgprev[0] >= 0) for (int nn = 2; nn <= L.nj - 1; ++nn) fi[PH(L, 1, nn, 1)] = B.rem[1][nn];
        if (B.d.edgprev[1] >= 0) for (int nn = 2; nn <= L.ni - 1; ++nn) fi[PH(L, nn, L.nj, 1)] = B.rem[2][nn];
        if (B.d.edgprev[2] >= 0) for (int nn = 2; nn <= L.nj - 1; ++nn) fi[PH(L, L.ni, nn, 1)] = B.rem[3][nn];
        if (B.d.edgprev[3] >= 0) for (int nn = 2; nn <= L.ni - 1; ++nn) fi[PH(L, nn, 1, 1)] = B.rem[4][nn];
        if (B.d.edgprev[4] >= 0) for (int nn = 2; nn <= L.nk - 1; ++nn) fi[PH(L, 1, 1, nn)] = B.rem[5][nn];
        if (B.d.edgprev[5] >= 0) for (int nn = 2; nn <= L.nk - 1; ++nn) fi[PH(L, 1, L.nj, nn)] = B.rem[6][nn];
        const int uni[4] = {L.ni, L.ni, 1, 1}, unj[4] = {L.nj, 1, 1, L.nj};
        for (int q = 0; q < 4; ++q)
          if (B.d.cornext[q] >= 0) fi[PH(L, uni[q], unj[q], L.nk)] = B.rcp[q + 1];
        if (B.d.edgnext[0] >= 0) for (int nn = 2; nn <= L.nj - 1; ++nn) fi[PH(L, L.ni, nn, L.nk)] = B.rep[1][nn];
        if (B.d.edgnext[1] >= 0) for (int nn = 2; nn <= L.ni - 1; ++nn) fi[PH(L, nn, 1, L.nk)] = B.rep[2][nn];
        if (B.d.edgnext[2] >= 0) for (int nn = 2; nn <= L.nj - 1; ++nn) fi[PH(L, 1, nn, L.nk)] = B.rep[3][nn];
        if (B.d.edgnext[3] >= 0) for (int nn = 2; nn <= L.ni - 1; ++nn) fi[PH(L, nn, L.nj, L.nk)] = B.rep[4][nn];
        if (B.d.edgnext[4] >= 0) for (int nn = 2; nn <= L.nk - 1; ++nn) fi[PH(L, L.ni, L.nj, nn)] = B.rep[5][nn];
        if (B.d.edgnext[5] >= 0) for (int nn = 2; nn <= L.nk - 1; ++nn) fi[PH(L, L.ni, 1, nn)] = B.rep[6][nn];
      }
    }
  }
  mgbound(C, g);
  if (C.periodic) exchbc_mgpp(C, g);
}

/* ------------------------------------------------------------------ */
/* mgrelax (mgsolver.for:371-617)                                        */
/* ------------------------------------------------------------------ */
void mgrelax(Ctx &C, int g, int it) {
  for (int itr = 1; itr <= it; ++itr) {
    par_blocks((int)C.b.size(), [&](int ib_) { Blk &B = C.b[ib_];
      Lev L = lev(C, B, g);
      int ni = L.ni, nj = L.nj, nk = L.nk, nij = L.nij;
      long nij2 = (long)(ni - 2) * (nj - 2);
      long incr = (long)(ni - 2) * (nj - 2) * (nk - 2);
      double *cf = B.cof.data();
      long fz = B.faz[g];
      auto W = [&](int i, int j, int k) -> long { return fz + (long)(k - 2) * nij2 + (long)(i - 2) * (nj - 2) + (j - 1); };
      if (C.mg_itrsch == 1 || C.mg_itrsch == 3) {
        for (int pass = 0; pass < (C.mg_itrsch == 3 ? 2 : 1); ++pass)
          for (int k = 2; k <= nk - 1; ++k)
            for (int j = 2; j <= nj - 1; ++j)
              for (int i = 2; i <= ni - 1; ++i) {
                if (C.mg_itrsch == 3 && ((i + j + k) % 2) != pass) continue;
                long ph = PH(L, i, j, k);
                long w = W(i, j, k);
                cf[ph] = ((cf[w + 7 * incr] -
                           (cf[w] * cf[ph - nj] + cf[w + incr] * cf[ph + nj] + cf[w + 2 * incr] * cf[ph - 1] +
                            cf[w + 3 * incr] * cf[ph + 1] + cf[w + 4 * incr] * cf[ph - nij] +
                            cf[w + 5 * incr] * cf[ph + nij])) /
                          cf[w + 6 * incr]);
              }
      } else if (C.mg_itrsch == 2) {
        int ngg = std::max({ni, nj, nk}) + 2;
        std::vector<double> a(ngg + 1, 0.0), c(ngg + 1, 0.0);
        /* j-lines */
        for (int k = 2; k <= nk - 1; ++k)
          for (int i = 2; i <= ni - 1; ++i) {
            c[1] = cf[PH(L, i, 1, k)];
            for (int j = 2; j <= nj - 1; ++j) {
              long ph = PH(L, i, j, k), w = W(i, j, k);
              double apr = 1.0 / (cf[w + 6 * incr] - cf[w + 2 * incr] * a[j - 1]);
              a[j] = cf[w + 3 * incr] * apr;
              c[j] = (cf[w + 7 * incr] - cf[w + incr] * cf[ph + nj] - cf[w] * cf[ph - nj] -
                      cf[w + 5 * incr] * cf[ph + nij] - cf[w + 4 * incr] * cf[ph - nij] -
                      cf[w + 2 * incr] * c[j - 1]) * apr;
            }
            for (int j = nj - 1; j >= 2; --j) { long ph = PH(L, i, j, k); cf[ph] = (c[j] - a[j] * cf[ph + 1]); }
          }
        /* i-lines */
        for (int k = 2; k <= nk - 1; ++k)
          for (int j = 2; j <= nj - 1; ++j) {
            c[1] = cf[PH(L, 1, j, k)];
            for (int i = 2; i <= ni - 1; ++i) {
              long ph = PH(L, i, j, k), w = W(i, j, k);
              double apr = 1.0 / (cf[w + 6 * incr] - cf[w] * a[i - 1]);
              a[i] = cf[w + incr] * apr;
              c[i] = (cf[w + 7 * incr] - cf[w + 3 * incr] * cf[ph + 1] - cf[w + 2 * incr] * cf[ph - 1] -
                      cf[w + 5 * incr] * cf[ph + nij] - cf[w + 4 * incr] * cf[ph - nij] -
                      cf[w] * c[i - 1]) * apr;
            }
            for (int i = ni - 1; i >= 2; --i) { long ph = PH(L, i, j, k); cf[ph] = (c[i] - a[i] * cf[ph + nj]); }
          }
        /* k-lines */
        for (int i = 2; i <= ni - 1; ++i)
          for (int j = 2; j <= nj - 1; ++j) {
            c[1] = cf[PH(L, i, j, 1)];
            for (int k = 2; k <= nk - 1; ++k) {
              long ph = PH(L, i, j, k), w = W(i, j, k);
              double apr = 1.0 / (cf[w + 6 * incr] - cf[w + 4 * incr] * a[k - 1]);
              a[k] = cf[w + 5 * incr] * apr;
              c[k] = (cf[w + 7 * incr] - cf[w + 3 * incr] * cf[ph + 1] - cf[w + 2 * incr] * cf[ph - 1] -
                      cf[w + incr] * cf[ph + nj] - cf[w] * cf[ph - nj] -
                      cf[w + 4 * incr] * c[k - 1]) * apr;
            }
            for (int k = nk - 1; k >= 2; --k) { long ph = PH(L, i, j, k); cf[ph] = (c[k] - a[k] * cf[ph + nij]); }
          }
      }
    });
    mgbound(C, g);
    exchangepp(C, g);
  }
}

/* ------------------------------------------------------------------ */
/* mgrestr (mgsolver.for:619-761), coarsening branch + EXT weights.     */
/* ------------------------------------------------------------------ */
void mgrestr(Ctx &C, int g) {
  par_blocks((int)C.b.size(), [&](int ib_) { Blk &B = C.b[ib_];
    Lev Lc = lev(C, B, g), Lf = lev(C, B, g - 1);
    int nic = Lc.ni, njc = Lc.nj, nkc = Lc.nk;
    long nijc2 = (long)(nic - 2) * (njc - 2), incr_c = (long)(nic - 2) * (njc - 2) * (nkc - 2);
    double *cf = B.cof.data();
    for (int k = 1; k <= nkc; ++k) for (int i = 1; i <= nic; ++i) for (int j = 1; j <= njc; ++j) cf[PH(Lc, i, j, k)] = 0.0;
    for (int k = 2; k <= nkc - 1; ++k) for (int i = 2; i <= nic - 1; ++i) for (int j = 2; j <= njc - 1; ++j)
      cf[B.faz[g] + (long)(k - 2) * nijc2 + (long)(i - 2) * (njc - 2) + (j - 1) + 7 * incr_c] = 0.0;
    int nif = Lf.ni, njf = Lf.nj, nkf = Lf.nk;
    long nijf2 = (long)(nif - 2) * (njf - 2), incr_f = (long)(nif - 2) * (njf - 2) * (nkf - 2);
    std::vector<double> resf((size_t)nif * njf * nkf, 0.0);
    auto R = [&](int i, int j, int k) -> double & { return resf[(size_t)(i - 1) + (size_t)nif * ((j - 1) + (size_t)njf * (k - 1))]; };
    for (int k = 2; k <= nkf - 1; ++k) for (int i = 2; i <= nif - 1; ++i) for (int j = 2; j <= njf - 1; ++j) {
      long ph = PH(Lf, i, j, k);
      long w = B.faz[g - 1] + (long)(k - 2) * nijf2 + (long)(i - 2) * (njf - 2) + (j - 1);
      R(i, j, k) = cf[w + 7 * incr_f] -
                   (cf[w] * cf[ph - njf] + cf[w + incr_f] * cf[ph + njf] + cf[w + 2 * incr_f] * cf[ph - 1] +
                    cf[w + 3 * incr_f] * cf[ph + 1] + cf[w + 4 * incr_f] * cf[ph - Lf.nij] +
                    cf[w + 5 * incr_f] * cf[ph + Lf.nij] + cf[w + 6 * incr_f] * cf[ph]);
    }
    int gf = g - 1, gc = g;
    for (int k = 2; k <= nkc - 1; ++k) for (int i = 2; i <= nic - 1; ++i) for (int j = 2; j <= njc - 1; ++j) {
      long su = B.faz[g] + (long)(k - 2) * nijc2 + (long)(i - 2) * (njc - 2) + (j - 1) + 7 * incr_c;
      if (g > B.ngrid) {
        /* LMR: a block past its own last level keeps its size; the rhs is
         * the residual itself (mgsolver.for:714-727) */
        cf[su] = R(i, j, k);
      } else if (!B.stretched) {
        cf[su] = 0.125 * (R(2 * i - 2, 2 * j - 2, 2 * k - 2) + R(2 * i - 1, 2 * j - 2, 2 * k - 2) +
                          R(2 * i - 2, 2 * j - 1, 2 * k - 2) + R(2 * i - 1, 2 * j - 1, 2 * k - 2) +
                          R(2 * i - 2, 2 * j - 2, 2 * k - 1) + R(2 * i - 1, 2 * j - 2, 2 * k - 1) +
                          R(2 * i - 2, 2 * j - 1, 2 * k - 1) + R(2 * i - 1, 2 * j - 1, 2 * k - 1));
      } else {
        /* EXT: volume-weighted average, s = 8 (hx_f/Hx_c)(hy_f/Hy_c)(hz_f/Hz_c),
         * s == 1.0 exactly on a uniform grid. */
        double t[8];
        int q = 0;
        for (int dk = 0; dk < 2; ++dk) for (int dj = 0; dj < 2; ++dj) for (int di = 0; di < 2; ++di) {
          int fi_ = 2 * i - 2 + di, fj = 2 * j - 2 + dj, fk = 2 * k - 2 + dk;
          double s = 8.0 * (B.hx[gf][fi_ - 1] / B.hx[gc][i - 1]) * (B.hy[gf][fj - 1] / B.hy[gc][j - 1]) *
                     (B.hz[gf][fk - 1] / B.hz[gc][k - 1]);
          t[q++] = R(fi_, fj, fk) * s;
        }
        cf[su] = 0.125 * (t[0] + t[1] + t[2] + t[3] + t[4] + t[5] + t[6] + t[7]);
      }
    }
  });
}

/* ------------------------------------------------------------------ */
/* mgcorr (mgsolver.for:763-905), coarsening branch.                     */
/* ------------------------------------------------------------------ */
void mgcorr(Ctx &C, int g) {
  par_blocks((int)C.b.size(), [&](int ib_) { Blk &B = C.b[ib_];
    Lev Lf = lev(C, B, g), Lc = lev(C, B, g + 1);
    double *cf = B.cof.data();
    if (g >= B.ngrid) {
      /* LMR: both levels have the block's last size; the correction is
       * added on every cell, ghosts included (mgsolver.for:806-818) */
      for (int kc = 1; kc <= Lc.nk; ++kc) for (int ic = 1; ic <= Lc.ni; ++ic) for (int jc = 1; jc <= Lc.nj; ++jc)
        cf[PH(Lf, ic, jc, kc)] = cf[PH(Lf, ic, jc, kc)] + cf[PH(Lc, ic, jc, kc)];
      return;
    }
    int nijf = Lf.nij, njf = Lf.nj, nijc = Lc.nij, njc = Lc.nj;
    for (int kc = 1; kc <= Lc.nk - 1; ++kc) {
      int k = 2 * kc - 1;
      for (int ic = 1; ic <= Lc.ni - 1; ++ic) {
        int i = 2 * ic - 1;
        for (int jc = 1; jc <= Lc.nj - 1; ++jc) {
          int j = 2 * jc - 1;
          long c0 = PH(Lc, ic, jc, kc), f0 = PH(Lf, i, j, k);
          const double *q = cf;
          double C000 = q[c0], C010 = q[c0 + 1], C001 = q[c0 + nijc], C011 = q[c0 + nijc + 1];
          double C100 = q[c0 + njc], C110 = q[c0 + njc + 1], C101 = q[c0 + njc + nijc], C111 = q[c0 + 1 + njc + nijc];
          cf[f0] = cf[f0] + (27.0 * C000 + 9.0 * C010 + 9.0 * C001 + 3.0 * C011 + 9.0 * C100 + 3.0 * C110 + 3.0 * C101 + 1.0 * C111) / 64.0;
          cf[f0 + njf] = cf[f0 + njf] + (9.0 * C000 + 3.0 * C010 + 3.0 * C001 + 1.0 * C011 + 27.0 * C100 + 9.0 * C110 + 9.0 * C101 + 3.0 * C111) / 64.0;
          cf[f0 + 1] = cf[f0 + 1] + (9.0 * C000 + 27.0 * C010 + 3.0 * C001 + 9.0 * C011 + 3.0 * C100 + 9.0 * C110 + 1.0 * C101 + 3.0 * C111) / 64.0;
          cf[f0 + nijf] = cf[f0 + nijf] + (9.0 * C000 + 3.0 * C010 + 27.0 * C001 + 9.0 * C011 + 3.0 * C100 + 1.0 * C110 + 9.0 * C101 + 3.0 * C111) / 64.0;
          cf[f0 + njf + 1] = cf[f0 + njf + 1] + (3.0 * C000 + 9.0 * C010 + 1.0 * C001 + 3.0 * C011 + 9.0 * C100 + 27.0 * C110 + 3.0 * C101 + 9.0 * C111) / 64.0;
          cf[f0 + nijf + njf] = cf[f0 + nijf + njf] + (3.0 * C000 + 1.0 * C010 + 9.0 * C001 + 3.0 * C011 + 9.0 * C100 + 3.0 * C110 + 27.0 * C101 + 9.0 * C111) / 64.0;
          cf[f0 + nijf + 1] = cf[f0 + nijf + 1] + (3.0 * C000 + 9.0 * C010 + 9.0 * C001 + 27.0 * C011 + 1.0 * C100 + 3.0 * C110 + 3.0 * C101 + 9.0 * C111) / 64.0;
          cf[f0 + nijf + njf + 1] = cf[f0 + nijf + njf + 1] + (1.0 * C000 + 3.0 * C010 + 3.0 * C001 + 9.0 * C011 + 3.0 * C100 + 9.0 * C110 + 9.0 * C101 + 27.0 * C111) / 64.0;
        }
      }
    }
  });
  mgbound(C, g);
}

/* ------------------------------------------------------------------ */
/* mgkcyc (mgsolver.for:224-369): copy pp/su in, V-cycle, copy pp out.   */
/* ------------------------------------------------------------------ */
void mgkcyc(Ctx &C) {
  int pl = C.pl;
  par_blocks((int)C.b.size(), [&](int ib_) { Blk &B = C.b[ib_];
    Lev L = lev(C, B, 1);
    for (int k = 1; k <= L.nk; ++k) for (int i = 1; i <= L.ni; ++i) for (int j = 1; j <= L.nj; ++j)
      B.cof[(long)(k - 1) * L.nij + (long)(i - 1) * L.nj + j] = F(B, B.pp.data(), i + pl - 1, j + pl - 1, k + pl - 1);
    long incrp = 7L * (L.ni - 2) * (L.nj - 2) * (L.nk - 2);
    for (int k = 2; k <= L.nk - 1; ++k) for (int i = 2; i <= L.ni - 1; ++i) for (int j = 2; j <= L.nj - 1; ++j)
      B.cof[B.faz[1] + (long)(k - 2) * (L.ni - 2) * (L.nj - 2) + (long)(i - 2) * (L.nj - 2) + (j - 1) + incrp] =
          F(B, B.su.data(), i + pl - 1, j + pl - 1, k + pl - 1);
  });
  int ngrd = C.ngrd_gl;
  int glevel = 1, kcycle = 1, nrel;
  std::vector<int> kount(ngrd + 1, 0);
  mgrelax(C, 1, C.irestr);
  if (ngrd != 1) {
    mgrestr(C, glevel + 1);
    for (int l = 1; l <= ngrd; ++l) kount[l] = 0;
    glevel = glevel + 1;
    nrel = C.irestr;
    for (;;) {
      if (glevel == 1) break;
      kount[glevel] = kount[glevel] + 1;
      mgrelax(C, glevel, nrel);
      if (kount[glevel] == kcycle + 1) {
        mgcorr(C, glevel - 1);
        kount[glevel] = 0;
        glevel = glevel - 1;
        nrel = C.iproln;
      } else if (glevel < ngrd) {
        mgrestr(C, glevel + 1);
        glevel = glevel + 1;
        nrel = C.irestr;
      } else {
        mgrelax(C, glevel, C.iproln);
        mgcorr(C, glevel - 1);
        nrel = C.iproln;
        glevel = ngrd - 1;
      }
    }
  }
  mgrelax(C, 1, C.iproln);
  for (auto &B : C.b) {
    Lev L = lev(C, B, 1);
    for (int k = 1; k <= L.nk; ++k) for (int i = 1; i <= L.ni; ++i) for (int j = 1; j <= L.nj; ++j)
      F(B, B.pp.data(), i + pl - 1, j + pl - 1, k + pl - 1) = B.cof[(long)(k - 1) * L.nij + (long)(i - 1) * L.nj + j];
  }
}

/* ------------------------------------------------------------------ */
/* Field halos exchange(op) for op 1..4 (exchange.for:2-23): periodic   */
/* exchange_bc (exchange_bc.for:2-841) then exchange_smlvl              */
/* (exchange.for:343-2498).  Layers ly = 0..nly, nly = pl_ex for u, v, w */
/* and 0 for p (exchange.for:14-20).                                    */
/* ------------------------------------------------------------------ */
double *field_of(Blk &B, int op) {
  return op == 1 ? B.u : op == 2 ? B.v : op == 3 ? B.w : op == 44 ? B.pp.data() : B.p;
}
void franges(Blk &B, int op, int &is, int &ie, int &js, int &je, int &ks, int &ke) {
  if (op == 1) { is = B.isu; ie = B.ieu; js = B.jsu; je = B.jeu; ks = B.ksu; ke = B.keu; }
  else if (op == 2) { is = B.isv; ie = B.iev; js = B.jsv; je = B.jev; ks = B.ksv; ke = B.kev; }
  else if (op == 3) { is = B.isw; ie = B.iew; js = B.jsw; je = B.jew; ks = B.ksw; ke = B.kew; }
  else { is = B.isp; ie = B.iep; js = B.jsp; je = B.jep; ks = B.ksp; ke = B.kep; }
}

/* exchange_bc (exchange_bc.for:2-841) with every block on one MPI rank
 * (the `dom_ad(a) .eq. dom_ad(b)` path), layers ly = 0..nly.  Per layer the
 * reference walks the blocks three times, face by face W, E, S, N, B, T
 * (:16-320, :322-640, :642-838).  The first two walks copy a block that is
 * alone along a periodic axis onto itself (full ghost-inclusive planes) and
 * pack every other periodic face straight into the partner's receive
 * buffer - the second pack overwrites the first, from the state the first
 * walk's self-copies left; the third walk unpacks. */
void bc_face(Ctx &C, Blk &B, int op, int ly, int f, bool unpack) {
  const int ax = f / 2;
  const bool high = f & 1;
  const int bcs[6] = {B.d.bc_west, B.d.bc_east, B.d.bc_south, B.d.bc_north, B.d.bc_bottom, B.d.bc_top};
  const int nbr[6] = {B.d.iprev, B.d.inext, B.d.jprev, B.d.jnext, B.d.kprev, B.d.knext};
  const int per[6] = {B.d.per_ip, B.d.per_in, B.d.per_jp, B.d.per_jn, B.d.per_kp, B.d.per_kn};
  if (!(bcs[f] == 5 && nbr[f] < 0)) return;
  const bool alone = nbr[f ^ 1] < 0;
  int is, ie, js, je, ks, ke;
  franges(B, op, is, ie, js, je, ks, ke);
  double *fi = field_of(B, op);
  int s0 = ax == 0 ? is : ax == 1 ? js : ks, e0 = ax == 0 ? ie : ax == 1 ? je : ke;
  int n1 = ax == 0 ? B.ttc_j : B.ttc_i, n2 = ax == 2 ? B.ttc_j : B.ttc_k;
  auto at = [&](int a, int s, int t) -> double & {
    if (ax == 0) return F(B, fi, a, s, t);
    if (ax == 1) return F(B, fi, s, a, t);
    return F(B, fi, s, t, a);
  };
  const int ghost = high ? e0 + 1 + ly : s0 - 1 - ly;
  if (unpack) {
    if (alone) return;
    std::vector<double> &R = high ? B.frp[ax + 1] : B.frm[ax + 1];
    for (int t = 1; t <= n2; ++t) for (int s = 1; s <= n1; ++s) at(ghost, s, t) = R[(size_t)(t - 1) * n1 + s];
    return;
  }
  if (alone) {
    const int src = high ? s0 + ly : e0 - ly;
    for (int t = 1; t <= n2; ++t) for (int s = 1; s <= n1; ++s) at(ghost, s, t) = at(src, s, t);
    return;
  }
  Blk &P = C.b[C.indid.at(per[f])];
  std::vector<double> &R = high ? P.frm[ax + 1] : P.frp[ax + 1];
  R.assign((size_t)n1 * n2 + 1, 0.0);
  const int src = high ? e0 - ly : s0 + ly;
  for (int t = 1; t <= n2; ++t) for (int s = 1; s <= n1; ++s) R[(size_t)(t - 1) * n1 + s] = at(src, s, t);
}

void exchange_bc(Ctx &C, int op, int nly) {
  for (int ly = 0; ly <= nly; ++ly) {
    for (int walk = 0; walk < 2; ++walk)
      for (auto &B : C.b)
        for (int f = 0; f < 6; ++f) bc_face(C, B, op, ly, f, false);
    for (auto &B : C.b)
      for (int f = 0; f < 6; ++f) bc_face(C, B, op, ly, f, true);
  }
}

/* Corner and edge neighbours of exchange_smlvl, as the direction of the
 * neighbour along x, y, z (-1 low side, +1 high side, 0 the axis an edge
 * runs along).  corprev[c] / cornext[c] and edgprev[e] / edgnext[e] of
 * mf3d_block_desc (alloc_dom.for), in the order exchange.for packs and
 * unpacks them (:671-1201, :2120-2397). */
const int kCorPrev[4][3] = {{-1, -1, -1}, {-1, 1, -1}, {1, 1, -1}, {1, -1, -1}};
const int kCorNext[4][3] = {{1, 1, 1}, {1, -1, 1}, {-1, -1, 1}, {-1, 1, 1}};
const int kEdgPrev[6][3] = {{-1, 0, -1}, {0, 1, -1}, {1, 0, -1}, {0, -1, -1}, {-1, -1, 0}, {-1, 1, 0}};
const int kEdgNext[6][3] = {{1, 0, 1}, {0, -1, 1}, {-1, 0, 1}, {0, 1, 1}, {1, 1, 0}, {1, -1, 0}};

/* exchange_smlvl (exchange.for:343-2498) with every block on one rank (the
 * `dom_ad(a) .eq. dom_ad(b)` path: a sender packs straight into the
 * receiver's buffer).  Per layer ly every block packs from the state at the
 * start of the layer - faces (plane is+ly / ie-ly of the field's range,
 * full ghost-inclusive ttc planes) and, for ly = 0 only, the (pl+1)^3 corner
 * cubes and the (pl+1)^2 x n edge bars at the block's corners and edges,
 * from index spr-1 (low side) or epr+1 (high side) of the pressure range
 * inward (:671-1201).  Then every block unpacks: the corners, at spr-pl..spr
 * or epr..epr+pl, only cells outside the field's range is..ie in some axis
 * (:2120-2229); the edges alike over the interior of the edge's axis
 * (:2231-2397); last the faces, ghost plane is-1-ly / ie+1+ly over the
 * interior tangential range (:2405-2490). */
void exchange_smlvl(Ctx &C, int op, int nly) {
  const int pl = C.pl, pll = (pl + 1) * (pl + 1);
  const size_t nb = C.b.size();
  for (int ly = 0; ly <= nly; ++ly) {
  /* receive buffers of every block: faces bm/bp per axis, corners rcm/rcp, edges rem/rep */
  std::vector<std::vector<double>> bm(nb * 4), bp(nb * 4);
  std::vector<std::vector<double>> rcm(nb * 4), rcp(nb * 4), rem(nb * 6), rep(nb * 6);
  for (size_t ib = 0; ib < nb; ++ib) {
    Blk &B = C.b[ib];
    int is, ie, js, je, ks, ke;
    franges(B, op, is, ie, js, je, ks, ke);
    double *fi = field_of(B, op);
    const int ni = B.ttc_i, nj = B.ttc_j, nk = B.ttc_k;
    const int spr[3] = {pl + 1, pl + 1, pl + 1}, epr[3] = {ni - pl, nj - pl, nk - pl}, nn3[3] = {ni, nj, nk};
    int nbr_p[3] = {B.d.iprev, B.d.jprev, B.d.kprev}, nbr_n[3] = {B.d.inext, B.d.jnext, B.d.knext};
    for (int ax = 0; ax < 3; ++ax) {
      int n1 = ax == 0 ? B.ttc_j : B.ttc_i, n2 = ax == 2 ? B.ttc_j : B.ttc_k;
      auto at = [&](int a, int s, int t) -> double & {
        if (ax == 0) return F(B, fi, a, s, t);
        if (ax == 1) return F(B, fi, s, a, t);
        return F(B, fi, s, t, a);
      };
      int s0 = ax == 0 ? is : ax == 1 ? js : ks, e0 = ax == 0 ? ie : ax == 1 ? je : ke;
      if (nbr_p[ax] >= 0) { /* prev neighbour receives my first plane in its recvb_p */
        auto &R = bp[C.indid.at(nbr_p[ax]) * 4 + ax + 1];
        R.assign((size_t)n1 * n2 + 1, 0.0);
        for (int t = 1; t <= n2; ++t) for (int s = 1; s <= n1; ++s) R[(size_t)(t - 1) * n1 + s] = at(s0 + ly, s, t);
      }
      if (nbr_n[ax] >= 0) {
        auto &R = bm[C.indid.at(nbr_n[ax]) * 4 + ax + 1];
        R.assign((size_t)n1 * n2 + 1, 0.0);
        for (int t = 1; t <= n2; ++t) for (int s = 1; s <= n1; ++s) R[(size_t)(t - 1) * n1 + s] = at(e0 - ly, s, t);
      }
    }
    if (ly != 0) continue;
    /* sender index along an axis toward side d of the neighbour, layer q = 0..pl */
    auto sidx = [&](int ax, int d, int q) { return d < 0 ? spr[ax] - 1 + q : epr[ax] + 1 - q; };
    for (int c = 0; c < 8; ++c) {
      const bool prev = c < 4;
      const int *dir = prev ? kCorPrev[c] : kCorNext[c - 4];
      const int nbr = prev ? B.d.corprev[c] : B.d.cornext[c - 4];
      if (nbr < 0) continue;
      /* corprev c fills the receiver's rc(c)p, cornext c its rc(c)m */
      auto &R = (prev ? rcp : rcm)[C.indid.at(nbr) * 4 + (c & 3)];
      R.assign((size_t)(pl + 1) * pll + 1, 0.0);
      for (int p1 = 0; p1 <= pl; ++p1) for (int p2 = 0; p2 <= pl; ++p2) for (int p3 = 0; p3 <= pl; ++p3)
        R[(size_t)p1 * pll + p2 * (pl + 1) + p3 + 1] = F(B, fi, sidx(0, dir[0], p1), sidx(1, dir[1], p2), sidx(2, dir[2], p3));
    }
    for (int e = 0; e < 12; ++e) {
      const bool prev = e < 6;
      const int *dir = prev ? kEdgPrev[e] : kEdgNext[e - 6];
      const int nbr = prev ? B.d.edgprev[e] : B.d.edgnext[e - 6];
      if (nbr < 0) continue;
      const int along = dir[0] == 0 ? 0 : dir[1] == 0 ? 1 : 2;
      const int ta = along == 0 ? 1 : 0, tb = along == 2 ? 1 : 2;  /* transverse axes, in x, y, z order */
      auto &R = (prev ? rep : rem)[C.indid.at(nbr) * 6 + (e % 6)];
      R.assign((size_t)nn3[along] * pll + 1, 0.0);
      for (int p1 = 0; p1 <= pl; ++p1) for (int p2 = 0; p2 <= pl; ++p2) for (int nn = 1; nn <= nn3[along]; ++nn) {
        int idx[3];
        idx[along] = nn;
        idx[ta] = sidx(ta, dir[ta], p1);
        idx[tb] = sidx(tb, dir[tb], p2);
        R[(size_t)(nn - 1) * pll + p1 * (pl + 1) + p2 + 1] = F(B, fi, idx[0], idx[1], idx[2]);
      }
    }
  }
  /* unpack: corners and edges (ly = 0), then the faces over the interior
   * tangential range pl+1 .. n-pl (exchange.for:2402-2490) */
  for (size_t ib = 0; ib < nb; ++ib) {
    Blk &B = C.b[ib];
    int is, ie, js, je, ks, ke;
    franges(B, op, is, ie, js, je, ks, ke);
    double *fi = field_of(B, op);
    const int ni = B.ttc_i, nj = B.ttc_j, nk = B.ttc_k;
    const int spr[3] = {pl + 1, pl + 1, pl + 1}, epr[3] = {ni - pl, nj - pl, nk - pl};
    const int lo[3] = {is, js, ks}, hi[3] = {ie, je, ke};
    /* receiver index toward side d, layer q = 0..pl; `out` when beyond the field's range */
    auto ridx = [&](int ax, int d, int q) { return d < 0 ? spr[ax] - q : epr[ax] + q; };
    auto out = [&](int ax, int d, int v) { return d < 0 ? v < lo[ax] : v > hi[ax]; };
    if (ly == 0) {
      for (int c = 0; c < 8; ++c) {
        const bool prev = c < 4;
        const int *dir = prev ? kCorPrev[c] : kCorNext[c - 4];
        const int nbr = prev ? B.d.corprev[c] : B.d.cornext[c - 4];
        if (nbr < 0) continue;
        const auto &R = (prev ? rcm : rcp)[ib * 4 + (c & 3)];
        for (int p1 = 0; p1 <= pl; ++p1) for (int p2 = 0; p2 <= pl; ++p2) for (int p3 = 0; p3 <= pl; ++p3) {
          const int i = ridx(0, dir[0], p1), j = ridx(1, dir[1], p2), k = ridx(2, dir[2], p3);
          if (out(0, dir[0], i) || out(1, dir[1], j) || out(2, dir[2], k))
            F(B, fi, i, j, k) = R[(size_t)p1 * pll + p2 * (pl + 1) + p3 + 1];
        }
      }
      for (int e = 0; e < 12; ++e) {
        const bool prev = e < 6;
        const int *dir = prev ? kEdgPrev[e] : kEdgNext[e - 6];
        const int nbr = prev ? B.d.edgprev[e] : B.d.edgnext[e - 6];
        if (nbr < 0) continue;
        const int along = dir[0] == 0 ? 0 : dir[1] == 0 ? 1 : 2;
        const int ta = along == 0 ? 1 : 0, tb = along == 2 ? 1 : 2;
        const auto &R = (prev ? rem : rep)[ib * 6 + (e % 6)];
        for (int p1 = 0; p1 <= pl; ++p1) for (int p2 = 0; p2 <= pl; ++p2)
          for (int nn = spr[along]; nn <= epr[along]; ++nn) {
            int idx[3];
            idx[along] = nn;
            idx[ta] = ridx(ta, dir[ta], p1);
            idx[tb] = ridx(tb, dir[tb], p2);
            if (out(ta, dir[ta], idx[ta]) || out(tb, dir[tb], idx[tb]))
              F(B, fi, idx[0], idx[1], idx[2]) = R[(size_t)(nn - 1) * pll + p1 * (pl + 1) + p2 + 1];
          }
      }
    }
    int nbr_p[3] = {B.d.iprev, B.d.jprev, B.d.kprev}, nbr_n[3] = {B.d.inext, B.d.jnext, B.d.knext};
    for (int ax = 0; ax < 3; ++ax) {
      int n1 = ax == 0 ? B.ttc_j : B.ttc_i;
      int sp1 = pl + 1, ep1 = (ax == 0 ? B.ttc_j : B.ttc_i) - pl;
      int sp2 = pl + 1, ep2 = (ax == 2 ? B.ttc_j : B.ttc_k) - pl;
      auto at = [&](int a, int s, int t) -> double & {
        if (ax == 0) return F(B, fi, a, s, t);
        if (ax == 1) return F(B, fi, s, a, t);
        return F(B, fi, s, t, a);
      };
      int s0 = ax == 0 ? is : ax == 1 ? js : ks, e0 = ax == 0 ? ie : ax == 1 ? je : ke;
      if (nbr_p[ax] >= 0) {
        auto &R = bm[ib * 4 + ax + 1];
        for (int t = sp2; t <= ep2; ++t) for (int s = sp1; s <= ep1; ++s) at(s0 - 1 - ly, s, t) = R[(size_t)(t - 1) * n1 + s];
      }
      if (nbr_n[ax] >= 0) {
        auto &R = bp[ib * 4 + ax + 1];
        for (int t = sp2; t <= ep2; ++t) for (int s = sp1; s <= ep1; ++s) at(e0 + 1 + ly, s, t) = R[(size_t)(t - 1) * n1 + s];
      }
    }
  }
  }
}

void exchange(Ctx &C, int op) {
  const int nly = (op == 4 || op == 44) ? 0 : C.pl_ex;
  if (C.periodic) exchange_bc(C, op, nly);
  exchange_smlvl(C, op, nly);
}

/* pbound (press.for:77-137) */
void pbound(Ctx &C) {
  for (auto &B : C.b) {
    double *p = B.p;
    int isp = B.isp, iep = B.iep, jsp = B.jsp, jep = B.jep, ksp = B.ksp, kep = B.kep;
    if (B.d.iprev < 0 && B.d.bc_west != 5)
      for (int k = ksp - 1; k <= kep + 1; ++k) for (int j = jsp - 1; j <= jep + 1; ++j) F(B, p, isp - 1, j, k) = F(B, p, isp, j, k);
    if (B.d.inext < 0 && B.d.bc_east != 5)
      for (int k = ksp - 1; k <= kep + 1; ++k) for (int j = jsp - 1; j <= jep + 1; ++j) F(B, p, iep + 1, j, k) = F(B, p, iep, j, k);
    if (B.d.jprev < 0 && B.d.bc_south != 5)
      for (int k = ksp - 1; k <= kep + 1; ++k) for (int i = isp - 1; i <= iep + 1; ++i) F(B, p, i, jsp - 1, k) = F(B, p, i, jsp, k);
    if (B.d.jnext < 0 && B.d.bc_north != 5)
      for (int k = ksp - 1; k <= kep + 1; ++k) for (int i = isp - 1; i <= iep + 1; ++i) F(B, p, i, jep + 1, k) = F(B, p, i, jep, k);
    if (B.d.kprev < 0 && B.d.bc_bottom != 5)
      for (int j = jsp - 1; j <= jep + 1; ++j) for (int i = isp - 1; i <= iep + 1; ++i) F(B, p, i, j, ksp - 1) = F(B, p, i, j, ksp);
    if (B.d.knext < 0 && B.d.bc_top != 5)
      for (int j = jsp - 1; j <= jep + 1; ++j) for (int i = isp - 1; i <= iep + 1; ++i) F(B, p, i, j, kep + 1) = F(B, p, i, j, kep);
  }
}

/* boundu, boundv, boundw (bounds.for:2-916), restated for the codes 1
 * (inflow), 2 (outflow), 3 (symmetry), 4 (wall) and 5 (periodic); set-up
 * rejects the codes whose branch reads files, phi, uoo or wall functions.
 * The periodic copy, then per layer ly = 0..pl_ex each block's faces W, E,
 * S, N, B, T over the component's ranges widened by one cell:
 *   normal component (u on x faces, ...): wall -> 0; symmetry -> 0 on y and
 *     z faces, nothing on x faces;
 *   tangential component: wall -> -(the cell ly inside); symmetry -> +(the
 *     same) on y and z faces, nothing on x faces;
 *   inflow on the west: u = ubulk, v = w = 0 (bounds.for:42-53, 374-377,
 *     662-665); on the bottom u = v = 0, w = 1.1 (226-229, 536-539, 873-876);
 *   outflow on the east, alfabc = 1: ghost layer ly = the last face ie
 *     (bounds.for:136-170, 444-470 and the same branch of boundw);
 *   any other (face, code) pair: nothing.
 * (bounds.for:36-42, 136-140, 179-186, 212-219, 246-259, 301-308 for u;
 * 369-373, 444-448, 505-533, 535-548, 588-595 for v; 657-661, 738-742,
 * 799-806, 833-840, 866-876, 900-908 for w.) */
bool bounds_code_unsupported(int f, int code, bool lsm, int alfabc, bool have_oo = false) {
  /* the branches that read data outside the projection: the convective
   * outflow (east 21) unless uoo, voo, woo are at hand, wall functions
   * (61 to 65) without Re (and fric for 62) or under L_LSM (mu/dens), codes
   * above 65, phi-gated inflow/outflow under L_LSM.  The inlet files of the
   * west codes 7 and 8 come from g_inlets. */
  if (code >= 61 && (code > 65 || lsm || g_re == 0.0 || (code == 62 && g_fric == 0.0))) return true;
  if (f == 1 && code == 21 && alfabc == 1 && !have_oo) return true;
  if (lsm && ((f == 0 && code == 1) || (f == 1 && (code == 2 || code == 21) && alfabc == 1))) return true;
  return false;
}
/* Cell-centre coordinate of field index c (1-based) along an axis of a
 * block: x(1) = xsl + (1-pl)*dx, x(c) = x(c-1) + dx, xc(c) = x(c) - 0.5*dx
 * (initial.for:341-365), the running sum in the reference's order. */
double centre(double lo, double h, int pl, int c) {
  double x = lo + (double)(-pl + 1) * h;
  for (int i = 2; i <= c; ++i) x = x + h;
  return x - 0.5 * h;
}
/* The 1/7 power-law inlet in y (bounds.for:105-112, 127-133, 86-93) */
double power_law_y(const Ctx &C, double yc) {
  const double H = C.yen - C.yst;
  if (yc < H / 2) return C.ubulk * (1.0 + 1.0 / 7.0) * std::pow(std::fabs(2 * yc / H), 1. / 7.);
  return C.ubulk * (1.0 + 1.0 / 7.0) * std::pow(std::fabs(2 * (H - yc) / H), 1.0 / 7.0);
}
/* ... times the same law in z (bounds.for:113-114, 94-95) */
double power_law_z(const Ctx &C, double u, double zc) {
  return u * (1.0 + 1. / 7.) * std::pow(std::fabs(zc / (C.zen - C.zst)), 1. / 7.);
}

/* boundu's, boundv's and boundw's west branches of the codes 7, 8, 12 and
 * 13 on ghost layer ly for component op (bounds.for:55-135, 397-438,
 * 686-730).  The inlet file's values are u's, then v's, then w's, each over
 * the component's own ranges: code 7 reads rows js-1..je+1 and planes
 * ks-1..ke+1 per component (boundv skips u's lines, boundw u's and v's);
 * code 8 reads rows js-1..je and planes ks-1..ke, u as the fluctuation up
 * (the first column) on ubulk or on the code-12 profile (UPROF_SEM = 12),
 * v and w as the second and third columns. */
void bound_inlet(const Ctx &C, Blk &B, int op, int ly) {
  const int code = B.d.bc_west, pl = C.pl;
  int is, ie, js, je, ks, ke;
  franges(B, op, is, ie, js, je, ks, ke);
  double *fi = field_of(B, op);
  if (code == 7 || code == 8) {
    const InletFile &in = g_inlets.at(B.d.id);
    size_t r = 0;
    for (int c = 1; c < op; ++c) {  /* the lines of the components before this one */
      int cis, cie, cjs, cje, cks, cke;
      franges(B, c, cis, cie, cjs, cje, cks, cke);
      r += code == 7 ? (size_t)(cje - cjs + 3) * (cke - cks + 3) : (size_t)(cje - cjs + 2) * (cke - cks + 2);
    }
    if (code == 7) {
      for (int k = ks - 1; k <= ke + 1; ++k)
        for (int j = js - 1; j <= je + 1; ++j) F(B, fi, is - 1 - ly, j, k) = in.v[r++];
    } else {
      for (int kk = 1; kk <= ke - ks + 2; ++kk)
        for (int jj = 1; jj <= je - js + 2; ++jj) {
          const int k = kk + pl - 1, j = jj + pl - 1;
          const double x = in.v[r++];
          double &u = F(B, fi, is - 1 - ly, j, k);
          if (op != 1) {
            u = x;
          } else if (in.uprof == 12) {
            u = power_law_y(C, centre(B.d.ysl, B.d.dy, pl, j));
            u = power_law_z(C, u, centre(B.d.zsl, B.d.dz, pl, k)) + x;
          } else {
            u = C.ubulk + x;
          }
        }
    }
  } else if ((code == 12 || code == 13) && op == 1) {  /* :105-135 */
    for (int k = ks - 1; k <= ke + 1; ++k)
      for (int j = js - 1; j <= je + 1; ++j) {
        double &u = F(B, B.u, is - 1 - ly, j, k);
        u = power_law_y(C, centre(B.d.ysl, B.d.dy, pl, j));
        if (code == 12) u = power_law_z(C, u, centre(B.d.zsl, B.d.dz, pl, k));
      }
  }
}

/* The wall stresses of the six faces of each block (tauww, tauwe, tauws,
 * tauwn, tauwb, tauwt and their "2" arrays, initial.for:288-299): zero at
 * the start (initial.for:878-883) and kept across calls, as the reference
 * keeps them across time steps.  Element of face f (W, E, S, N, B, T) at
 * the two tangential field indices (j,k), (j,k), (i,k), (i,k), (i,j), (i,j);
 * which = 0: tau, 1: tau2. */
std::map<int, std::array<std::vector<double>, 12>> g_tau; /* per block id: tau[6], tau2[6] */
double &tau_at(Blk &B, int which, int f, int a, int b) {
  std::vector<double> &v = g_tau[B.d.id][6 * which + f];
  const int n1 = f < 2 ? B.ttc_j : B.ttc_i, n2 = f < 4 ? B.ttc_k : B.ttc_j;
  if (v.empty()) v.assign((size_t)n1 * n2, 0.0);
  return v[(size_t)(a - 1) + (size_t)n1 * (b - 1)];
}

/* log_law(bound, ib) (log_law.for:2-310, codes 61 smooth and 62 rough) and
 * wall_function(bound, ib) (wall_function.for:2-250, the power laws of
 * codes 63, 64, 65) for face f of block B: per cell of the face's plane
 * (the cell ranges widened by one) the tangential speed of the first cell
 * layer and the wall stress tau, tau2 = tau/vtan.  log_law keeps the old
 * tau2 where y+ is below 11.067 (11.63 on the top face).  Returns false
 * where the smooth-wall iteration does not converge (the reference prints
 * "USTAR DOESNT CONVERGE" and stops). */
bool wall_law(const Ctx &C, Blk &B, int f) {
  const int code = f == 0 ? B.d.bc_west : f == 1 ? B.d.bc_east : f == 2 ? B.d.bc_south : f == 3 ? B.d.bc_north
                   : f == 4 ? B.d.bc_bottom : B.d.bc_top;
  const double rrey = 1.0 / g_re, small = 1.e-30, kappa = 0.41, Ecte = 9.0;
  const int ax = f / 2;
  const double delta = ax == 0 ? B.d.dx : ax == 1 ? B.d.dy : B.d.dz;
  const double nx = ax == 0 ? (f == 0 ? 1.0 : -1.0) : 0.0, ny = ax == 1 ? (f == 2 ? 1.0 : -1.0) : 0.0,
               nz = ax == 2 ? (f == 4 ? 1.0 : -1.0) : 0.0;
  /* wall_function's constants; the reference sets aaa, bbb by DATA
   * statements inside the CASE arms (wall_function.for:34-49); taken here by
   * the arms' intent: 1/6, 1/7 and 1/8 power laws */
  double aaa = 8.3, bbb = code == 63 ? 0.1666666666 : code == 64 ? 0.1428571429 : 0.125;
  const double const1 = 0.5 * (1. - bbb) * std::pow(aaa, (1. + bbb) / (1. - bbb));
  const double const2 = (1. + bbb) / aaa;
  const double const3 = std::pow(aaa, 2. / (1. - bbb));
  const double const4 = 2. / (1. + bbb);
  bool ok = true;
  /* loops: W/E k outer, j inner at i = isp/iep; S/N k outer, i inner at
   * j = jsp/jep; B/T j outer, i inner at k = ksp/kep */
  const int fix = f == 0 ? B.isp : f == 1 ? B.iep : f == 2 ? B.jsp : f == 3 ? B.jep : f == 4 ? B.ksp : B.kep;
  const int o0 = ax == 2 ? B.jsp : B.ksp, o1 = ax == 2 ? B.jep : B.kep;
  const int i0 = ax == 0 ? B.jsp : B.isp, i1 = ax == 0 ? B.jep : B.iep;
  for (int o = o0 - 1; o <= o1 + 1; ++o)
    for (int q = i0 - 1; q <= i1 + 1; ++q) {
      const int i = ax == 0 ? fix : q, j = ax == 0 ? q : ax == 1 ? fix : o, k = ax == 2 ? fix : o;
      const double uc = 0.5 * (F(B, B.u, i, j, k) + F(B, B.u, i - 1, j, k));
      const double vc = 0.5 * (F(B, B.v, i, j, k) + F(B, B.v, i, j - 1, k));
      const double wc = 0.5 * (F(B, B.w, i, j, k) + F(B, B.w, i, j, k - 1));
      const double vnor = nx * uc + ny * vc + nz * wc;
      const double vtan = std::sqrt(std::fabs(uc * uc + vc * vc + wc * wc - vnor * vnor + small));
      double &tau = tau_at(B, 0, f, q, o), &tau2 = tau_at(B, 1, f, q, o);
      if (code >= 63) {
        const double dycell = 2. * delta, rycell = 1. / dycell;
        const double vtankr = 0.5 * rrey * rycell * const3;
        const double dvtan = vtankr - vtan;
        const double sub = std::max(std::copysign(1., dvtan), 0.);
        const double tausub = rrey * vtan / delta;
        const double taupow = std::pow(const1 * std::pow(rrey * rycell, 1. + bbb) +
                                       (const2 * std::pow(rrey * rycell, bbb)) * vtan, const4);
        tau = (sub * tausub + (1. - sub) * taupow);
        tau2 = tau / vtan;
        continue;
      }
      double ustar = 0.0, yplus = 0.0;
      if (code == 62) {
        ustar = kappa * vtan / std::log(30.0 * delta / g_fric);
        yplus = delta * ustar / rrey;
      } else if (code == 61) {
        double conv = 1., ustarold;
        int icont = 0;
        const int tkmax = 10;
        ustar = 1.;
        while (conv > 1.e-3 && icont < tkmax) {
          ++icont;
          ustarold = ustar;
          yplus = std::max(1.0000001, delta * ustar / rrey);
          ustar = vtan * kappa / std::log(Ecte * yplus);
          conv = std::fabs((ustar - ustarold) / ustar);
        }
        if (icont == tkmax) ok = false;
      }
      if (yplus < (f == 5 ? 11.63 : 11.067)) {
        tau = rrey * vtan / delta;
      } else {
        tau = ustar * ustar;  /* ustar**2.0 */
        tau2 = tau / vtan;
      }
    }
  return ok;
}

/* boundu/v/w's wall-function branch (codes 61 and up) for the tangential
 * component op on face f at layer ly (bounds.for:187-206, 221-239, 260-283,
 * 309-329 for u; 378-397, 480-499, 549-568, 596-615 for v; 666-685,
 * 773-792, 808-827, 841-860 for w).  Layer 0: the face's wall law, then per
 * face cell F = sign(tau2*c(first)/h_c, -c(first)), c(first) += F*alfapr*dt
 * and c(ghost 0) = -c(first), h_c the spacing along the component's own
 * axis; deeper layers mirror the first cell (u on the S, N and B faces:
 * the cell ly inside). */
bool bound_wall_law(const Ctx &C, Blk &B, int op, int ly, int f) {
  const int ax = f / 2, comp = op - 1;
  const bool high = f & 1;
  int is, ie, js, je, ks, ke;
  franges(B, op, is, ie, js, je, ks, ke);
  double *fi = field_of(B, op);
  const int s0 = ax == 0 ? is : ax == 1 ? js : ks, e0 = ax == 0 ? ie : ax == 1 ? je : ke;
  const int sa = ax == 0 ? js : is, ea = ax == 0 ? je : ie;
  const int ta = ax == 2 ? js : ks, tb = ax == 2 ? je : ke;
  auto at = [&](int a, int s, int t) -> double & {
    if (ax == 0) return F(B, fi, a, s, t);
    if (ax == 1) return F(B, fi, s, a, t);
    return F(B, fi, s, t, a);
  };
  const int first = high ? e0 : s0;
  if (ly == 0) {
    const bool ok = wall_law(C, B, f);
    const double h = comp == 0 ? B.d.dx : comp == 1 ? B.d.dy : B.d.dz;
    for (int t = ta - 1; t <= tb + 1; ++t)
      for (int s = sa - 1; s <= ea + 1; ++s) {
        double &c = at(first, s, t);
        double fw = tau_at(B, 1, f, s, t) * c / h;
        fw = std::copysign(std::fabs(fw), -c);  /* SIGN(Fwall, -c) */
        c = c + fw * C.alfapr * C.dt;
        at(high ? e0 + 1 : s0 - 1, s, t) = -c;
      }
    return ok;
  }
  const bool deep = comp == 0 && f != 5;
  for (int t = ta - 1; t <= tb + 1; ++t)
    for (int s = sa - 1; s <= ea + 1; ++s)
      at(high ? e0 + 1 + ly : s0 - 1 - ly, s, t) = -at(deep ? (high ? e0 - ly : s0 + ly) : first, s, t);
  return true;
}

void bound_face(const Ctx &C, Blk &B, int op, int ly, int f) {
  const int ax = f / 2, comp = op - 1;
  const bool high = f & 1;
  const int bcs[6] = {B.d.bc_west, B.d.bc_east, B.d.bc_south, B.d.bc_north, B.d.bc_bottom, B.d.bc_top};
  const int nbr[6] = {B.d.iprev, B.d.inext, B.d.jprev, B.d.jnext, B.d.kprev, B.d.knext};
  if (nbr[f] >= 0) return;
  const int code = bcs[f];
  if (f == 0 && ((code == 7 || code == 8) || (op == 1 && (code == 12 || code == 13)))) {
    bound_inlet(C, B, op, ly);
    return;
  }
  const bool normal = ax == comp;
  if (code >= 61 && !normal) {  /* the wall functions of the tangential components */
    if (!bound_wall_law(C, B, op, ly, f)) g_wall_fail = true;
    return;
  }
  int mode = 0; /* 0 nothing, 1 the constant cv, 2 -mirror, 3 +mirror, 4 copy of face ie */
  double cv = 0.0;
  if (code == 4) mode = normal ? 1 : 2;
  else if (code >= 61) mode = 1;  /* the normal component at a wall-function face: 0 */
  else if (code == 3 && ax != 0) mode = normal ? 1 : 3;
  else if (code == 1 && f == 0) { mode = 1; cv = comp == 0 ? C.ubulk : 0.0; }
  else if (code == 12 && f == 0) { mode = 1; cv = 0.0; } /* v, w (bounds.for:374-377, 662-665) */
  else if (code == 1 && f == 4) { mode = 1; cv = comp == 2 ? 1.1 : 0.0; }
  else if (code == 2 && f == 1 && C.alfabc == 1) mode = 4;
  else if (code == 21 && f == 1 && C.alfabc == 1 && B.oo[op - 1]) mode = 5;
  if (!mode) return;
  int is, ie, js, je, ks, ke;
  franges(B, op, is, ie, js, je, ks, ke);
  double *fi = field_of(B, op);
  int s0 = ax == 0 ? is : ax == 1 ? js : ks, e0 = ax == 0 ? ie : ax == 1 ? je : ke;
  /* the other two axes, in the reference's loop order (outer t, inner s) */
  int sa = ax == 0 ? js : is, ea = ax == 0 ? je : ie;
  int ta = ax == 2 ? js : ks, tb = ax == 2 ? je : ke;
  auto at = [&](int a, int s, int t) -> double & {
    if (ax == 0) return F(B, fi, a, s, t);
    if (ax == 1) return F(B, fi, s, a, t);
    return F(B, fi, s, t, a);
  };
  const int ghost = high ? e0 + 1 + ly : s0 - 1 - ly, mirror = mode >= 4 ? e0 : high ? e0 - ly : s0 + ly;
  if (mode == 5) {  /* convective outflow (bounds.for:143-170 and boundv/w's branch) */
    const double *oo = B.oo[op - 1];
    const double dt = C.dt, alfapr = C.alfapr, dx = B.d.dx;
    for (int t = ta - 1; t <= tb + 1; ++t)
      for (int s = sa - 1; s <= ea + 1; ++s) {
        const double og = F(B, oo, ghost, s, t), oe = F(B, oo, e0, s, t);
        at(ghost, s, t) = og - dt * alfapr * (og - oe) / dx;
      }
    return;
  }
  for (int t = ta - 1; t <= tb + 1; ++t)
    for (int s = sa - 1; s <= ea + 1; ++s)
      at(ghost, s, t) = mode == 1 ? cv : mode == 2 ? -at(mirror, s, t) : at(mirror, s, t);
}

void bound(Ctx &C, int op) {
  if (C.periodic) exchange_bc(C, op, C.pl_ex);
  for (int ly = 0; ly <= C.pl_ex; ++ly)
    for (auto &B : C.b)
      for (int f = 0; f < 6; ++f) bound_face(C, B, op, ly, f);
}

/* One Runge-Kutta stage of the velocity predictor, the reference's branch
 * without L_LSM, immersed boundaries or wall functions:
 * rungek_conv2nd (rungek.for:314-412) - boundu, the u loop, boundv, the v
 * loop, boundw, the w loop, each loop
 *   star = (oo - dt*alfapr*(conv)), conv the 2nd-order conservative terms
 *   in the order the reference sums them -
 * then rungek_diff2nd (rungek.for:584-779): per component over the same
 * ranges, with visc the viscosity of the cell past the face,
 *   aw = ae = -visc/dxx, an = as = -visc/dyy, at = ab = -visc/dzz,
 *   ap = -1.0*(aw+ae+as+an+ab+at),
 *   diff = -(ap*c + an*c(j+1) + as*c(j-1) + ae*c(i+1) + aw*c(i-1)
 *            + at*c(k+1) + ab*c(k-1)),
 *   star = (star + dt*alfapr*diff),
 * and for u under pressureforce star = star + dt*alfapr*forcn (:650-652).
 * The u loop reads v and w before boundv/boundw refresh their ghosts. */
void diff2nd(Ctx &C, const double *const *vis, bool pforce, double forcn);
void rungek_2nd(Ctx &C, const double *const *uoo, const double *const *voo, const double *const *woo,
                const double *const *vis, bool pforce, double forcn) {
  const double dt = C.dt, alfapr = C.alfapr;
  for (int op = 1; op <= 3; ++op) {
    bound(C, op);
    par_blocks((int)C.b.size(), [&](int ib) { Blk &B = C.b[ib];
      const double dx = B.d.dx, dy = B.d.dy, dz = B.d.dz;
      double *st = op == 1 ? B.ustar : op == 2 ? B.vstar : B.wstar;
      const double *oo = op == 1 ? uoo[ib] : op == 2 ? voo[ib] : woo[ib];
      int is, ie, js, je, ks, ke;
      franges(B, op, is, ie, js, je, ks, ke);
      auto u = [&](int i, int j, int k) { return F(B, B.u, i, j, k); };
      auto v = [&](int i, int j, int k) { return F(B, B.v, i, j, k); };
      auto w = [&](int i, int j, int k) { return F(B, B.w, i, j, k); };
      for (int k = ks; k <= ke; ++k) for (int i = is; i <= ie; ++i) for (int j = js; j <= je; ++j) {
        double c1, c2, c3;
        if (op == 1) {
          const double up12 = 0.5 * (u(i, j, k) + u(i + 1, j, k)), um12 = 0.5 * (u(i, j, k) + u(i - 1, j, k));
          c1 = (up12 * up12 - um12 * um12) / dx;
          c2 = 0.25 * ((v(i, j, k) + v(i + 1, j, k)) * (u(i, j, k) + u(i, j + 1, k)) -
                       (v(i, j - 1, k) + v(i + 1, j - 1, k)) * (u(i, j, k) + u(i, j - 1, k))) / dy;
          c3 = 0.25 * ((w(i, j, k) + w(i + 1, j, k)) * (u(i, j, k) + u(i, j, k + 1)) -
                       (w(i, j, k - 1) + w(i + 1, j, k - 1)) * (u(i, j, k) + u(i, j, k - 1))) / dz;
        } else if (op == 2) {
          const double vp12 = 0.5 * (v(i, j, k) + v(i, j + 1, k)), vm12 = 0.5 * (v(i, j, k) + v(i, j - 1, k));
          c2 = (vp12 * vp12 - vm12 * vm12) / dy;
          c1 = 0.25 * ((u(i, j, k) + u(i, j + 1, k)) * (v(i, j, k) + v(i + 1, j, k)) -
                       (u(i - 1, j, k) + u(i - 1, j + 1, k)) * (v(i, j, k) + v(i - 1, j, k))) / dx;
          c3 = 0.25 * ((w(i, j, k) + w(i, j + 1, k)) * (v(i, j, k) + v(i, j, k + 1)) -
                       (w(i, j, k - 1) + w(i, j + 1, k - 1)) * (v(i, j, k) + v(i, j, k - 1))) / dz;
        } else {
          const double wp12 = 0.5 * (w(i, j, k) + w(i, j, k + 1)), wm12 = 0.5 * (w(i, j, k) + w(i, j, k - 1));
          c3 = (wp12 * wp12 - wm12 * wm12) / dz;
          c1 = 0.25 * ((u(i, j, k) + u(i, j, k + 1)) * (w(i, j, k) + w(i + 1, j, k)) -
                       (u(i - 1, j, k) + u(i - 1, j, k + 1)) * (w(i, j, k) + w(i - 1, j, k))) / dx;
          c2 = 0.25 * ((v(i, j, k) + v(i, j, k + 1)) * (w(i, j, k) + w(i, j + 1, k)) -
                       (v(i, j - 1, k) + v(i, j - 1, k + 1)) * (w(i, j, k) + w(i, j - 1, k))) / dy;
        }
        F(B, st, i, j, k) = (F(B, oo, i, j, k) - dt * alfapr * (c1 + c2 + c3));
      }
    });
  }
  diff2nd(C, vis, pforce, forcn);
}

/* rungek_diff2nd (rungek.for:584-779), the branch without L_LSM. */
void diff2nd(Ctx &C, const double *const *vis, bool pforce, double forcn) {
  const double dt = C.dt, alfapr = C.alfapr;
  par_blocks((int)C.b.size(), [&](int ib) { Blk &B = C.b[ib];
    const double dxx = B.d.dx * B.d.dx, dyy = B.d.dy * B.d.dy, dzz = B.d.dz * B.d.dz;
    for (int op = 1; op <= 3; ++op) {
      double *st = op == 1 ? B.ustar : op == 2 ? B.vstar : B.wstar;
      double *c = field_of(B, op);
      int is, ie, js, je, ks, ke;
      franges(B, op, is, ie, js, je, ks, ke);
      for (int k = ks; k <= ke; ++k) for (int i = is; i <= ie; ++i) for (int j = js; j <= je; ++j) {
        const double visc = op == 1 ? F(B, vis[ib], i + 1, j, k) : op == 2 ? F(B, vis[ib], i, j + 1, k)
                                                                           : F(B, vis[ib], i, j, k + 1);
        const double aw = -visc / dxx, ae = -visc / dxx, an = -visc / dyy, as = -visc / dyy;
        const double at = -visc / dzz, ab = -visc / dzz;
        const double ap = -1.0 * (aw + ae + as + an + ab + at);
        const double diff = -(ap * F(B, c, i, j, k) + an * F(B, c, i, j + 1, k) + as * F(B, c, i, j - 1, k) +
                              ae * F(B, c, i + 1, j, k) + aw * F(B, c, i - 1, j, k) + at * F(B, c, i, j, k + 1) +
                              ab * F(B, c, i, j, k - 1));
        F(B, st, i, j, k) = (F(B, st, i, j, k) + dt * alfapr * diff);
        if (op == 1 && pforce) F(B, st, i, j, k) = F(B, st, i, j, k) + dt * alfapr * forcn;
      }
    }
  });
}

/* One Runge-Kutta stage of rungek_conv4th (rungek.for:2-212) and
 * rungek_diff4th (rungek.for:214-312) in the reference's order: boundu, the
 * u loop, boundv, the v loop, boundw, the w loop; then the diffusion of u,
 * v, w.  9.0, 16.0, 27.0, 24.0, 30.0, 12.0 are double (-fdefault-real-8);
 * x**2 is x*x. */
void rungek_4th(Ctx &C, const double *const *uoo, const double *const *voo, const double *const *woo,
                const double *const *vis, bool pforce, double forcn) {
  const double dt = C.dt, alfapr = C.alfapr;
  for (int op = 1; op <= 3; ++op) {
    bound(C, op);
    par_blocks((int)C.b.size(), [&](int ib) { Blk &B = C.b[ib];
      const double dx = B.d.dx, dy = B.d.dy, dz = B.d.dz;
      double *st = op == 1 ? B.ustar : op == 2 ? B.vstar : B.wstar;
      const double *oo = op == 1 ? uoo[ib] : op == 2 ? voo[ib] : woo[ib];
      int is, ie, js, je, ks, ke;
      franges(B, op, is, ie, js, je, ks, ke);
      auto u = [&](int i, int j, int k) { return F(B, B.u, i, j, k); };
      auto v = [&](int i, int j, int k) { return F(B, B.v, i, j, k); };
      auto w = [&](int i, int j, int k) { return F(B, B.w, i, j, k); };
      /* (-f(+1) + 9 f(0) + 9 f(-1) - f(-2)) / 16 */
      auto q4 = [](double p1, double p0, double m1, double m2) { return (-p1 + 9.0 * p0 + 9.0 * m1 - m2) / 16.0; };
      /* (-s(+1) + 27 s(0) - 27 s(-1) + s(-2)) / (24 h) */
      auto d4 = [](double p1, double p0, double m1, double m2, double h) {
        return (-p1 + 27.0 * p0 - 27.0 * m1 + m2) / (24.0 * h);
      };
      for (int k = ks; k <= ke; ++k) for (int i = is; i <= ie; ++i) for (int j = js; j <= je; ++j) {
        double t1, t2, t3;
        if (op == 1) {
          auto sx = [&](int ii) { double a = q4(u(ii + 1, j, k), u(ii, j, k), u(ii - 1, j, k), u(ii - 2, j, k)); return a * a; };
          t1 = d4(sx(i + 2), sx(i + 1), sx(i), sx(i - 1), dx);  /* du2dx */
          auto py = [&](int jj) {
            return q4(u(i, jj + 2, k), u(i, jj + 1, k), u(i, jj, k), u(i, jj - 1, k)) *
                   q4(v(i + 2, jj, k), v(i + 1, jj, k), v(i, jj, k), v(i - 1, jj, k));
          };
          t2 = d4(py(j + 1), py(j), py(j - 1), py(j - 2), dy);  /* duvdy */
          auto pz = [&](int kk) {
            return q4(u(i, j, kk + 2), u(i, j, kk + 1), u(i, j, kk), u(i, j, kk - 1)) *
                   q4(w(i + 2, j, kk), w(i + 1, j, kk), w(i, j, kk), w(i - 1, j, kk));
          };
          t3 = d4(pz(k + 1), pz(k), pz(k - 1), pz(k - 2), dz);  /* duwdz */
        } else if (op == 2) {
          auto sy = [&](int jj) { double a = q4(v(i, jj + 1, k), v(i, jj, k), v(i, jj - 1, k), v(i, jj - 2, k)); return a * a; };
          t2 = d4(sy(j + 2), sy(j + 1), sy(j), sy(j - 1), dy);  /* dv2dy */
          auto px = [&](int ii) {
            return q4(v(ii + 2, j, k), v(ii + 1, j, k), v(ii, j, k), v(ii - 1, j, k)) *
                   q4(u(ii, j + 2, k), u(ii, j + 1, k), u(ii, j, k), u(ii, j - 1, k));
          };
          t1 = d4(px(i + 1), px(i), px(i - 1), px(i - 2), dx);  /* duvdx */
          auto pz = [&](int kk) {
            return q4(v(i, j, kk + 2), v(i, j, kk + 1), v(i, j, kk), v(i, j, kk - 1)) *
                   q4(w(i, j + 2, kk), w(i, j + 1, kk), w(i, j, kk), w(i, j - 1, kk));
          };
          t3 = d4(pz(k + 1), pz(k), pz(k - 1), pz(k - 2), dz);  /* dvwdz */
        } else {
          auto sz = [&](int kk) { double a = q4(w(i, j, kk + 1), w(i, j, kk), w(i, j, kk - 1), w(i, j, kk - 2)); return a * a; };
          t3 = d4(sz(k + 2), sz(k + 1), sz(k), sz(k - 1), dz);  /* dw2dz */
          auto px = [&](int ii) {
            return q4(w(ii + 2, j, k), w(ii + 1, j, k), w(ii, j, k), w(ii - 1, j, k)) *
                   q4(u(ii, j, k + 2), u(ii, j, k + 1), u(ii, j, k), u(ii, j, k - 1));
          };
          t1 = d4(px(i + 1), px(i), px(i - 1), px(i - 2), dx);  /* duwdx */
          auto py = [&](int jj) {
            return q4(w(i, jj + 2, k), w(i, jj + 1, k), w(i, jj, k), w(i, jj - 1, k)) *
                   q4(v(i, jj, k + 2), v(i, jj, k + 1), v(i, jj, k), v(i, jj, k - 1));
          };
          t2 = d4(py(j + 1), py(j), py(j - 1), py(j - 2), dy);  /* dvwdy */
        }
        F(B, st, i, j, k) = (F(B, oo, i, j, k) - dt * alfapr * (t1 + t2 + t3));
      }
    });
  }
  par_blocks((int)C.b.size(), [&](int ib) { Blk &B = C.b[ib];
    const double dxx = B.d.dx * B.d.dx, dyy = B.d.dy * B.d.dy, dzz = B.d.dz * B.d.dz;
    for (int op = 1; op <= 3; ++op) {
      double *st = op == 1 ? B.ustar : op == 2 ? B.vstar : B.wstar;
      double *c = field_of(B, op);
      int is, ie, js, je, ks, ke;
      franges(B, op, is, ie, js, je, ks, ke);
      auto f = [&](int i, int j, int k) { return F(B, c, i, j, k); };
      for (int k = ks; k <= ke; ++k) for (int i = is; i <= ie; ++i) for (int j = js; j <= je; ++j) {
        /* u takes the viscosity of its own cell, v and w the one past the face (rungek.for:230, 262, 290) */
        const double visc = op == 1 ? F(B, vis[ib], i, j, k) : op == 2 ? F(B, vis[ib], i, j + 1, k)
                                                                       : F(B, vis[ib], i, j, k + 1);
        const double diff = visc * (
            ((-f(i + 2, j, k) + 16.0 * f(i + 1, j, k) - 30.0 * f(i, j, k) + 16.0 * f(i - 1, j, k) - f(i - 2, j, k)) /
             (12.0 * dxx)) +
            ((-f(i, j + 2, k) + 16.0 * f(i, j + 1, k) - 30.0 * f(i, j, k) + 16.0 * f(i, j - 1, k) - f(i, j - 2, k)) /
             (12.0 * dyy)) +
            ((-f(i, j, k + 2) + 16.0 * f(i, j, k + 1) - 30.0 * f(i, j, k) + 16.0 * f(i, j, k - 1) - f(i, j, k - 2)) /
             (12.0 * dzz)));
        F(B, st, i, j, k) = (F(B, st, i, j, k) + dt * alfapr * diff);
        if (op == 1 && pforce) F(B, st, i, j, k) = F(B, st, i, j, k) + dt * alfapr * forcn;
      }
    }
  });
}

/* HJ_WENO_dx/dy/dz (weno.for:2-354) of field fi of component op along
 * axis ax: the divided differences D1 over 1..n-1 of the axis, then the
 * fifth-order one-sided derivatives at 4..n-3 (plus: D1(L+5)..D1(L+1) with
 * L = I; minus: D1(L+1)..D1(L+5) with L = I-1), zero elsewhere; n, nq, nr
 * are the component's range ends plus pl_ex + 1.  REAL is double
 * (-fdefault-real-8): 1.0E-6, 1.0E-99, 13.0/12.0, 1.0/3.0, ... are double;
 * x**2 is x*x; MAX of the five squares. */
double weno5(double v1, double v2, double v3, double v4, double v5) {
  const double v11 = v1 * v1, v22 = v2 * v2, v33 = v3 * v3, v44 = v4 * v4, v55 = v5 * v5;
  const double e = (1.0E-6) * std::max(std::max(std::max(std::max(v11, v22), v33), v44), v55) + 1.0E-99;
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
void hj_weno(Blk &B, const double *fi, int ax, int npp, int nq, int nr, double h, std::vector<double> &plus,
             std::vector<double> &minus) {
  const size_t n = (size_t)B.ttc_i * B.ttc_j * B.ttc_k;
  std::vector<double> D1(n, 0.0);
  plus.assign(n, 0.0);
  minus.assign(n, 0.0);
  const int lim[3] = {npp, nq, nr};
  auto id = [&](int i, int j, int k) {
    return (size_t)(i - 1) + (size_t)B.ttc_i * ((size_t)(j - 1) + (size_t)B.ttc_j * (size_t)(k - 1));
  };
  auto shift = [&](int i, int j, int k, int d, int &a, int &b, int &c) {
    a = i + (ax == 0 ? d : 0); b = j + (ax == 1 ? d : 0); c = k + (ax == 2 ? d : 0);
  };
  /* divided differences over 1..lim-1 along ax, 1..lim of the others */
  for (int k = 1; k <= lim[2] - (ax == 2); ++k) for (int i = 1; i <= lim[0] - (ax == 0); ++i)
    for (int j = 1; j <= lim[1] - (ax == 1); ++j) {
      int a, b, c;
      shift(i, j, k, 1, a, b, c);
      D1[id(i, j, k)] = (fi[id(a, b, c)] - fi[id(i, j, k)]) / h;
    }
  for (int k = 1; k <= lim[2] - (ax == 2 ? 6 : 0); ++k) for (int i = 1; i <= lim[0] - (ax == 0 ? 6 : 0); ++i)
    for (int j = 1; j <= lim[1] - (ax == 1 ? 6 : 0); ++j) {
      auto d1 = [&](int m) { int a, b, c; shift(i, j, k, m, a, b, c); return D1[id(a, b, c)]; };
      int a, b, c;
      shift(i, j, k, 3, a, b, c);
      plus[id(a, b, c)] = weno5(d1(5), d1(4), d1(3), d1(2), d1(1));    /* L = I */
      minus[id(a, b, c)] = weno5(d1(0), d1(1), d1(2), d1(3), d1(4));   /* L = I - 1 */
    }
}

/* One Runge-Kutta stage of rungek_convWENO (rungek.for:414-582) then
 * rungek_diff2nd, as flosol.for:157-170 runs them for differencing = 3:
 * boundu, HJ_WENO along x, y, z of u, the u loop (each derivative upwinded
 * by the sign of the advecting velocity at the face, 0 where it is 0), and
 * so on for v and w. */
void rungek_weno(Ctx &C, const double *const *uoo, const double *const *voo, const double *const *woo,
                 const double *const *vis, bool pforce, double forcn) {
  const double dt = C.dt, alfapr = C.alfapr;
  const int pll = C.pl_ex + 1;
  for (int op = 1; op <= 3; ++op) {
    bound(C, op);
    par_blocks((int)C.b.size(), [&](int ib) { Blk &B = C.b[ib];
      int is, ie, js, je, ks, ke;
      franges(B, op, is, ie, js, je, ks, ke);
      const double *fi = field_of(B, op);
      std::vector<double> px, mx, py, my, pz, mz;
      hj_weno(B, fi, 0, ie + pll, je + pll, ke + pll, B.d.dx, px, mx);
      hj_weno(B, fi, 1, ie + pll, je + pll, ke + pll, B.d.dy, py, my);
      hj_weno(B, fi, 2, ie + pll, je + pll, ke + pll, B.d.dz, pz, mz);
      double *st = op == 1 ? B.ustar : op == 2 ? B.vstar : B.wstar;
      const double *oo = op == 1 ? uoo[ib] : op == 2 ? voo[ib] : woo[ib];
      auto u = [&](int i, int j, int k) { return F(B, B.u, i, j, k); };
      auto v = [&](int i, int j, int k) { return F(B, B.v, i, j, k); };
      auto w = [&](int i, int j, int k) { return F(B, B.w, i, j, k); };
      auto up = [&](double a, const std::vector<double> &mn, const std::vector<double> &pls, int i, int j, int k) {
        const double m = F(B, mn.data(), i, j, k), pv = F(B, pls.data(), i, j, k);
        return a > 0.0 ? m : a < 0.0 ? pv : 0.0;
      };
      for (int k = ks; k <= ke; ++k) for (int i = is; i <= ie; ++i) for (int j = js; j <= je; ++j) {
        double t1, t2, t3;
        if (op == 1) {
          const double uc = u(i, j, k);
          const double vijk = 0.25 * (v(i, j, k) + v(i + 1, j, k) + v(i, j - 1, k) + v(i + 1, j - 1, k));
          const double wijk = 0.25 * (w(i, j, k) + w(i + 1, j, k) + w(i, j, k - 1) + w(i + 1, j, k - 1));
          t1 = uc * up(uc, mx, px, i, j, k);
          t2 = vijk * up(vijk, my, py, i, j, k);
          t3 = wijk * up(wijk, mz, pz, i, j, k);
        } else if (op == 2) {
          const double vc = v(i, j, k);
          const double uijk = 0.25 * (u(i, j, k) + u(i, j + 1, k) + u(i - 1, j, k) + u(i - 1, j + 1, k));
          const double wijk = 0.25 * (w(i, j, k) + w(i, j + 1, k) + w(i, j, k - 1) + w(i, j + 1, k - 1));
          t1 = uijk * up(uijk, mx, px, i, j, k);
          t2 = vc * up(vc, my, py, i, j, k);
          t3 = wijk * up(wijk, mz, pz, i, j, k);
        } else {
          const double wc = w(i, j, k);
          const double uijk = 0.25 * (u(i, j, k) + u(i, j, k + 1) + u(i - 1, j, k) + u(i - 1, j, k + 1));
          const double vijk = 0.25 * (v(i, j, k) + v(i, j, k + 1) + v(i, j - 1, k) + v(i, j - 1, k + 1));
          t1 = uijk * up(uijk, mx, px, i, j, k);
          t2 = vijk * up(vijk, my, py, i, j, k);
          t3 = wc * up(wc, mz, pz, i, j, k);
        }
        F(B, st, i, j, k) = (F(B, oo, i, j, k) - dt * alfapr * (t1 + t2 + t3));
      }
    });
  }
  diff2nd(C, vis, pforce, forcn);
}

/* EXT: distance between the centres of cells a and a+1 along an axis,
 * equal to dx on a uniform grid. */
inline double dface(const std::vector<double> &w, int a0) { return 0.5 * (w[a0] + w[a0 + 1]); }

/* calvel (press.for:139-200), both branches. */
void calvel(Ctx &C) {
  double dt = C.dt, alfapr = C.alfapr;
  par_blocks((int)C.b.size(), [&](int ib_) { Blk &B = C.b[ib_];
    int o = B.isp - 1; /* field index i <-> level-1 ghost-inclusive index i - o */
    if (C.lsm) { /* press.for:152-190 */
      double *d = B.dens;
      for (int k = B.ksu; k <= B.keu; ++k) for (int i = B.isu; i <= B.ieu; ++i) for (int j = B.jsu; j <= B.jeu; ++j)
        F(B, B.u, i, j, k) = (F(B, B.ustar, i, j, k) - dt * alfapr * (F(B, B.p, i + 1, j, k) - F(B, B.p, i, j, k)) /
                              B.d.dx / (0.5 * (F(B, d, i, j, k) + F(B, d, i + 1, j, k))));
      for (int k = B.ksv; k <= B.kev; ++k) for (int i = B.isv; i <= B.iev; ++i) for (int j = B.jsv; j <= B.jev; ++j)
        F(B, B.v, i, j, k) = (F(B, B.vstar, i, j, k) - dt * alfapr * (F(B, B.p, i, j + 1, k) - F(B, B.p, i, j, k)) /
                              B.d.dy / (0.5 * (F(B, d, i, j, k) + F(B, d, i, j + 1, k))));
      for (int k = B.ksw; k <= B.kew; ++k) for (int i = B.isw; i <= B.iew; ++i) for (int j = B.jsw; j <= B.jew; ++j)
        F(B, B.w, i, j, k) = (F(B, B.wstar, i, j, k) - dt * alfapr * (F(B, B.p, i, j, k + 1) - F(B, B.p, i, j, k)) /
                              B.d.dz / (0.5 * (F(B, d, i, j, k) + F(B, d, i, j, k + 1))));
      return;
    }
    for (int k = B.ksu; k <= B.keu; ++k) for (int i = B.isu; i <= B.ieu; ++i) for (int j = B.jsu; j <= B.jeu; ++j) {
      double dxl = B.stretched ? dface(B.hx[1], i - o) : B.d.dx;
      F(B, B.u, i, j, k) = (F(B, B.ustar, i, j, k) - dt * alfapr * (F(B, B.p, i + 1, j, k) - F(B, B.p, i, j, k)) / dxl);
    }
    for (int k = B.ksv; k <= B.kev; ++k) for (int i = B.isv; i <= B.iev; ++i) for (int j = B.jsv; j <= B.jev; ++j) {
      double dyl = B.stretched ? dface(B.hy[1], j - o) : B.d.dy;
      F(B, B.v, i, j, k) = (F(B, B.vstar, i, j, k) - dt * alfapr * (F(B, B.p, i, j + 1, k) - F(B, B.p, i, j, k)) / dyl);
    }
    for (int k = B.ksw; k <= B.kew; ++k) for (int i = B.isw; i <= B.iew; ++i) for (int j = B.jsw; j <= B.jew; ++j) {
      double dzl = B.stretched ? dface(B.hz[1], k - o) : B.d.dz;
      F(B, B.w, i, j, k) = (F(B, B.wstar, i, j, k) - dt * alfapr * (F(B, B.p, i, j, k + 1) - F(B, B.p, i, j, k)) / dzl);
    }
  });
  exchange(C, 1);
  exchange(C, 2);
  exchange(C, 3);
}

/* calmas (press.for:2-75): the 4th-order branch (differencing 2, :13-35;
 * uniform spacing only, 27.0 and 24.0 are double under -fdefault-real-8)
 * and the 2nd-order one (differencing 1 or 3, :38-67) with both L_LSM
 * branches. */
void calmas(Ctx &C) {
  double rmax = 0.0;
  std::vector<double> bmax(C.b.size(), 0.0);
  if (C.differencing == 2) {
    par_blocks((int)C.b.size(), [&](int ib_) { Blk &B = C.b[ib_]; double rmax = 0.0, resor;
      const double dx = B.d.dx, dy = B.d.dy, dz = B.d.dz;
      for (int k = B.ksp; k <= B.kep; ++k) for (int i = B.isp; i <= B.iep; ++i) for (int j = B.jsp; j <= B.jep; ++j) {
        double fact = ((-F(B, B.u, i + 1, j, k) + 27.0 * F(B, B.u, i, j, k) - 27.0 * F(B, B.u, i - 1, j, k) +
                        F(B, B.u, i - 2, j, k)) / (24.0 * dx) +
                       (-F(B, B.v, i, j + 1, k) + 27.0 * F(B, B.v, i, j, k) - 27.0 * F(B, B.v, i, j - 1, k) +
                        F(B, B.v, i, j - 2, k)) / (24.0 * dy) +
                       (-F(B, B.w, i, j, k + 1) + 27.0 * F(B, B.w, i, j, k) - 27.0 * F(B, B.w, i, j, k - 1) +
                        F(B, B.w, i, j, k - 2)) / (24.0 * dz));
        F(B, B.su.data(), i, j, k) = fact / C.dt;
        double fact1 = fact * dx * dy * dz;
        resor = std::max(rmax, std::fabs(fact1));
        rmax = std::max(resor, std::fabs(fact1));
      }
      bmax[ib_] = rmax;
    });
    for (double m : bmax) rmax = std::max(rmax, m);
    C.rmax = rmax;
    return;
  }
  par_blocks((int)C.b.size(), [&](int ib_) { Blk &B = C.b[ib_]; double rmax = 0.0, resor;
    int o = B.isp - 1;
    for (int k = B.ksp; k <= B.kep; ++k) for (int i = B.isp; i <= B.iep; ++i) for (int j = B.jsp; j <= B.jep; ++j) {
      double hxl = B.stretched ? B.hx[1][i - o] : B.d.dx;
      double hyl = B.stretched ? B.hy[1][j - o] : B.d.dy;
      double hzl = B.stretched ? B.hz[1][k - o] : B.d.dz;
      double fact = ((F(B, B.u, i, j, k) - F(B, B.u, i - 1, j, k)) / hxl +
                     (F(B, B.v, i, j, k) - F(B, B.v, i, j - 1, k)) / hyl +
                     (F(B, B.w, i, j, k) - F(B, B.w, i, j, k - 1)) / hzl);
      if (C.lsm) /* press.for:51-53: sup, copied to the rhs by mgkcyc */
        F(B, B.su.data(), i, j, k) = fact * B.d.dx * B.d.dy * B.d.dz / C.dt;
      else
        F(B, B.su.data(), i, j, k) = fact / C.dt;
      double fact1 = fact * hxl * hyl * hzl;
      resor = std::max(rmax, std::fabs(fact1));
      rmax = std::max(resor, std::fabs(fact1));
    }
    bmax[ib_] = rmax;
  });
  /* blocks reduce like the ranks of MPI_ALLREDUCE(MAX): order-free */
  for (double m : bmax) rmax = std::max(rmax, m);
  C.rmax = rmax;
}

/* newsolv_mg (newsolv_mg.for:2-102) */
int newsolv_mg(Ctx &C, double *hist, int cap, mf3d_solve_info *info) {
  stamp(0);
  if (C.lsm) coeff(C); /* newsolv_mg.for:12-14 */
  calvel(C);
  calmas(C);
  stamp(1);
  double rmax0 = C.rmax;
  for (auto &B : C.b) std::fill(B.pp.begin(), B.pp.end(), 0.0);
  double eps = C.eps_relative ? C.eps * rmax0 : C.eps;
  int iter;
  bool conv = false;
  for (iter = 1; iter <= C.maxcy; ++iter) {
    mgkcyc(C);
    double ppref = 0.0;
    par_blocks((int)C.b.size(), [&](int ib_) { Blk &B = C.b[ib_];
      for (int k = B.ksp - 1; k <= B.kep + 1; ++k) for (int i = B.isp - 1; i <= B.iep + 1; ++i) for (int j = B.jsp - 1; j <= B.jep + 1; ++j) {
        F(B, B.p, i, j, k) = (F(B, B.p, i, j, k) + (F(B, B.pp.data(), i, j, k) - ppref));
        F(B, B.pp.data(), i, j, k) = 0.0;
      }
    });
    exchange(C, 4);
    pbound(C);
    calvel(C);
    calmas(C);
    if (hist && iter - 1 < cap) hist[iter - 1] = C.rmax;
    stamp(iter + 1);
    if (C.rmax < eps && iter > 1) { conv = true; break; }
  }
  int status = MF3D_OK;
  int iters = conv ? iter : C.maxcy;
  if (!conv) status = MF3D_NOT_CONVERGED;
  if (C.rmax > 100.0) status = MF3D_DIVERGED;
  /* newsolv_mg.for:84-88 (the reference stops first when rmax > 100) */
  if (C.bounds && status != MF3D_DIVERGED) {
    g_wall_fail = false;
    bound(C, 1); bound(C, 2); bound(C, 3);
    if (g_wall_fail) { g_err = "log_law: USTAR DOESNT CONVERGE"; return MF3D_E_INVALID; }
  }
  if (info) {
    info->rmax = C.rmax; info->rmax0 = rmax0; info->iter = iters; info->status = status; info->ms_device = 0.0;
  }
  return status;
}

/* ------------------------------------------------------------------ */
/* solver = 1: pressure_1sweep (press.for:274-420) with Stone's SIP      */
/* (sipsol.for:2-206, ifi = 44), every block on one rank.                */
/* ------------------------------------------------------------------ */
/* The per-cell coefficients pressure_1sweep sets (press.for:294-320):
 * 1/(dx*dx) etc., zeroed on Neumann faces, ap = -(sum) in order. */
struct SipCoef { double aw, ae, as, an, ab, at, ap; };
SipCoef sip_coef(const Blk &B, int i, int j, int k) {
  SipCoef c;
  c.aw = 1.0 / (B.d.dx * B.d.dx); c.ae = 1.0 / (B.d.dx * B.d.dx);
  c.an = 1.0 / (B.d.dy * B.d.dy); c.as = 1.0 / (B.d.dy * B.d.dy);
  c.at = 1.0 / (B.d.dz * B.d.dz); c.ab = 1.0 / (B.d.dz * B.d.dz);
  if (B.d.iprev < 0 && B.d.bc_west != 5 && i == B.isp) c.aw = 0.0;
  if (B.d.inext < 0 && B.d.bc_east != 5 && i == B.iep) c.ae = 0.0;
  if (B.d.jprev < 0 && B.d.bc_south != 5 && j == B.jsp) c.as = 0.0;
  if (B.d.jnext < 0 && B.d.bc_north != 5 && j == B.jep) c.an = 0.0;
  if (B.d.kprev < 0 && B.d.bc_bottom != 5 && k == B.ksp) c.ab = 0.0;
  if (B.d.knext < 0 && B.d.bc_top != 5 && k == B.kep) c.at = 0.0;
  c.ap = -1.0 * (c.aw + c.ae + c.as + c.an + c.ab + c.at);
  return c;
}

/* sipsol(44): the ILU factors (recomputed at every call, as the reference
 * does), then up to nswp sweeps of residual, forward and backward
 * substitution, each followed by exchange(44); the sweep loop stops when
 * the summed |residual| falls to 0.001 of the first sweep's or changes by
 * at most 1e-5 of it between sweeps.  Arrays indexed as the reference:
 * ijk = j + (i-1)*nj + (k-1)*nij over the ghost-inclusive box, j fastest,
 * zero outside the interior. */
void sipsol44(Ctx &C) {
  const double alfa = 0.92, small = 1e-20;
  size_t nmax = 0;
  for (auto &B : C.b) nmax = std::max(nmax, (size_t)B.ttc_i * B.ttc_j * B.ttc_k);
  size_t nb = C.b.size();
  std::vector<double> ue(nb * (nmax + 1), 0.0), un(ue), ut(ue), lw(ue), ls(ue), lb(ue), lpr(ue), res(ue);
  for (size_t ib = 0; ib < nb; ++ib) {
    Blk &B = C.b[ib];
    const long nj = B.ttc_j, nij = (long)B.ttc_i * B.ttc_j;
    const size_t o = ib * (nmax + 1);
    for (int k = B.ksp; k <= B.kep; ++k) for (int i = B.isp; i <= B.iep; ++i) for (int j = B.jsp; j <= B.jep; ++j) {
      const long ijk = j + (long)(i - 1) * nj + (long)(k - 1) * nij;
      const SipCoef c = sip_coef(B, i, j, k);
      const size_t q = o + ijk;
      lb[q] = c.ab / (1. + alfa * (un[q - nij] + ue[q - nij]));
      lw[q] = c.aw / (1. + alfa * (un[q - nj] + ut[q - nj]));
      ls[q] = c.as / (1. + alfa * (ue[q - 1] + ut[q - 1]));
      const double p1 = alfa * (lb[q] * un[q - nij] + lw[q] * un[q - nj]);
      const double p2 = alfa * (lb[q] * ue[q - nij] + ls[q] * ue[q - 1]);
      const double p3 = alfa * (lw[q] * ut[q - nj] + ls[q] * ut[q - 1]);
      lpr[q] = 1. / (c.ap + p1 + p2 + p3 - lb[q] * ut[q - nij] - lw[q] * ue[q - nj] - ls[q] * un[q - 1] + small);
      un[q] = (c.an - p1) * lpr[q];
      ue[q] = (c.ae - p2) * lpr[q];
      ut[q] = (c.at - p3) * lpr[q];
    }
  }
  double relast = 0.0, res1 = 0.0;
  int nsweep;
  bool stop = false;
  for (nsweep = 1; nsweep <= C.nswp; ++nsweep) {
    double resab = 0.0;
    for (size_t ib = 0; ib < nb; ++ib) {
      Blk &B = C.b[ib];
      double *fi = B.pp.data(), *su = B.su.data();
      const long nj = B.ttc_j, nij = (long)B.ttc_i * B.ttc_j;
      const size_t o = ib * (nmax + 1);
      for (int k = B.ksp; k <= B.kep; ++k) for (int i = B.isp; i <= B.iep; ++i) for (int j = B.jsp; j <= B.jep; ++j) {
        const size_t q = o + j + (long)(i - 1) * nj + (long)(k - 1) * nij;
        const SipCoef c = sip_coef(B, i, j, k);
        res[q] = (F(B, su, i, j, k) - c.ap * F(B, fi, i, j, k) - c.an * F(B, fi, i, j + 1, k) -
                  c.as * F(B, fi, i, j - 1, k) - c.ae * F(B, fi, i + 1, j, k) - c.aw * F(B, fi, i - 1, j, k) -
                  c.ab * F(B, fi, i, j, k - 1) - c.at * F(B, fi, i, j, k + 1));
        resab = resab + std::fabs(res[q]);
      }
      for (int k = B.ksp; k <= B.kep; ++k) for (int i = B.isp; i <= B.iep; ++i) for (int j = B.jsp; j <= B.jep; ++j) {
        const size_t q = o + j + (long)(i - 1) * nj + (long)(k - 1) * nij;
        res[q] = (res[q] - lb[q] * res[q - nij] - lw[q] * res[q - nj] - ls[q] * res[q - 1]) * lpr[q];
      }
      for (int k = B.kep; k >= B.ksp; --k) for (int i = B.iep; i >= B.isp; --i) for (int j = B.jep; j >= B.jsp; --j) {
        const size_t q = o + j + (long)(i - 1) * nj + (long)(k - 1) * nij;
        res[q] = res[q] - un[q] * res[q + 1] - ue[q] * res[q + nj] - ut[q] * res[q + nij];
        F(B, fi, i, j, k) = F(B, fi, i, j, k) + res[q];
      }
    }
    if (nsweep == 1) res1 = resab;
    const double rsm = resab / (res1 + small);
    exchange(C, 44);
    const double reldif = std::fabs(rsm - relast);
    relast = rsm;
    if (rsm <= 0.001 || reldif <= 0.00001) { stop = true; break; }
  }
  if (!stop) nsweep = nsweep - 1; /* the loop variable ends at nswp+1 */
  C.sip_sweeps += nsweep;
}

/* pressure_1sweep (press.for:274-420): calvel, then up to niter (= maxcy)
 * rounds of calmas, the convergence test (rmax < eps and iter > 1), sipsol,
 * p += pp, exchange(4), pbound, calvel.  hist[q] = rmax of the calmas that
 * opens round q+2 (the last round, when the loop runs out, has none: the
 * reported rmax and su are then those from before its sipsol, as in the
 * reference); info.iter = SIP calls. */
int pressure_1sweep(Ctx &C, double *hist, int cap, mf3d_solve_info *info) {
  stamp(0);
  for (auto &B : C.b) {
    std::fill(B.pp.begin(), B.pp.end(), 0.0);
    std::fill(B.su.begin(), B.su.end(), 0.0);
  }
  calvel(C);
  calmas(C);
  stamp(1);
  const double rmax0 = C.rmax;
  const double eps = C.eps_relative ? C.eps * rmax0 : C.eps;
  C.sip_sweeps = 0;
  int calls = 0;
  bool conv = false;
  for (int iter = 1; iter <= C.maxcy; ++iter) {
    if (iter > 1) {
      if (C.rmax < eps) { conv = true; break; }
    }
    sipsol44(C);
    ++calls;
    const double ppref = 0.0;
    for (auto &B : C.b)
      for (int k = B.ksp - 1; k <= B.kep + 1; ++k) for (int i = B.isp - 1; i <= B.iep + 1; ++i) for (int j = B.jsp - 1; j <= B.jep + 1; ++j) {
        F(B, B.p, i, j, k) = (F(B, B.p, i, j, k) + (F(B, B.pp.data(), i, j, k) - ppref));
        F(B, B.pp.data(), i, j, k) = 0.0;
      }
    exchange(C, 4);
    pbound(C);
    calvel(C);
    stamp(calls + 1);
    if (iter == C.maxcy) break; /* `if (iter.lt.niter) goto 1000` fails: no further calmas */
    calmas(C); /* the next sipsol call starts from it (press.for:323) */
    if (hist && calls - 1 < cap) hist[calls - 1] = C.rmax;
  }
  int status = conv ? MF3D_OK : MF3D_NOT_CONVERGED;
  if (C.rmax > 100.0) status = MF3D_DIVERGED;
  if (C.bounds && status != MF3D_DIVERGED) {
    g_wall_fail = false;
    bound(C, 1); bound(C, 2); bound(C, 3);
    if (g_wall_fail) { g_err = "log_law: USTAR DOESNT CONVERGE"; return MF3D_E_INVALID; }
  }
  if (info) {
    info->rmax = C.rmax; info->rmax0 = rmax0; info->iter = calls; info->status = status; info->ms_device = 0.0;
  }
  return status;
}


/* An inlet code on a west face without a neighbour: its file is there, and
 * the profile codes read uniform cell centres (initial.for:341-365). */
int inlet_check(const Blk &B) {
  const int code = B.d.bc_west;
  if (B.d.iprev >= 0 || !(code == 7 || code == 8 || code == 12 || code == 13)) return MF3D_OK;
  if (code == 7 || code == 8) {
    auto it = g_inlets.find(B.d.id);
    if (it == g_inlets.end() || it->second.code != code) { g_err = "inlet values not set"; return MF3D_E_INVALID; }
    /* u's, v's and w's lines over their own ranges */
    const int js[3] = {B.jsu, B.jsv, B.jsw}, je[3] = {B.jeu, B.jev, B.jew};
    const int ks[3] = {B.ksu, B.ksv, B.ksw}, ke[3] = {B.keu, B.kev, B.kew};
    size_t n = 0;
    for (int c = 0; c < 3; ++c)
      n += code == 7 ? (size_t)(je[c] - js[c] + 3) * (ke[c] - ks[c] + 3) : (size_t)(je[c] - js[c] + 2) * (ke[c] - ks[c] + 2);
    if (it->second.v.size() != n) { g_err = "inlet values: wrong count"; return MF3D_E_INVALID; }
  }
  if (code != 7 && (B.d.hy || B.d.hz)) { g_err = "power-law inlet on a stretched grid"; return MF3D_E_UNSUPPORTED; }
  return MF3D_OK;
}

int setup(Ctx &C, const mf3d_block_desc *blocks, int nb, const mf3d_params *prm) {
  if (nb <= 0 || !blocks || !prm) { g_err = "bad arguments"; return MF3D_E_INVALID; }
  if (prm->mg_itrsch < 1 || prm->mg_itrsch > 3) { g_err = "mg_itrsch"; return MF3D_E_INVALID; }
  if (prm->differencing < 1 || prm->differencing > 3) { g_err = "differencing"; return MF3D_E_INVALID; }
  /* the 4th-order divergence reads u(i-2): two ghost layers */
  if (prm->differencing == 2 && prm->pl < 2) { g_err = "differencing 2 needs pl >= 2"; return MF3D_E_INVALID; }
  if (prm->differencing == 2 && prm->lsm) { g_err = "differencing 2 with L_LSM"; return MF3D_E_INVALID; }
  C.differencing = prm->differencing;
  C.ngrd_gl = prm->ngrid; C.mg_itrsch = prm->mg_itrsch; C.irestr = prm->irestr; C.iproln = prm->iproln;
  C.maxcy = prm->maxcy; C.eps = prm->eps; C.eps_relative = prm->eps_relative; C.pl = prm->pl;
  C.pl_ex = prm->pl_ex;
  if (C.pl_ex < 0 || C.pl_ex >= C.pl) { g_err = "pl_ex"; return MF3D_E_INVALID; }
  C.lsm = prm->lsm != 0;
  C.bounds = prm->bounds != 0;
  C.alfabc = prm->alfabc;
  C.ubulk = prm->ubulk;
  C.solver = prm->solver == 1 ? 1 : 2;
  C.nswp = prm->nswp;
  if (C.solver == 1 && (C.nswp < 1 || C.lsm)) { g_err = "solver 1: nswp >= 1, no lsm"; return MF3D_E_INVALID; }
  C.periodic = false;
  C.b.resize(nb);
  C.yst = blocks[0].ysl; C.yen = blocks[0].yel; C.zst = blocks[0].zsl; C.zen = blocks[0].zel;
  for (int ib = 1; ib < nb; ++ib) {
    C.yst = std::min(C.yst, blocks[ib].ysl); C.yen = std::max(C.yen, blocks[ib].yel);
    C.zst = std::min(C.zst, blocks[ib].zsl); C.zen = std::max(C.zen, blocks[ib].zel);
  }
  /* LMR (localparameters.for:26-102): a block's refinement rdiv is its
   * spacing against the coarsest block's, a power of two; ngrd_gl =
   * ngrid_input + log2(max rdiv) is the level count passed in, and a block
   * of refinement r keeps ngrid_input + log2(r) levels of its own. */
  std::vector<int> rdiv(nb, 1);
  int lg_max = 0;
  {
    double hmax = 0.0;
    for (int ib = 0; ib < nb; ++ib) hmax = std::max(hmax, blocks[ib].dx);
    for (int ib = 0; ib < nb; ++ib) {
      const mf3d_block_desc &d = blocks[ib];
      const double r = hmax / d.dx;
      const long q = std::lround(r);
      if (q < 1 || (q & (q - 1)) || std::fabs(r - (double)q) > 1e-8 * r ||
          std::fabs(blocks[0].dx / blocks[0].dy * d.dy - d.dx) > 1e-8 * d.dx ||
          std::fabs(blocks[0].dx / blocks[0].dz * d.dz - d.dx) > 1e-8 * d.dx) {
        g_err = "LMR: block spacings are not powers of two of one another"; return MF3D_E_INVALID;
      }
      rdiv[ib] = (int)q;
      if (q > 1) C.lmr = true;
      int lg = 0;
      while ((1L << lg) < q) ++lg;
      lg_max = std::max(lg_max, lg);
    }
    if (C.lmr) {
      if (prm->ngrid - lg_max < 1) { g_err = "LMR: ngrid below log2(max rdiv) + 1"; return MF3D_E_INVALID; }
      if (C.lsm) { g_err = "LMR with L_LSM"; return MF3D_E_UNSUPPORTED; }
      if (C.solver == 1) { g_err = "LMR with solver 1"; return MF3D_E_UNSUPPORTED; }
      for (int ib = 0; ib < nb; ++ib)
        if (blocks[ib].hx || blocks[ib].hy || blocks[ib].hz) { g_err = "LMR on a stretched grid"; return MF3D_E_UNSUPPORTED; }
    }
  }
  for (int ib = 0; ib < nb; ++ib) {
    Blk &B = C.b[ib];
    B.d = blocks[ib];
    B.rdiv = rdiv[ib];
    {
      int lg = 0;
      while ((1 << lg) < B.rdiv) ++lg;
      B.ngrid = prm->ngrid - lg_max + lg; /* localparameters.for:42-45 */
    }
    int pl = prm->pl;
    int pow2 = 1 << (B.ngrid - 1);
    if (B.d.nx % pow2 || B.d.ny % pow2 || B.d.nz % pow2) { g_err = "not divisible"; return MF3D_E_INVALID; }
    if (B.d.nx <= C.pl_ex || B.d.ny <= C.pl_ex || B.d.nz <= C.pl_ex) { g_err = "block edge <= pl_ex"; return MF3D_E_INVALID; }
    C.indid[B.d.id] = ib;
    B.isp = 1 + pl; B.iep = B.d.nx + B.isp - 1;
    B.jsp = 1 + pl; B.jep = B.d.ny + B.jsp - 1;
    B.ksp = 1 + pl; B.kep = B.d.nz + B.ksp - 1;
    B.isu = B.isv = B.isw = B.isp; B.ieu = B.iev = B.iew = B.iep;
    B.jsu = B.jsv = B.jsw = B.jsp; B.jeu = B.jev = B.jew = B.jep;
    B.ksu = B.ksv = B.ksw = B.ksp; B.keu = B.kev = B.kew = B.kep;
    if (B.d.inext < 0 && B.d.bc_east != 5) B.ieu = B.ieu - 1;
    if (B.d.jnext < 0 && B.d.bc_north != 5) B.jev = B.jev - 1;
    if (B.d.knext < 0 && B.d.bc_top != 5) B.kew = B.kew - 1;
    B.ttc_i = B.d.nx + 2 * pl; B.ttc_j = B.d.ny + 2 * pl; B.ttc_k = B.d.nz + 2 * pl;
    if (B.d.bc_west == 5 || B.d.bc_east == 5 || B.d.bc_south == 5 || B.d.bc_north == 5 || B.d.bc_bottom == 5 || B.d.bc_top == 5)
      C.periodic = true;
    B.stretched = B.d.hx || B.d.hy || B.d.hz;
    if (C.lsm && B.stretched) { g_err = "L_LSM on a stretched grid"; return MF3D_E_UNSUPPORTED; }
    if (C.differencing == 2 && B.stretched) { g_err = "differencing 2 on a stretched grid"; return MF3D_E_UNSUPPORTED; }
    if (C.bounds) {
      const int bcs[6] = {B.d.bc_west, B.d.bc_east, B.d.bc_south, B.d.bc_north, B.d.bc_bottom, B.d.bc_top};
      const int nbr[6] = {B.d.iprev, B.d.inext, B.d.jprev, B.d.jnext, B.d.kprev, B.d.knext};
      for (int f = 0; f < 6; ++f)
        if (nbr[f] < 0 && bounds_code_unsupported(f, bcs[f], C.lsm, C.alfabc, (size_t)ib < g_old.size()))
          { g_err = "bounds: face code"; return MF3D_E_UNSUPPORTED; }
      if (int st = inlet_check(B)) return st;
      if ((size_t)ib < g_old.size())
        for (int a = 0; a < 3; ++a) B.oo[a] = g_old[ib][a];
    }
    B.hx = level_widths(B.d.hx, B.d.nx, B.d.dx, B.ngrid);
    B.hy = level_widths(B.d.hy, B.d.ny, B.d.dy, B.ngrid);
    B.hz = level_widths(B.d.hz, B.d.nz, B.d.dz, B.ngrid);
    size_t ttc = (size_t)B.ttc_i * B.ttc_j * B.ttc_k;
    B.su.assign(ttc, 0.0);
    B.pp.assign(ttc, 0.0);
  }
  /* rdv(dom, g) (localparameters.for:47-57): the block's refinement on the
   * levels the coarsest blocks have, halving on its extra levels, 1 below
   * its own last level */
  const int act_ngrid = prm->ngrid - lg_max;
  for (auto &B : C.b) {
    B.rdv.assign(C.ngrd_gl + 1, 1);
    for (int g = 1; g <= C.ngrd_gl; ++g) {
      if (g > B.ngrid) B.rdv[g] = 1;
      else if (g <= act_ngrid) B.rdv[g] = B.rdiv;
      else B.rdv[g] = B.rdv[g - 1] / 2;
    }
  }
  if (C.lmr) {
    /* alloc_dom.for:12-230: neighbours differ by a factor of 2 at most, and
     * periodic partners not at all */
    for (auto &B : C.b) {
      const int nbr[6] = {B.d.iprev, B.d.inext, B.d.jprev, B.d.jnext, B.d.kprev, B.d.knext};
      std::vector<int> all(nbr, nbr + 6);
      for (int q = 0; q < 4; ++q) { all.push_back(B.d.corprev[q]); all.push_back(B.d.cornext[q]); }
      for (int q = 0; q < 6; ++q) { all.push_back(B.d.edgprev[q]); all.push_back(B.d.edgnext[q]); }
      for (int id : all) {
        if (id < 0) continue;
        auto it = C.indid.find(id);
        if (it == C.indid.end()) { g_err = "neighbour id not in the layout"; return MF3D_E_INVALID; }
        const int r = C.b[it->second].rdiv;
        if (r != B.rdiv && r != 2 * B.rdiv && 2 * r != B.rdiv) { g_err = "wrong rdiv"; return MF3D_E_INVALID; }
      }
      const int per[6] = {B.d.per_ip, B.d.per_in, B.d.per_jp, B.d.per_jn, B.d.per_kp, B.d.per_kn};
      for (int id : per)
        if (id >= 0 && C.indid.count(id) && C.b[C.indid.at(id)].rdiv != B.rdiv) {
          g_err = "wrong rdiv for a periodic partner"; return MF3D_E_INVALID;
        }
    }
  }
  coeff(C);
  return MF3D_OK;
}

} /* namespace */

extern "C" {

const char *orc_last_error(void) { return g_err.c_str(); }

/* The content of block `id`'s inlet file (west code 7: u per line; code 8:
 * the first column "up" of the SEM file, UPROF_SEM = uprof); n values. */
int orc_set_inlet(int id, int code, int uprof, const double *v, long long n) {
  if ((code != 7 && code != 8) || n < 0 || (n && !v)) { g_err = "orc_set_inlet: bad arguments"; return MF3D_E_INVALID; }
  g_inlets[id] = InletFile{code, uprof, std::vector<double>(v, v + n)};
  return MF3D_OK;
}
void orc_clear_inlets(void) { g_inlets.clear(); }

/* Re and fric (control.cin) of the wall functions; re = 0 withdraws them.
 * Clears the kept wall stresses. */
int orc_set_wall_model(double re, double fric) {
  g_re = re;
  g_fric = fric;
  g_tau.clear();
  return MF3D_OK;
}

/* uoo, voo, woo of every block (position order) for the solve's convective
 * outflow faces; nb = 0 unbinds. */
int orc_bind_old_velocity(int nb, const double *const *uoo, const double *const *voo, const double *const *woo) {
  g_old.clear();
  for (int b = 0; b < nb; ++b) g_old.push_back({uoo[b], voo[b], woo[b]});
  return MF3D_OK;
}

/* Threads for the per-block loops (1 = serial, the default). */
void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

/* LMR: the value of the receive-buffer entries that no sender writes (the
 * ring of a fine block's face buffer next to a coarser neighbour). */
void orc_set_lmr_ring(double v) { g_lmr_ring = v; }

/* Wall-clock stamps of the next orc_newsolv_mg: t[0] at entry, t[1] after
 * the initial calvel/calmas, t[1+q] after outer iteration q (NULL = off). */
void orc_set_timestamps(double *t, int cap) { g_tstamp = t; g_tcap = t ? cap : 0; }

/* The whole projection on host arrays, in place. */
int orc_newsolv_mg(const mf3d_block_desc *blocks, int nb, const mf3d_params *prm, const mf3d_fields *fields,
                   double dt, double alfapr, mf3d_solve_info *info, double *hist, int cap) {
  Ctx C;
  int st = setup(C, blocks, nb, prm);
  if (st) return st;
  if (C.lmr) { g_err = "LMR: the field exchanges at refinement interfaces (exchangep.for, exchangeu/v/w.for) are not restated"; return MF3D_E_UNSUPPORTED; }
  C.dt = dt; C.alfapr = alfapr;
  for (int ib = 0; ib < nb; ++ib) {
    Blk &B = C.b[ib];
    B.ustar = fields[ib].ustar; B.vstar = fields[ib].vstar; B.wstar = fields[ib].wstar;
    B.u = fields[ib].u; B.v = fields[ib].v; B.w = fields[ib].w; B.p = fields[ib].p;
    B.dens = fields[ib].dens;
    if (C.lsm && !B.dens) { g_err = "L_LSM needs dens"; return MF3D_E_INVALID; }
  }
  st = C.solver == 1 ? pressure_1sweep(C, hist, cap, info) : newsolv_mg(C, hist, cap, info);
  for (int ib = 0; ib < nb; ++ib)
    if (fields[ib].su) std::memcpy(fields[ib].su, C.b[ib].su.data(), C.b[ib].su.size() * sizeof(double));
  return st;
}

/* One Runge-Kutta stage of the predictor (rungek_conv2nd + rungek_diff2nd)
 * on host arrays: u, v, w in (ghosts refreshed by boundu/v/w), ustar, vstar,
 * wstar out.  alfabc as the reference sets it per stage. */
int orc_rungek_2nd(const mf3d_block_desc *blocks, int nb, const mf3d_params *prm, const mf3d_fields *fields,
                   const mf3d_rk_fields *rk, double dt, double alfapr, int alfabc, int pressureforce, double forcn) {
  Ctx C;
  mf3d_params p = *prm;
  p.bounds = 0;  /* the face codes are checked below, with uoo at hand */
  p.alfabc = alfabc;
  int st = setup(C, blocks, nb, &p);
  if (st) return st;
  if (C.lmr) { g_err = "LMR: the field exchanges at refinement interfaces (exchangep.for, exchangeu/v/w.for) are not restated"; return MF3D_E_UNSUPPORTED; }
  if (C.lsm) { g_err = "rungek_2nd: no L_LSM branch"; return MF3D_E_UNSUPPORTED; }
  C.bounds = true;
  for (auto &B : C.b) {
    const int bcs[6] = {B.d.bc_west, B.d.bc_east, B.d.bc_south, B.d.bc_north, B.d.bc_bottom, B.d.bc_top};
    const int nbr[6] = {B.d.iprev, B.d.inext, B.d.jprev, B.d.jnext, B.d.kprev, B.d.knext};
    for (int f = 0; f < 6; ++f)
      if (nbr[f] < 0 && bounds_code_unsupported(f, bcs[f], false, alfabc, true)) { g_err = "bounds: face code"; return MF3D_E_UNSUPPORTED; }
    if (int e = inlet_check(B)) return e;
  }
  C.dt = dt; C.alfapr = alfapr;
  std::vector<const double *> uoo(nb), voo(nb), woo(nb), vis(nb);
  for (int ib = 0; ib < nb; ++ib) {
    Blk &B = C.b[ib];
    if (B.stretched) { g_err = "rungek_2nd: uniform spacing only"; return MF3D_E_UNSUPPORTED; }
    B.ustar = fields[ib].ustar; B.vstar = fields[ib].vstar; B.wstar = fields[ib].wstar;
    B.u = fields[ib].u; B.v = fields[ib].v; B.w = fields[ib].w; B.p = fields[ib].p;
    uoo[ib] = rk[ib].uoo; voo[ib] = rk[ib].voo; woo[ib] = rk[ib].woo; vis[ib] = rk[ib].vis;
    B.oo[0] = rk[ib].uoo; B.oo[1] = rk[ib].voo; B.oo[2] = rk[ib].woo;
  }
  if (C.differencing == 2) {
    /* rungek_conv4th reads u(i-3) .. u(i+3) */
    if (C.pl < 3) { g_err = "rungek 4th order: needs pl >= 3"; return MF3D_E_INVALID; }
    rungek_4th(C, uoo.data(), voo.data(), woo.data(), vis.data(), pressureforce != 0, forcn);
  } else if (C.differencing == 3) {
    /* HJ_WENO's stencils reach 3 cells and its ranges pl_ex + 1 past the
     * component's end; initial.for:114-117 sets pl_ex = 2 for WENO */
    if (C.pl < 3 || C.pl_ex + 1 > C.pl) { g_err = "rungek WENO: needs pl >= 3"; return MF3D_E_INVALID; }
    rungek_weno(C, uoo.data(), voo.data(), woo.data(), vis.data(), pressureforce != 0, forcn);
  } else {
    rungek_2nd(C, uoo.data(), voo.data(), woo.data(), vis.data(), pressureforce != 0, forcn);
  }
  return MF3D_OK;
}

/* boundu, boundv, boundw alone on host arrays (bounds.for:2-916): u, v, w
 * in/out, with dt, alfapr and alfabc as the caller's time step has them. */
int orc_bounds(const mf3d_block_desc *blocks, int nb, const mf3d_params *prm, const mf3d_fields *fields, double dt,
               double alfapr, int alfabc) {
  Ctx C;
  mf3d_params p = *prm;
  p.bounds = 1;
  p.alfabc = alfabc;
  int st = setup(C, blocks, nb, &p);
  if (st) return st;
  if (C.lmr) { g_err = "LMR: the field exchanges at refinement interfaces (exchangep.for, exchangeu/v/w.for) are not restated"; return MF3D_E_UNSUPPORTED; }
  C.dt = dt; C.alfapr = alfapr;
  for (int ib = 0; ib < nb; ++ib) {
    Blk &B = C.b[ib];
    B.u = fields[ib].u; B.v = fields[ib].v; B.w = fields[ib].w;
  }
  g_wall_fail = false;
  bound(C, 1); bound(C, 2); bound(C, 3);
  if (g_wall_fail) { g_err = "log_law: USTAR DOESNT CONVERGE"; return MF3D_E_INVALID; }
  return MF3D_OK;
}

/* exchange(op) alone on host arrays (exchange.for:2-23), op 1..3 = u, v, w
 * with pl_ex layers, 4 = p with one layer followed by pbound. */
int orc_exchange(const mf3d_block_desc *blocks, int nb, const mf3d_params *prm, const mf3d_fields *fields, int op) {
  if (op < 1 || op > 4) { g_err = "op"; return MF3D_E_INVALID; }
  Ctx C;
  int st = setup(C, blocks, nb, prm);
  if (st) return st;
  if (C.lmr) { g_err = "LMR: the field exchanges at refinement interfaces (exchangep.for, exchangeu/v/w.for) are not restated"; return MF3D_E_UNSUPPORTED; }
  for (int ib = 0; ib < nb; ++ib) {
    Blk &B = C.b[ib];
    B.u = fields[ib].u; B.v = fields[ib].v; B.w = fields[ib].w; B.p = fields[ib].p;
  }
  exchange(C, op);
  if (op == 4) pbound(C);
  return MF3D_OK;
}

/* calvel alone (press.for:139-198 with its exchange(1..3)) on host arrays. */
int orc_calvel(const mf3d_block_desc *blocks, int nb, const mf3d_params *prm, const mf3d_fields *fields, double dt,
               double alfapr) {
  Ctx C;
  int st = setup(C, blocks, nb, prm);
  if (st) return st;
  if (C.lmr) { g_err = "LMR: the field exchanges at refinement interfaces (exchangep.for, exchangeu/v/w.for) are not restated"; return MF3D_E_UNSUPPORTED; }
  if (C.lsm) { g_err = "calvel: no L_LSM here"; return MF3D_E_UNSUPPORTED; }
  C.dt = dt; C.alfapr = alfapr;
  for (int ib = 0; ib < nb; ++ib) {
    Blk &B = C.b[ib];
    B.ustar = fields[ib].ustar; B.vstar = fields[ib].vstar; B.wstar = fields[ib].wstar;
    B.u = fields[ib].u; B.v = fields[ib].v; B.w = fields[ib].w; B.p = fields[ib].p;
  }
  calvel(C);
  return MF3D_OK;
}

/* One V-cycle: su[b] (ttc) in, pp[b] (ttc) out, starting from pp = 0. */
int orc_mgkcyc(const mf3d_block_desc *blocks, int nb, const mf3d_params *prm, double *const *su, double *const *pp) {
  Ctx C;
  int st = setup(C, blocks, nb, prm);
  if (st) return st;
  for (int ib = 0; ib < nb; ++ib) {
    Blk &B = C.b[ib];
    std::memcpy(B.su.data(), su[ib], B.su.size() * sizeof(double));
  }
  mgkcyc(C);
  for (int ib = 0; ib < nb; ++ib) std::memcpy(pp[ib], C.b[ib].pp.data(), C.b[ib].pp.size() * sizeof(double));
  return MF3D_OK;
}

/* exchangepp (+ mgbound + exchbc_mgpp) on level `level` of arrays given
 * ghost-inclusive, i fastest: fi[b][(k*(ny+2) + j)*(nx+2) + i]. */
int orc_exchangepp(const mf3d_block_desc *blocks, int nb, int ngrid, int level, double *const *fi) {
  mf3d_params prm;
  std::memset(&prm, 0, sizeof prm);
  prm.ngrid = ngrid; prm.mg_itrsch = 3; prm.irestr = 1; prm.iproln = 1; prm.maxcy = 1; prm.pl = 1; prm.differencing = 1;
  Ctx C;
  int st = setup(C, blocks, nb, &prm);
  if (st) return st;
  for (int ib = 0; ib < nb; ++ib) {
    Blk &B = C.b[ib];
    Lev L = lev(C, B, level);
    for (int k = 1; k <= L.nk; ++k) for (int j = 1; j <= L.nj; ++j) for (int i = 1; i <= L.ni; ++i)
      B.cof[PH(L, i, j, k)] = fi[ib][((size_t)(k - 1) * L.nj + (j - 1)) * L.ni + (i - 1)];
  }
  mgbound(C, level); /* the halo refresh mgrelax runs after a sweep (mgsolver.for:610-611) */
  exchangepp(C, level);
  for (int ib = 0; ib < nb; ++ib) {
    Blk &B = C.b[ib];
    Lev L = lev(C, B, level);
    for (int k = 1; k <= L.nk; ++k) for (int j = 1; j <= L.nj; ++j) for (int i = 1; i <= L.ni; ++i)
      fi[ib][((size_t)(k - 1) * L.nj + (j - 1)) * L.ni + (i - 1)] = B.cof[PH(L, i, j, k)];
  }
  return MF3D_OK;
}

/* Apply the level-1 operator A (the residual form of mgrestr,
 * mgsolver.for:702-709, with rhs = 0, negated) to phi given ghost-inclusive
 * i fastest; ghosts are taken as given.  out = sum a_nb phi_nb + ap phi. */
int orc_apply_operator(const mf3d_block_desc *blocks, int nb, int ngrid, int level, double *const *phi, double *const *out) {
  mf3d_params prm;
  std::memset(&prm, 0, sizeof prm);
  prm.ngrid = ngrid; prm.mg_itrsch = 3; prm.irestr = 1; prm.iproln = 1; prm.maxcy = 1; prm.pl = 1; prm.differencing = 1;
  Ctx C;
  int st = setup(C, blocks, nb, &prm);
  if (st) return st;
  for (int ib = 0; ib < nb; ++ib) {
    Blk &B = C.b[ib];
    Lev L = lev(C, B, level);
    long nij2 = (long)(L.ni - 2) * (L.nj - 2), incr = nij2 * (L.nk - 2);
    auto G = [&](double *a, int i, int j, int k) -> double & { return a[((size_t)(k - 1) * L.nj + (j - 1)) * L.ni + (i - 1)]; };
    for (int k = 2; k <= L.nk - 1; ++k) for (int i = 2; i <= L.ni - 1; ++i) for (int j = 2; j <= L.nj - 1; ++j) {
      long w = B.faz[level] + (long)(k - 2) * nij2 + (long)(i - 2) * (L.nj - 2) + (j - 1);
      const double *c = B.cof.data();
      G(out[ib], i, j, k) = (c[w] * G(phi[ib], i - 1, j, k) + c[w + incr] * G(phi[ib], i + 1, j, k) +
                             c[w + 2 * incr] * G(phi[ib], i, j - 1, k) + c[w + 3 * incr] * G(phi[ib], i, j + 1, k) +
                             c[w + 4 * incr] * G(phi[ib], i, j, k - 1) + c[w + 5 * incr] * G(phi[ib], i, j, k + 1) +
                             c[w + 6 * incr] * G(phi[ib], i, j, k));
    }
  }
  return MF3D_OK;
}

/* Neighbour search restated from alloc_dom.for:456-1150 (tolerance 1e-8),
 * over block extents; xst..zen = the bounding box (the domain extents). */
int orc_build_topology(int nb, const double *ext, const int *bc6, double dx, double dy, double dz, mf3d_block_desc *out) {
  double xst = 1e300, xen = -1e300, yst = 1e300, yen = -1e300, zst = 1e300, zen = -1e300;
  for (int i = 0; i < nb; ++i) {
    xst = std::min(xst, ext[6 * i]); xen = std::max(xen, ext[6 * i + 1]);
    yst = std::min(yst, ext[6 * i + 2]); yen = std::max(yen, ext[6 * i + 3]);
    zst = std::min(zst, ext[6 * i + 4]); zen = std::max(zen, ext[6 * i + 5]);
  }
  auto X = [&](int i, int c) { return ext[6 * i + c]; };
  auto eq = [](double a, double b) { return std::fabs(a - b) < 1e-8; };
  for (int b = 0; b < nb; ++b) {
    mf3d_block_desc &d = out[b];
    std::memset(&d, 0, sizeof d);
    d.id = b; d.dx = dx; d.dy = dy; d.dz = dz;
    d.xsl = X(b, 0); d.xel = X(b, 1); d.ysl = X(b, 2); d.yel = X(b, 3); d.zsl = X(b, 4); d.zel = X(b, 5);
    d.nx = (int)std::lround((d.xel - d.xsl) / dx);
    d.ny = (int)std::lround((d.yel - d.ysl) / dy);
    d.nz = (int)std::lround((d.zel - d.zsl) / dz);
    d.bc_west = bc6[0]; d.bc_east = bc6[1]; d.bc_south = bc6[2]; d.bc_north = bc6[3]; d.bc_bottom = bc6[4]; d.bc_top = bc6[5];
    int say;
    auto find = [&](auto pred) { int r = -1; say = 0; for (int i = 0; i < nb; ++i) if (i != b && pred(i)) { r = i; ++say; } return r; };
    d.iprev = find([&](int i) { return eq(d.xsl, X(i, 1)) && eq(d.ysl, X(i, 2)) && eq(d.yel, X(i, 3)) && eq(d.zsl, X(i, 4)) && eq(d.zel, X(i, 5)); });
    if (say > 1) { g_err = "more than one previous neighbour in x"; return MF3D_E_INVALID; }
    d.inext = find([&](int i) { return eq(d.xel, X(i, 0)) && eq(d.ysl, X(i, 2)) && eq(d.yel, X(i, 3)) && eq(d.zsl, X(i, 4)) && eq(d.zel, X(i, 5)); });
    if (say > 1) { g_err = "more than one next neighbour in x"; return MF3D_E_INVALID; }
    d.jprev = find([&](int i) { return eq(d.ysl, X(i, 3)) && eq(d.xsl, X(i, 0)) && eq(d.xel, X(i, 1)) && eq(d.zsl, X(i, 4)) && eq(d.zel, X(i, 5)); });
    if (say > 1) { g_err = "more than one previous neighbour in y"; return MF3D_E_INVALID; }
    d.jnext = find([&](int i) { return eq(d.yel, X(i, 2)) && eq(d.xsl, X(i, 0)) && eq(d.xel, X(i, 1)) && eq(d.zsl, X(i, 4)) && eq(d.zel, X(i, 5)); });
    if (say > 1) { g_err = "more than one next neighbour in y"; return MF3D_E_INVALID; }
    d.kprev = find([&](int i) { return eq(d.zsl, X(i, 5)) && eq(d.xsl, X(i, 0)) && eq(d.xel, X(i, 1)) && eq(d.ysl, X(i, 2)) && eq(d.yel, X(i, 3)); });
    if (say > 1) { g_err = "more than one previous neighbour in z"; return MF3D_E_INVALID; }
    d.knext = find([&](int i) { return eq(d.zel, X(i, 4)) && eq(d.xsl, X(i, 0)) && eq(d.xel, X(i, 1)) && eq(d.ysl, X(i, 2)) && eq(d.yel, X(i, 3)); });
    if (say > 1) { g_err = "more than one next neighbour in z"; return MF3D_E_INVALID; }
    /* corners (alloc_dom.for:632-750) */
    d.corprev[0] = find([&](int i) { return eq(d.xsl, X(i, 1)) && eq(d.ysl, X(i, 3)) && eq(d.zsl, X(i, 5)); });
    d.corprev[1] = find([&](int i) { return eq(d.xsl, X(i, 1)) && eq(d.yel, X(i, 2)) && eq(d.zsl, X(i, 5)); });
    d.corprev[2] = find([&](int i) { return eq(d.xel, X(i, 0)) && eq(d.yel, X(i, 2)) && eq(d.zsl, X(i, 5)); });
    d.corprev[3] = find([&](int i) { return eq(d.xel, X(i, 0)) && eq(d.ysl, X(i, 3)) && eq(d.zsl, X(i, 5)); });
    d.cornext[0] = find([&](int i) { return eq(d.xel, X(i, 0)) && eq(d.yel, X(i, 2)) && eq(d.zel, X(i, 4)); });
    d.cornext[1] = find([&](int i) { return eq(d.xel, X(i, 0)) && eq(d.ysl, X(i, 3)) && eq(d.zel, X(i, 4)); });
    d.cornext[2] = find([&](int i) { return eq(d.xsl, X(i, 1)) && eq(d.ysl, X(i, 3)) && eq(d.zel, X(i, 4)); });
    d.cornext[3] = find([&](int i) { return eq(d.xsl, X(i, 1)) && eq(d.yel, X(i, 2)) && eq(d.zel, X(i, 4)); });
    /* edges (alloc_dom.for:752-968) */
    auto ysame = [&](int i) { return eq(d.ysl, X(i, 2)) && eq(d.yel, X(i, 3)); };
    auto xsame = [&](int i) { return eq(d.xsl, X(i, 0)) && eq(d.xel, X(i, 1)); };
    auto zsame = [&](int i) { return eq(d.zsl, X(i, 4)) && eq(d.zel, X(i, 5)); };
    d.edgprev[0] = find([&](int i) { return eq(d.xsl, X(i, 1)) && eq(d.zsl, X(i, 5)) && ysame(i); });
    d.edgprev[1] = find([&](int i) { return eq(d.yel, X(i, 2)) && eq(d.zsl, X(i, 5)) && xsame(i); });
    d.edgprev[2] = find([&](int i) { return eq(d.xel, X(i, 0)) && eq(d.zsl, X(i, 5)) && ysame(i); });
    d.edgprev[3] = find([&](int i) { return eq(d.ysl, X(i, 3)) && eq(d.zsl, X(i, 5)) && xsame(i); });
    d.edgprev[4] = find([&](int i) { return eq(d.xsl, X(i, 1)) && eq(d.ysl, X(i, 3)) && zsame(i); });
    d.edgprev[5] = find([&](int i) { return eq(d.xsl, X(i, 1)) && eq(d.yel, X(i, 2)) && zsame(i); });
    d.edgnext[0] = find([&](int i) { return eq(d.xel, X(i, 0)) && eq(d.zel, X(i, 4)) && ysame(i); });
    d.edgnext[1] = find([&](int i) { return eq(d.ysl, X(i, 3)) && eq(d.zel, X(i, 4)) && xsame(i); });
    d.edgnext[2] = find([&](int i) { return eq(d.xsl, X(i, 1)) && eq(d.zel, X(i, 4)) && ysame(i); });
    d.edgnext[3] = find([&](int i) { return eq(d.yel, X(i, 2)) && eq(d.zel, X(i, 4)) && xsame(i); });
    d.edgnext[4] = find([&](int i) { return eq(d.xel, X(i, 0)) && eq(d.yel, X(i, 2)) && zsame(i); });
    d.edgnext[5] = find([&](int i) { return eq(d.xel, X(i, 0)) && eq(d.ysl, X(i, 3)) && zsame(i); });
    /* periodic partners (alloc_dom.for:971-1150) */
    d.per_ip = d.per_in = d.per_jp = d.per_jn = d.per_kp = d.per_kn = -1;
    if (d.bc_west == 5 && d.iprev < 0) d.per_ip = find([&](int i) { return eq(xen, X(i, 1)) && ysame(i) && zsame(i); });
    if (d.bc_east == 5 && d.inext < 0) d.per_in = find([&](int i) { return eq(xst, X(i, 0)) && ysame(i) && zsame(i); });
    if (d.bc_south == 5 && d.jprev < 0) d.per_jp = find([&](int i) { return eq(yen, X(i, 3)) && xsame(i) && zsame(i); });
    if (d.bc_north == 5 && d.jnext < 0) d.per_jn = find([&](int i) { return eq(yst, X(i, 2)) && xsame(i) && zsame(i); });
    if (d.bc_bottom == 5 && d.kprev < 0) d.per_kp = find([&](int i) { return eq(zen, X(i, 5)) && xsame(i) && ysame(i); });
    if (d.bc_top == 5 && d.knext < 0) d.per_kn = find([&](int i) { return eq(zst, X(i, 4)) && xsame(i) && ysame(i); });
  }
  return MF3D_OK;
}

} /* extern "C" */
