// The coarse end of the red-black V-cycle in one launch: levels g0..L of a
// domain of at most 8 blocks, one CTA per block, the domain's CTAs one
// thread-block cluster.  Each CTA holds its block's phi and rhs of those
// levels in shared memory (the level arrays' own colour-split layout); the
// halo refresh after every sweep reads the neighbouring blocks' cells
// through distributed shared memory.  Cluster barriers separate the phases.
//
// It replaces, operation for operation and with the same arithmetic in the
// same order, what the separate launches do for these levels
// (mgsolver.for:224-369): on each level going down, ir sweeps (the first
// red half-sweep was formed by the restriction into the level), the halo
// after each sweep (mgbound + exchangepp + exchbc_mgpp as the domain's copy
// map), and the restriction into the next level (mgrestr, with the next
// level's from-zero red half-sweep); on the coarsest level ip more sweeps;
// going up, the prolongation (mgcorr + mgbound) and ip sweeps.  So the
// values are bit-identical to the launch-per-phase path.  The few hundred
// cells of these levels made that path launch-bound (about 5 us per launch
// for 40 launches per V-cycle).
#pragma once

#include <cooperative_groups.h>

#include "kernels.cuh"

namespace mf3d {

constexpr int CC_THREADS = 512;
constexpr int CC_MAX_LEVELS = 8;    // levels held by one launch at most
constexpr int CC_MAX_BLOCKS = 8;    // blocks of a domain (portable cluster size)

// A block's halo pairs at one level (destination in this block).
struct CcHalo {
  const HaloCopy *pairs;
  int n;
};

// t / d for t * d < 2^32 without a division: ceil(2^32 / d) by a high
// multiply (exact in that range: the rounding of the reciprocal adds less
// than 1/d to t/d).
struct FastDiv {
  unsigned d, m;
  FastDiv() = default;
  __device__ explicit FastDiv(unsigned d_) : d(d_), m(d_ > 1 ? 0xffffffffu / d_ + 1u : 0u) {}
  __device__ __forceinline__ unsigned div(unsigned t) const { return d > 1 ? __umulhi(t, m) : t; }
};

// Kernel arguments.
struct CcArgs {
  const BlkLev *tab[CC_MAX_LEVELS];   // per held level (g0 + l): the view's level table (global arrays)
  const CcHalo *halo;                 // [l * nb + b]
  int blk0;                           // view index of the domain's first block (cluster rank 0)
  int nb, nlev, g0, lc;               // blocks, levels held, first level, first FP64 level (coarse64)
  int ir, ip;                         // pre-/post-smoothing sweeps
  int dom;                            // the domain (act)
  int bufn;                           // halo staging slots per CTA
  long long coef_off;                 // shared-memory byte offset of the levels' coefficient and
                                      // restriction-ratio arrays (cc_coef_bytes each, level order)
};

// shared-memory bytes of one level's 1-D coefficients (six arrays) and
// restriction ratios (three) in element size elem, 16-byte aligned
__host__ __device__ inline long long cc_coef_bytes(const BlkLev &B, int elem) {
  return ((long long)(3 * (B.nx + B.ny + B.nz + 6)) * elem + 15) / 16 * 16;
}

// shared-memory layout of one block's held levels: phi (2*cstr) then rhs
// (2*cstr) per level, each 16-byte aligned; returns the bytes
__host__ __device__ inline long long cc_level_bytes(const BlkLev &B, int elem) {
  return ((long long)2 * B.cstr * elem + 15) / 16 * 16;
}

// One item of a red-black half-sweep: the cell of colour `colour` in
// compact column q of row j, plane k (none where i = 2q+2-s passes nx);
// FROM_ZERO: every neighbour reads as 0 (the first red half-sweep after
// mgrestr zeroed the level).  The arithmetic of k_rbgs / k_rbgs_small.
template <typename T, bool FROM_ZERO>
__device__ __forceinline__ void sweep_cell(const BlkLev &B, const Coef<T> &cf, T *phi, const T *rhs, int colour, int q,
                                           int j, int k) {
  const int s = (colour + j + k + 1) & 1;
  const int i = 2 * q + 2 - s;
  if (i > B.nx) return;
  const long long rs = (long long)(B.ny + 2) * B.hp;
  const T *O = phi + (1 - colour) * B.cstr;
  T *M = phi + colour * B.cstr;
  const T *R = rhs + colour * B.cstr;
  const long long base = (long long)k * rs + (long long)j * B.hp;
  const int h = q + 1 - s;
  T w = (T)0, e = (T)0, so = (T)0, no = (T)0, bo = (T)0, to = (T)0;
  if (!FROM_ZERO) {
    w = O[base + q]; e = O[base + q + 1]; so = O[base - B.hp + h]; no = O[base + B.hp + h];
    bo = O[base - rs + h]; to = O[base + rs + h];
  }
  T aw, ae, as, an, ab, at;
  cell_coefs(B, cf, i, j, k, aw, ae, as, an, ab, at);
  const T ap = (T)-1.0 * (aw + ae + as + an + ab + at);
  M[base + h] = ((R[base + h] - (aw * w + ae * e + as * so + an * no + ab * bo + at * to)) / ap);
}

template <typename T>
__device__ __forceinline__ void cc_sweep(const BlkLev &B, T *phi, const T *rhs, int colour) {
  const int Q = (B.nx + 1) / 2;
  const int items = Q * B.ny * B.nz;
  const Coef<T> cf(B);
  const FastDiv fq((unsigned)Q), fy((unsigned)B.ny);
  for (int t = threadIdx.x; t < items; t += blockDim.x) {
    const int r = (int)fq.div((unsigned)t);
    const int q = t - r * Q;
    const int kk = (int)fy.div((unsigned)r);
    sweep_cell<T, false>(B, cf, phi, rhs, colour, q, r - kk * B.ny + 1, kk + 1);
  }
  __syncthreads();
}

// mgrestr from the fine level (Fb, P, R) into the coarse one (Cb, PC, RC):
// coarse phi := 0 on every cell, the interior coarse rhs from the 8
// children's residuals, and the coarse from-zero red half-sweep - k_restrict.
// One coarse cell (I, J, K) of mgrestr, ghost-inclusive indices: phi := 0;
// an interior cell also takes the rhs from its 8 children's residuals and,
// red, the level's from-zero red half-sweep - k_restrict_tma's arithmetic.
template <typename TF, typename TC>
__device__ __forceinline__ void restrict_cell(const BlkLev &Fb, const Coef<TF> &cf, const TF *P, const TF *R,
                                              const BlkLev &Cb, const Coef<TC> &cc, TC *PC, TC *RC, int I, int J,
                                              int K) {
  const TF *rx = (const TF *)Fb.geo, *ry = rx + (Fb.nx + 2), *rz = ry + (Fb.ny + 2);
  const long long cs = Fb.cstr, rowf = Fb.hp, plf = (long long)(Fb.ny + 2) * Fb.hp;
  auto fo = [&](int i, int j, int k) -> long long {
    return ((i + j + k + 1) & 1) * cs + k * plf + j * rowf + (i >> 1);
  };
  const long long co = cell_off(Cb, I, J, K);
  PC[co] = (TC)0;
  if (I < 1 || I > Cb.nx || J < 1 || J > Cb.ny || K < 1 || K > Cb.nz) return;
  TF sum = (TF)0;
#pragma unroll
  for (int dk = 0; dk < 2; ++dk) {
    const int fk = 2 * K - 1 + dk;
    const TF ab = cf.ab[fk], at = cf.at[fk], sz = rz[fk];
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int di = 0; di < 2; ++di) {
        const int fi = 2 * I - 1 + di, fj = 2 * J - 1 + dj;
        const TF cw = cf.aw[fi], ce = cf.ae[fi], cs_ = cf.as[fj], cn = cf.an[fj];
        const TF ap = (TF)-1.0 * (cw + ce + cs_ + cn + ab + at);
        const TF pw = P[fo(fi - 1, fj, fk)], pe = P[fo(fi + 1, fj, fk)];
        const TF ps = P[fo(fi, fj - 1, fk)], pn = P[fo(fi, fj + 1, fk)];
        const TF pb = P[fo(fi, fj, fk - 1)], pt = P[fo(fi, fj, fk + 1)];
        const TF pp = P[fo(fi, fj, fk)];
        const TF r = R[fo(fi, fj, fk)];
        const TF res = r - (cw * pw + ce * pe + cs_ * ps + cn * pn + ab * pb + at * pt + ap * pp);
        const TF s = (TF)8.0 * rx[fi] * ry[fj] * sz;
        const TF a = res * s;
        sum = (dk | dj | di) ? sum + a : a;
      }
  }
  const TF v = (TF)0.125 * sum;
  RC[co] = (TC)v;
  if (colour_of(I, J, K) == 0) {
    TC aw, ae, as, an, ab, at;
    cell_coefs(Cb, cc, I, J, K, aw, ae, as, an, ab, at);
    const TC ap = (TC)-1.0 * (aw + ae + as + an + ab + at);
    PC[co] = ((TC)v / ap);
  }
}

// mgrestr from the fine level (Fb, P, R) into the coarse one (Cb, PC, RC):
// coarse phi := 0 on every cell, the interior coarse rhs from the 8
// children's residuals, and the coarse from-zero red half-sweep - k_restrict.
template <typename TF, typename TC>
__device__ __forceinline__ void cc_restrict(const BlkLev &Fb, const TF *P, const TF *R, const BlkLev &Cb, TC *PC,
                                            TC *RC) {
  const int GX = Cb.nx + 2, GY = Cb.ny + 2, GZ = Cb.nz + 2;
  const Coef<TF> cf(Fb);
  const Coef<TC> cc(Cb);
  const FastDiv fx((unsigned)GX), fy((unsigned)GY);
  for (int t = threadIdx.x; t < GX * GY * GZ; t += blockDim.x) {
    const int r = (int)fx.div((unsigned)t), K = (int)fy.div((unsigned)r);
    restrict_cell<TF, TC>(Fb, cf, P, R, Cb, cc, PC, RC, t - r * GX, r - K * GY, K);
  }
  __syncthreads();
}

// mgcorr + mgbound from the coarse level (Cb, PC) onto the fine one (Fb, PF):
// one 2x2x2 fine group per thread - k_prolong.
// One fine group (2I..2I+1) x (2J..2J+1) x (2K..2K+1) of mgcorr + mgbound,
// from the coarse cells (I..I+1, J..J+1, K..K+1) - k_prolong's arithmetic.
template <typename TF, typename TC>
__device__ __forceinline__ void prolong_group(const BlkLev &Fb, TF *PF, const BlkLev &Cb, const TC *PC, int I, int J,
                                              int K) {
  const int m = Fb.nmask;
  const long long csf = Fb.cstr, rowf = Fb.hp, plf = (long long)(Fb.ny + 2) * Fb.hp;
  const bool xw = I == 0 && (m & 1), xe = I == Cb.nx && (m & 2);
  const bool ys = J == 0 && (m & 4), yn = J == Cb.ny && (m & 8);
  const bool zb = K == 0 && (m & 16), zt = K == Cb.nz && (m & 32);
  TF lo[2][2], hi[2][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      lo[a][b] = (TF)PC[cell_off(Cb, I + a, J + b, K)];
      hi[a][b] = (TF)PC[cell_off(Cb, I + a, J + b, K + 1)];
    }
  TF v[2][2][2];
#pragma unroll
  for (int dk = 0; dk < 2; ++dk)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int di = 0; di < 2; ++di) {
        auto w = [&](int a, int b, int c) -> TF {
          return (TF)((a == di ? 3 : 1) * (b == dj ? 3 : 1) * (c == dk ? 3 : 1));
        };
        const TF corr = (w(0, 0, 0) * lo[0][0] + w(0, 1, 0) * lo[0][1] + w(0, 0, 1) * hi[0][0] +
                         w(0, 1, 1) * hi[0][1] + w(1, 0, 0) * lo[1][0] + w(1, 1, 0) * lo[1][1] +
                         w(1, 0, 1) * hi[1][0] + w(1, 1, 1) * hi[1][1]) *
                        (TF)0.015625;
        const long long o = ((di + dj + dk + 1) & 1) * csf + (2 * K + dk) * plf + (2 * J + dj) * rowf + I;
        v[dk][dj][di] = PF[o] + corr;
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
        const TF a0 = si ? v[0][0][1] : v[0][0][0], a1 = si ? v[0][1][1] : v[0][1][0];
        const TF a2 = si ? v[1][0][1] : v[1][0][0], a3 = si ? v[1][1][1] : v[1][1][0];
        const TF b0 = sj ? a1 : a0, b1 = sj ? a3 : a2;
        PF[o] = sk ? b1 : b0;
      }
}

// mgcorr + mgbound from the coarse level (Cb, PC) onto the fine one (Fb, PF):
// one 2x2x2 fine group per thread - k_prolong.
template <typename TF, typename TC>
__device__ __forceinline__ void cc_prolong(const BlkLev &Fb, TF *PF, const BlkLev &Cb, const TC *PC) {
  const int GX = Cb.nx + 1, GY = Cb.ny + 1, GZ = Cb.nz + 1;
  const FastDiv fx((unsigned)GX), fy((unsigned)GY);
  for (int t = threadIdx.x; t < GX * GY * GZ; t += blockDim.x) {
    const int r = (int)fx.div((unsigned)t), K = (int)fy.div((unsigned)r);
    prolong_group<TF, TC>(Fb, PF, Cb, PC, t - r * GX, r - K * GY, K);
  }
  __syncthreads();
}

template <typename TF>
__global__ void __launch_bounds__(CC_THREADS, 1) k_coarse_cycle(const CcArgs a, const int *__restrict__ act) {
  pdl_wait();
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char cc_smem[];
  __shared__ long long off[CC_MAX_BLOCKS][CC_MAX_LEVELS];  // byte offset of each rank's level arrays
  __shared__ BlkLev sdesc[CC_MAX_LEVELS];  // this block's levels, coefficients in shared memory
  if (!act[a.dom]) return;  // the whole cluster is one domain: uniform
  const int b = (int)cluster.block_rank();
  if (threadIdx.x < a.nlev) sdesc[threadIdx.x] = a.tab[threadIdx.x][a.blk0 + b];
  if (threadIdx.x < a.nb) {
    long long o = 0;
    for (int l = 0; l < a.nlev; ++l) {
      const BlkLev &B = a.tab[l][a.blk0 + threadIdx.x];
      const int elem = a.g0 + l >= a.lc ? 8 : (int)sizeof(TF);
      off[threadIdx.x][l] = o;
      o += 2 * cc_level_bytes(B, elem);
    }
  }
  __syncthreads();
  long long total = 0;
  for (int l = 0; l < a.nlev; ++l) {
    const int elem = a.g0 + l >= a.lc ? 8 : (int)sizeof(TF);
    total += 2 * cc_level_bytes(a.tab[l][a.blk0 + b], elem);
  }
  double *buf = (double *)(cc_smem + (total + 15) / 16 * 16);  // halo staging: values as double
  // the 1-D coefficients and restriction ratios of every held level, read
  // at each cell of every sweep, restriction and residual: into shared memory
  {
    unsigned char *cp = cc_smem + a.coef_off;
    for (int l = 0; l < a.nlev; ++l) {
      const BlkLev B = sdesc[l];
      const int elem = a.g0 + l >= a.lc ? 8 : (int)sizeof(TF);
      const int nco = 2 * (B.nx + B.ny + B.nz + 6), ngeo = B.nx + B.ny + B.nz + 6;
      for (int e = threadIdx.x; e < nco + ngeo; e += blockDim.x) {
        const unsigned char *src = e < nco ? (const unsigned char *)B.coef + (long long)e * elem
                                           : (const unsigned char *)B.geo + (long long)(e - nco) * elem;
        if (elem == 8) ((double *)cp)[e] = *(const double *)src;
        else ((float *)cp)[e] = *(const float *)src;
      }
      __syncthreads();  // every thread has read sdesc[l] before it changes
      if (threadIdx.x == 0) {
        sdesc[l].coef = cp;
        sdesc[l].geo = cp + (long long)nco * elem;
      }
      cp += cc_coef_bytes(B, elem);
    }
    __syncthreads();
  }
  auto desc = [&](int l) -> BlkLev { return sdesc[l]; };
  auto phi_at = [&](int r, int l) -> unsigned char * { return cc_smem + off[r][l]; };
  auto rhs_at = [&](int l) -> unsigned char * {
    const int elem = a.g0 + l >= a.lc ? 8 : (int)sizeof(TF);
    return cc_smem + off[b][l] + cc_level_bytes(desc(l), elem);
  };
  // level g0 from global memory (rhs and phi, ghost shell included)
  {
    const BlkLev B = desc(0);
    const int elem = a.g0 >= a.lc ? 8 : (int)sizeof(TF);
    const long long n16 = cc_level_bytes(B, elem) / 16, used = 2 * B.cstr * elem;
    const int4 *gp = (const int4 *)B.phi, *gr = (const int4 *)B.rhs;
    int4 *sp = (int4 *)phi_at(b, 0), *sr = (int4 *)rhs_at(0);
    for (long long t = threadIdx.x; t < n16; t += blockDim.x) {
      if (t * 16 + 16 <= used) {
        sp[t] = gp[t];
        sr[t] = gr[t];
      }
    }
    // a partial last 16-byte word (odd element counts)
    for (long long e = (used / 16) * 16 / elem + threadIdx.x; e < 2 * B.cstr; e += blockDim.x) {
      if (elem == 8) {
        ((double *)phi_at(b, 0))[e] = ((const double *)B.phi)[e];
        ((double *)rhs_at(0))[e] = ((const double *)B.rhs)[e];
      } else {
        ((float *)phi_at(b, 0))[e] = ((const float *)B.phi)[e];
        ((float *)rhs_at(0))[e] = ((const float *)B.rhs)[e];
      }
    }
  }
  __syncthreads();
  // the halo refresh of level l: every source read (through DSMEM) before
  // any destination is written
  auto halo = [&](int l) {
    const CcHalo H = a.halo[l * a.nb + b];
    const bool f64 = a.g0 + l >= a.lc || sizeof(TF) == 8;
    cluster.sync();  // every block's sweep is complete
    for (int t = threadIdx.x; t < H.n; t += blockDim.x) {
      const HaloCopy c = H.pairs[t];
      unsigned char *src = (unsigned char *)cluster.map_shared_rank((void *)phi_at(c.sblk, l), c.sblk);
      buf[t] = f64 ? ((const double *)src)[c.soff] : (double)((const float *)src)[c.soff];
    }
    cluster.sync();  // every source is read
    for (int t = threadIdx.x; t < H.n; t += blockDim.x) {
      const HaloCopy c = H.pairs[t];
      if (f64) ((double *)phi_at(b, l))[c.doff] = buf[t];
      else ((float *)phi_at(b, l))[c.doff] = (float)buf[t];
    }
    __syncthreads();
  };
  auto sweep = [&](int l, int colour) {
    const BlkLev B = desc(l);
    if (a.g0 + l >= a.lc) cc_sweep<double>(B, (double *)phi_at(b, l), (const double *)rhs_at(l), colour);
    else cc_sweep<TF>(B, (TF *)phi_at(b, l), (const TF *)rhs_at(l), colour);
  };
  const int top = a.nlev - 1;
  // down: each level's first red half-sweep was formed by the restriction into it
  for (int l = 0; l <= top; ++l) {
    for (int itr = 0; itr < a.ir; ++itr) {
      if (itr > 0) sweep(l, 0);
      sweep(l, 1);
      halo(l);
    }
    if (l == top) {
      for (int itr = 0; itr < a.ip; ++itr) {
        sweep(l, 0);
        sweep(l, 1);
        halo(l);
      }
      break;
    }
    const BlkLev Fb = desc(l), Cb = desc(l + 1);
    const bool f64 = a.g0 + l >= a.lc, c64 = a.g0 + l + 1 >= a.lc;
    if (f64) cc_restrict<double, double>(Fb, (const double *)phi_at(b, l), (const double *)rhs_at(l), Cb,
                                         (double *)phi_at(b, l + 1), (double *)rhs_at(l + 1));
    else if (c64) cc_restrict<TF, double>(Fb, (const TF *)phi_at(b, l), (const TF *)rhs_at(l), Cb,
                                          (double *)phi_at(b, l + 1), (double *)rhs_at(l + 1));
    else cc_restrict<TF, TF>(Fb, (const TF *)phi_at(b, l), (const TF *)rhs_at(l), Cb, (TF *)phi_at(b, l + 1),
                             (TF *)rhs_at(l + 1));
  }
  // up
  for (int l = top - 1; l >= 0; --l) {
    const BlkLev Fb = desc(l), Cb = desc(l + 1);
    const bool f64 = a.g0 + l >= a.lc, c64 = a.g0 + l + 1 >= a.lc;
    if (f64) cc_prolong<double, double>(Fb, (double *)phi_at(b, l), Cb, (const double *)phi_at(b, l + 1));
    else if (c64) cc_prolong<TF, double>(Fb, (TF *)phi_at(b, l), Cb, (const double *)phi_at(b, l + 1));
    else cc_prolong<TF, TF>(Fb, (TF *)phi_at(b, l), Cb, (const TF *)phi_at(b, l + 1));
    for (int itr = 0; itr < a.ip; ++itr) {
      sweep(l, 0);
      sweep(l, 1);
      halo(l);
    }
  }
  // level g0's phi back to global memory (the prolongation into g0-1 reads it)
  {
    const BlkLev B = desc(0);
    const int elem = a.g0 >= a.lc ? 8 : (int)sizeof(TF);
    const long long n = 2 * B.cstr;
    if (elem == 8)
      for (long long e = threadIdx.x; e < n; e += blockDim.x) ((double *)B.phi)[e] = ((const double *)phi_at(b, 0))[e];
    else
      for (long long e = threadIdx.x; e < n; e += blockDim.x) ((float *)B.phi)[e] = ((const float *)phi_at(b, 0))[e];
  }
  cluster.sync();  // no block leaves while another may still read its shared memory
}

}  // namespace mf3d
