// LMR: the V-cycle across 2:1 refinement interfaces.
//
// A block of refinement rdiv keeps ngrid_input + log2(rdiv) levels of its
// own (localparameters.for:42-45); below its last level it stays at that
// size (mgsolver.for:27-31, 388-392): the restriction into such a level is
// the residual itself (mgrestr, :714-727) and the correction back from it is
// added on every cell, ghosts included (mgcorr, :806-818), before mgbound.
// The halo refresh of a level where refinements meet is a program of
// weighted sums (build_halo_lmr): nodes evaluated in order of depth from the
// state before the exchange, then the ghost writes.
#pragma once

#include "kernels.cuh"

namespace mf3d {

struct LmrTerm {
  int blk, off;  // blk >= 0: phi cell (view block, colour-split offset); -1: node `off`; -2: the constant 0
  double w;
};
struct LmrNode {
  int t0, nt;  // terms [t0, t0 + nt)
  double scale;
};
struct LmrWrite {
  int blk, off, node;  // node < 0: a copy of (sblk, soff), a cell no write touches
  int sblk, soff;
};

constexpr int LMR_MAX_TERMS = 8;   // the longest formula: an 8-cell average or blend
constexpr int LMR_SMEM_BLOCKS = 64; // view blocks whose phi pointers a CTA keeps in shared memory

// The phi pointer of view block b: from shared memory for the first
// LMR_SMEM_BLOCKS blocks (one dependent load fewer per term), else the table.
template <typename T>
__device__ __forceinline__ T *lmr_phi(const BlkLev *__restrict__ tab, T *const *sphi, int b) {
  return b < LMR_SMEM_BLOCKS ? sphi[b] : phi_of<T>(tab[b]);
}
template <typename T>
__device__ __forceinline__ void lmr_stage_phi(const BlkLev *__restrict__ tab, int nblk, T **sphi) {
  for (int b = threadIdx.x; b < nblk && b < LMR_SMEM_BLOCKS; b += blockDim.x) sphi[b] = phi_of<T>(tab[b]);
  __syncthreads();
}

// Nodes [n0, n1): val[n] = (w_0 x_0 + w_1 x_1 + ...) * scale, summed left to
// right as the reference writes each formula.  The terms' operands load
// first, all in flight at once; the sum then runs in order.
template <typename T>
__global__ void __launch_bounds__(256) k_lmr_nodes(const BlkLev *__restrict__ tab, int nblk,
                                                   const LmrTerm *__restrict__ terms, const LmrNode *__restrict__ nodes,
                                                   int n0, int n1, double *__restrict__ val) {
  pdl_wait();
  __shared__ T *sphi[LMR_SMEM_BLOCKS];
  lmr_stage_phi<T>(tab, nblk, sphi);
  const int n = n0 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (n >= n1) return;
  const LmrNode N = nodes[n];
  double x[LMR_MAX_TERMS], w[LMR_MAX_TERMS];
#pragma unroll
  for (int q = 0; q < LMR_MAX_TERMS; ++q) {
    if (q < N.nt) {
      const LmrTerm a = terms[N.t0 + q];
      w[q] = a.w;
      x[q] = a.blk >= 0 ? (double)lmr_phi<T>(tab, sphi, a.blk)[a.off] : a.blk == -1 ? val[a.off] : 0.0;
    }
  }
  double t = w[0] * x[0];
#pragma unroll
  for (int q = 1; q < LMR_MAX_TERMS; ++q)
    if (q < N.nt) t = t + w[q] * x[q];
  val[n] = t * N.scale;
}

template <typename T>
__global__ void __launch_bounds__(256) k_lmr_write(const BlkLev *__restrict__ tab, int nblk,
                                                   const LmrWrite *__restrict__ w, int n,
                                                   const double *__restrict__ val) {
  pdl_wait();
  __shared__ T *sphi[LMR_SMEM_BLOCKS];
  lmr_stage_phi<T>(tab, nblk, sphi);
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= n) return;
  const LmrWrite W = w[i];
  lmr_phi<T>(tab, sphi, W.blk)[W.off] = W.node >= 0 ? (T)val[W.node] : lmr_phi<T>(tab, sphi, W.sblk)[W.soff];
}

// The listed blocks' ghost-inclusive cells, item t: block list[b] with
// pre[b] <= t < pre[b+1], cell (i, j, k) of its level of table `tab`.
__device__ __forceinline__ bool lmr_item(const BlkLev *tab, const int *list, const long long *pre, int nlist,
                                         long long t, int &blk, int &i, int &j, int &k) {
  if (t >= pre[nlist]) return false;
  int lo = 0, hi = nlist - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  blk = list[lo];
  const BlkLev &B = tab[blk];
  long long r = t - pre[lo];
  i = (int)(r % (B.nx + 2));
  r /= (B.nx + 2);
  j = (int)(r % (B.ny + 2));
  k = (int)(r / (B.ny + 2));
  return true;
}

// mgrestr into a level past the block's own last (same size): phi := 0 on
// every cell, the interior rhs := the fine level's residual at the same
// cell, and with `red` the level's from-zero red half-sweep.  TF / TC: the
// fine and coarse levels' types (an FP32 V-cycle keeps its coarsest level
// in FP64); the residual is formed in TF as the regular restriction forms
// it, the red half-sweep in TC.
template <typename TF, typename TC>
__global__ void __launch_bounds__(256) k_lmr_inject(const BlkLev *__restrict__ ftab, const BlkLev *__restrict__ ctab,
                                                    const int *__restrict__ list, const long long *__restrict__ pre,
                                                    int nlist, const int *__restrict__ act, int red) {
  pdl_wait();
  int b, i, j, k;
  if (!lmr_item(ctab, list, pre, nlist, (long long)blockIdx.x * blockDim.x + threadIdx.x, b, i, j, k)) return;
  const BlkLev Cb = ctab[b], Fb = ftab[b];
  if (!act[Cb.dom]) return;
  TC *PC = phi_of<TC>(Cb), *RC = rhs_of<TC>(Cb);
  const TF *P = phi_of<TF>(Fb), *R = rhs_of<TF>(Fb);
  const long long co = cell_off(Cb, i, j, k);
  PC[co] = (TC)0;
  if (i < 1 || i > Cb.nx || j < 1 || j > Cb.ny || k < 1 || k > Cb.nz) return;
  TF cw, ce, cs, cn, cb, ct;
  cell_coefs(Fb, Coef<TF>(Fb), i, j, k, cw, ce, cs, cn, cb, ct);
  const TF ap = (TF)-1.0 * (cw + ce + cs + cn + cb + ct);
  const TF res = R[cell_off(Fb, i, j, k)] -
                 (cw * P[cell_off(Fb, i - 1, j, k)] + ce * P[cell_off(Fb, i + 1, j, k)] +
                  cs * P[cell_off(Fb, i, j - 1, k)] + cn * P[cell_off(Fb, i, j + 1, k)] +
                  cb * P[cell_off(Fb, i, j, k - 1)] + ct * P[cell_off(Fb, i, j, k + 1)] + ap * P[cell_off(Fb, i, j, k)]);
  RC[co] = (TC)res;
  if (red && colour_of(i, j, k) == 0) {
    TC aw, ae, as, an, ab, at;
    cell_coefs(Cb, Coef<TC>(Cb), i, j, k, aw, ae, as, an, ab, at);
    const TC apc = (TC)-1.0 * (aw + ae + as + an + ab + at);
    PC[co] = (TC)res / apc;
  }
}

// mgcorr from a level past the block's own last onto a level of the same
// size.  mode 0: phi_f += phi_c on every cell; mode 1 (after it): mgbound,
// each wall-face ghost taking the cell it mirrors - west, east, south,
// north, bottom, top in turn, so a ghost on two or three walls ends with the
// interior cell diagonal to it.
template <typename TF, typename TC>
__global__ void __launch_bounds__(256) k_lmr_add(const BlkLev *__restrict__ ftab, const BlkLev *__restrict__ ctab,
                                                 const int *__restrict__ list, const long long *__restrict__ pre,
                                                 int nlist, const int *__restrict__ act, int mode) {
  pdl_wait();
  int b, i, j, k;
  if (!lmr_item(ftab, list, pre, nlist, (long long)blockIdx.x * blockDim.x + threadIdx.x, b, i, j, k)) return;
  const BlkLev Fb = ftab[b], Cb = ctab[b];
  if (!act[Fb.dom]) return;
  TF *PF = phi_of<TF>(Fb);
  if (mode == 0) {
    const long long o = cell_off(Fb, i, j, k);
    PF[o] = PF[o] + (TF)phi_of<TC>(Cb)[cell_off(Cb, i, j, k)];
    return;
  }
  const int m = Fb.nmask;
  const int si = (i == 0 && (m & 1)) ? 1 : (i == Fb.nx + 1 && (m & 2)) ? Fb.nx : i;
  const int sj = (j == 0 && (m & 4)) ? 1 : (j == Fb.ny + 1 && (m & 8)) ? Fb.ny : j;
  const int sk = (k == 0 && (m & 16)) ? 1 : (k == Fb.nz + 1 && (m & 32)) ? Fb.nz : k;
  if (si == i && sj == j && sk == k) return;
  PF[cell_off(Fb, i, j, k)] = PF[cell_off(Fb, si, sj, sk)];
}

}  // namespace mf3d
