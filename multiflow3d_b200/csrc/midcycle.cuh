// The middle levels of the red-black V-cycle in one cooperative launch per
// direction: levels 2 .. (the first level of the coarse cluster launch, or
// the coarsest) have arrays that sit in L2 and a few million cells at most,
// so as separate launches each half-sweep, halo pass, restriction and
// prolongation cost a launch's latency and pipeline fill more than its
// work.  Here one persistent grid (one CTA per SM, all resident: a
// cooperative launch) walks a list of phases built on the host in exactly
// the order vcycle launches them - pre-smoothing sweeps with the halo after
// each (mgrelax, mgsolver.for:371-617), the restriction into the next level
// with its from-zero red half-sweep (mgrestr, :619-761), and on the way up
// the prolongation (mgcorr + mgbound, :763-905) and post-smoothing - with a
// grid barrier between phases.  Each phase's items are the cells, pairs or
// groups of one launch of the launch path, computed by the same per-item
// code (sweep_cell, restrict_cell, prolong_group, the halo copy), so the
// values are bit-identical to it.
#pragma once

#include "coarse.cuh"

namespace mf3d {

enum MidKind : int { MID_SWEEP = 0, MID_HALO_STAGE = 1, MID_HALO_APPLY = 2, MID_RESTRICT = 3, MID_PROLONG = 4 };

// One phase.  SWEEP: blocks list[0..nlist) of level table `tab`, item
// prefix pre (ceil(nx/2)*ny*nz per block).  RESTRICT / PROLONG: fine table
// `tab`, coarse table `tab2`, blocks list[], prefix pre over the coarse
// ghost-inclusive cells (restriction) or fine groups (prolongation).  HALO:
// the level's segments, staged slots and buffer.
struct MidPhase {
  int kind, colour, fz, nlist;
  long long items;
  const BlkLev *tab, *tab2;
  const int *list;
  const long long *pre;
  const HaloSeg *seg;
  int nseg, pad;
  long long nstaged;
  void *buf;
};

// Grid barrier state (zero-initialised; reusable across launches).
struct MidBar {
  unsigned count, gen;
};

constexpr int MID_THREADS = 512;
constexpr long long kMidSpinLimit = 1LL << 26;  // polls before a barrier gives up (a few seconds)

// All CTAs of the (co-resident) grid.  A CTA that waits past the poll limit
// records ERR_MID_BARRIER and leaves with the others' work unsynchronised:
// the call's results are then invalid and the host reports the error.
__device__ __forceinline__ bool mid_barrier(MidBar *bar, int *err) {
  __syncthreads();
  __shared__ int ok_s;
  if (threadIdx.x == 0) {
    ok_s = 1;
    __threadfence();
    const unsigned gen = *(volatile unsigned *)&bar->gen;
    if (atomicAdd(&bar->count, 1u) == gridDim.x - 1) {
      *(volatile unsigned *)&bar->count = 0u;
      __threadfence();
      atomicAdd(&bar->gen, 1u);
    } else {
      long long spins = 0;
      while (*(volatile unsigned *)&bar->gen == gen) {
        if (++spins > kMidSpinLimit) {
          atomicExch(err, ERR_MID_BARRIER);
          ok_s = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok_s != 0;
}

// The block of a flat item index: last list entry whose prefix <= t.
__device__ __forceinline__ int mid_block(const long long *pre, int n, long long t) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <typename T>
__global__ void __launch_bounds__(MID_THREADS, 1) k_mid_cycle(const MidPhase *__restrict__ phases, int nph,
                                                               const int *__restrict__ act, MidBar *bar,
                                                               int *__restrict__ err) {
  pdl_wait();
  if (*(volatile const int *)err) return;  // an earlier wait gave up: the call is failing already
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (int p = 0; p < nph; ++p) {
    const MidPhase P = phases[p];
    if (P.kind == MID_SWEEP) {
      for (long long t = t0; t < P.items; t += stride) {
        const int li = mid_block(P.pre, P.nlist, t);
        const BlkLev B = P.tab[P.list[li]];
        if (!act[B.dom]) continue;
        const int Q = (B.nx + 1) / 2;
        long long r = t - P.pre[li];
        const int q = (int)(r % Q);
        r /= Q;
        const int j = (int)(r % B.ny) + 1, k = (int)(r / B.ny) + 1;
        const Coef<T> cf(B);
        if (P.fz) sweep_cell<T, true>(B, cf, phi_of<T>(B), rhs_of<T>(B), P.colour, q, j, k);
        else sweep_cell<T, false>(B, cf, phi_of<T>(B), rhs_of<T>(B), P.colour, q, j, k);
      }
    } else if (P.kind == MID_HALO_STAGE) {
      T *buf = (T *)P.buf;
      for (long long t = t0; t < P.nstaged; t += stride) {
        const HaloSeg &S = P.seg[halo_segment<true>(P.seg, P.nseg, t)];
        if (!act[S.dom]) continue;
        const HaloCopy c = S.pairs[t - S.sstart];
        buf[t] = phi_of<T>(P.tab[S.blk_base + c.sblk])[c.soff];
      }
    } else if (P.kind == MID_HALO_APPLY) {
      const T *buf = (const T *)P.buf;
      for (long long t = t0; t < P.items; t += stride) {
        const HaloSeg &S = P.seg[halo_segment<false>(P.seg, P.nseg, t)];
        if (!act[S.dom]) continue;
        const long long u = t - S.start;
        const HaloCopy c = S.pairs[u];
        const T v = u < S.nstaged ? buf[S.sstart + u] : phi_of<T>(P.tab[S.blk_base + c.sblk])[c.soff];
        phi_of<T>(P.tab[S.blk_base + c.dblk])[c.doff] = v;
      }
    } else if (P.kind == MID_RESTRICT) {
      for (long long t = t0; t < P.items; t += stride) {
        const int li = mid_block(P.pre, P.nlist, t);
        const int b = P.list[li];
        const BlkLev Fb = P.tab[b], Cb = P.tab2[b];
        if (!act[Cb.dom]) continue;
        const int GX = Cb.nx + 2, GY = Cb.ny + 2;
        const long long r = t - P.pre[li];
        const int I = (int)(r % GX), J = (int)((r / GX) % GY), K = (int)(r / ((long long)GX * GY));
        restrict_cell<T, T>(Fb, Coef<T>(Fb), phi_of<T>(Fb), rhs_of<T>(Fb), Cb, Coef<T>(Cb), phi_of<T>(Cb),
                            rhs_of<T>(Cb), I, J, K);
      }
    } else {  // MID_PROLONG
      for (long long t = t0; t < P.items; t += stride) {
        const int li = mid_block(P.pre, P.nlist, t);
        const int b = P.list[li];
        const BlkLev Fb = P.tab[b], Cb = P.tab2[b];
        if (!act[Fb.dom]) continue;
        const int GX = Cb.nx + 1, GY = Cb.ny + 1;
        const long long r = t - P.pre[li];
        const int I = (int)(r % GX), J = (int)((r / GX) % GY), K = (int)(r / ((long long)GX * GY));
        prolong_group<T, T>(Fb, phi_of<T>(Fb), Cb, phi_of<T>(Cb), I, J, K);
      }
    }
    if (p + 1 < nph && !mid_barrier(bar, err)) return;
  }
}

}  // namespace mf3d
