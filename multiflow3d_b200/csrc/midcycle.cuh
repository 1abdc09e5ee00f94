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

constexpr int MID_MAX_LIST = 64;  // listed blocks a phase keeps in shared memory (more: read from the table)

template <typename T>
__global__ void __launch_bounds__(MID_THREADS, 1) k_mid_cycle(const MidPhase *__restrict__ phases, int nph,
                                                               const int *__restrict__ act, MidBar *bar,
                                                               int *__restrict__ err) {
  pdl_wait();
  if (*(volatile const int *)err) return;  // an earlier wait gave up: the call is failing already
  // the phase's listed blocks: fine (and coarse) descriptors, item prefix
  __shared__ BlkLev sf[MID_MAX_LIST], sc[MID_MAX_LIST];
  __shared__ long long spre[MID_MAX_LIST + 1];
  const unsigned stride = gridDim.x * blockDim.x;
  const unsigned t0 = blockIdx.x * blockDim.x + threadIdx.x;
  for (int p = 0; p < nph; ++p) {
    const MidPhase P = phases[p];
    const bool listed = P.kind == MID_SWEEP || P.kind == MID_RESTRICT || P.kind == MID_PROLONG;
    const bool cached = listed && P.nlist <= MID_MAX_LIST;
    if (cached) {
      for (int i = threadIdx.x; i < P.nlist; i += blockDim.x) {
        sf[i] = P.tab[P.list[i]];
        if (P.kind != MID_SWEEP) sc[i] = P.tab2[P.list[i]];
      }
      for (int i = threadIdx.x; i <= P.nlist; i += blockDim.x) spre[i] = P.pre[i];
      __syncthreads();
    }
    auto find = [&](unsigned t) -> int {
      const long long *pre = cached ? spre : P.pre;
      int lo = 0, hi = P.nlist - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= (long long)t) lo = mid;
        else hi = mid - 1;
      }
      return lo;
    };
    if (P.kind == MID_SWEEP) {
      for (unsigned t = t0; t < (unsigned long long)P.items; t += stride) {
        const int li = find(t);
        const BlkLev B = cached ? sf[li] : P.tab[P.list[li]];
        if (!act[B.dom]) continue;
        const unsigned Q = (unsigned)((B.nx + 1) / 2);
        const unsigned r0 = t - (unsigned)(cached ? spre[li] : P.pre[li]);
        const unsigned r = FastDiv(Q).div(r0), kk = FastDiv((unsigned)B.ny).div(r);
        const int q = (int)(r0 - r * Q), j = (int)(r - kk * (unsigned)B.ny) + 1, k = (int)kk + 1;
        const Coef<T> cf(B);
        if (P.fz) sweep_cell<T, true>(B, cf, phi_of<T>(B), rhs_of<T>(B), P.colour, q, j, k);
        else sweep_cell<T, false>(B, cf, phi_of<T>(B), rhs_of<T>(B), P.colour, q, j, k);
      }
    } else if (P.kind == MID_HALO_STAGE) {
      T *buf = (T *)P.buf;
      for (unsigned t = t0; t < (unsigned long long)P.nstaged; t += stride) {
        const HaloSeg &S = P.seg[halo_segment<true>(P.seg, P.nseg, t)];
        if (!act[S.dom]) continue;
        const HaloCopy c = S.pairs[t - S.sstart];
        buf[t] = phi_of<T>(P.tab[S.blk_base + c.sblk])[c.soff];
      }
    } else if (P.kind == MID_HALO_APPLY) {
      const T *buf = (const T *)P.buf;
      for (unsigned t = t0; t < (unsigned long long)P.items; t += stride) {
        const HaloSeg &S = P.seg[halo_segment<false>(P.seg, P.nseg, t)];
        if (!act[S.dom]) continue;
        const long long u = t - S.start;
        const HaloCopy c = S.pairs[u];
        const T v = u < S.nstaged ? buf[S.sstart + u] : phi_of<T>(P.tab[S.blk_base + c.sblk])[c.soff];
        phi_of<T>(P.tab[S.blk_base + c.dblk])[c.doff] = v;
      }
    } else {  // MID_RESTRICT, MID_PROLONG
      const int add = P.kind == MID_RESTRICT ? 2 : 1;  // coarse ghost-inclusive cells / fine groups
      for (unsigned t = t0; t < (unsigned long long)P.items; t += stride) {
        const int li = find(t);
        const BlkLev Fb = cached ? sf[li] : P.tab[P.list[li]];
        const BlkLev Cb = cached ? sc[li] : P.tab2[P.list[li]];
        if (!act[Cb.dom]) continue;
        const unsigned GX = (unsigned)(Cb.nx + add), GY = (unsigned)(Cb.ny + add);
        const unsigned r0 = t - (unsigned)(cached ? spre[li] : P.pre[li]);
        const unsigned r = FastDiv(GX).div(r0), K = FastDiv(GY).div(r);
        const int I = (int)(r0 - r * GX), J = (int)(r - K * GY);
        if (P.kind == MID_RESTRICT)
          restrict_cell<T, T>(Fb, Coef<T>(Fb), phi_of<T>(Fb), rhs_of<T>(Fb), Cb, Coef<T>(Cb), phi_of<T>(Cb),
                              rhs_of<T>(Cb), I, J, (int)K);
        else
          prolong_group<T, T>(Fb, phi_of<T>(Fb), Cb, phi_of<T>(Cb), I, J, (int)K);
      }
    }
    if (p + 1 < nph && !mid_barrier(bar, err)) return;  // (its __syncthreads also frees sf, sc, spre)
  }
}

}  // namespace mf3d
