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
constexpr long long kMidSpinLimit = 1LL << 25;  // polls before a barrier gives up (a few seconds)

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
      while (*(volatile unsigned *)&bar->gen == gen) {  // an L2 round trip per poll
        if (++spins > kMidSpinLimit) {
          atomicExch(err, ERR_MID_BARRIER);
          ok_s = 0;
          break;
        }
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

constexpr int MID_MAX_LIST = 64;   // listed blocks of a phase (the plan keeps to it)
constexpr int MID_CTAS_PER_SM = 1;

template <typename T>
__global__ void __launch_bounds__(MID_THREADS, MID_CTAS_PER_SM) k_mid_cycle(const MidPhase *__restrict__ phases,
                                                                             int nph, const int *__restrict__ act,
                                                                             MidBar *bar, int *__restrict__ err) {
  pdl_wait();
  if (*(volatile const int *)err) return;  // an earlier wait gave up: the call is failing already
  // the phase's listed blocks: fine (and coarse) descriptors, item prefix,
  // the divisors that split a block's item index
  __shared__ BlkLev sf[MID_MAX_LIST], sc[MID_MAX_LIST];
  __shared__ unsigned spre[MID_MAX_LIST + 1];
  __shared__ FastDiv sd1[MID_MAX_LIST], sd2[MID_MAX_LIST];
  __shared__ unsigned sn1[MID_MAX_LIST], sn2[MID_MAX_LIST];
  for (int p = 0; p < nph; ++p) {
    const MidPhase P = phases[p];
    const bool listed = P.kind == MID_SWEEP || P.kind == MID_RESTRICT || P.kind == MID_PROLONG;
    const unsigned items = (unsigned)(P.kind == MID_HALO_STAGE ? P.nstaged : P.items);
    if (listed) {
      for (int i = threadIdx.x; i < P.nlist; i += blockDim.x) {
        const BlkLev F = P.tab[P.list[i]];
        sf[i] = F;
        unsigned d1, d2;
        if (P.kind == MID_SWEEP) {
          d1 = (unsigned)((F.nx + 1) / 2);
          d2 = (unsigned)F.ny;
        } else {
          const BlkLev Cb = P.tab2[P.list[i]];
          sc[i] = Cb;
          const int add = P.kind == MID_RESTRICT ? 2 : 1;  // coarse ghost-inclusive cells / fine groups
          d1 = (unsigned)(Cb.nx + add);
          d2 = (unsigned)(Cb.ny + add);
        }
        sd1[i] = FastDiv(d1);
        sd2[i] = FastDiv(d2);
        sn1[i] = d1;
        sn2[i] = d2;
      }
      for (int i = threadIdx.x; i <= P.nlist; i += blockDim.x) spre[i] = (unsigned)P.pre[i];
      __syncthreads();
    }
    // each CTA a contiguous chunk of the phase's items, its threads striding
    // through it: a thread's block changes at most a few times per phase
    const unsigned chunk = (items + gridDim.x - 1) / gridDim.x;
    const unsigned c0 = blockIdx.x * chunk, c1 = min(items, c0 + chunk);
    int li = 0;
    if (listed && c0 < c1) {
      int lo = 0, hi = P.nlist - 1;  // last listed block whose first item <= c0
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (spre[mid] <= c0) lo = mid;
        else hi = mid - 1;
      }
      li = lo;
    }
    for (unsigned t = c0 + threadIdx.x; t < c1; t += blockDim.x) {
      if (listed)
        while (t >= spre[li + 1]) ++li;
      if (P.kind == MID_SWEEP) {
        const BlkLev &B = sf[li];
        if (!act[B.dom]) continue;
        const unsigned r0 = t - spre[li];
        const unsigned r = sd1[li].div(r0), kk = sd2[li].div(r);
        const int q = (int)(r0 - r * sn1[li]), j = (int)(r - kk * sn2[li]) + 1, k = (int)kk + 1;
        const Coef<T> cf(B);
        if (P.fz) sweep_cell<T, true>(B, cf, phi_of<T>(B), rhs_of<T>(B), P.colour, q, j, k);
        else sweep_cell<T, false>(B, cf, phi_of<T>(B), rhs_of<T>(B), P.colour, q, j, k);
      } else if (P.kind == MID_HALO_STAGE) {
        const HaloSeg &S = P.seg[halo_segment<true>(P.seg, P.nseg, t)];
        if (!act[S.dom]) continue;
        const HaloCopy c = S.pairs[t - S.sstart];
        ((T *)P.buf)[t] = phi_of<T>(P.tab[S.blk_base + c.sblk])[c.soff];
      } else if (P.kind == MID_HALO_APPLY) {
        const HaloSeg &S = P.seg[halo_segment<false>(P.seg, P.nseg, t)];
        if (!act[S.dom]) continue;
        const long long u = t - S.start;
        const HaloCopy c = S.pairs[u];
        const T v = u < S.nstaged ? ((const T *)P.buf)[S.sstart + u] : phi_of<T>(P.tab[S.blk_base + c.sblk])[c.soff];
        phi_of<T>(P.tab[S.blk_base + c.dblk])[c.doff] = v;
      } else {  // MID_RESTRICT, MID_PROLONG
        const BlkLev &Fb = sf[li], &Cb = sc[li];
        if (!act[Cb.dom]) continue;
        const unsigned r0 = t - spre[li];
        const unsigned r = sd1[li].div(r0), K = sd2[li].div(r);
        const int I = (int)(r0 - r * sn1[li]), J = (int)(r - K * sn2[li]);
        if (P.kind == MID_RESTRICT)
          restrict_cell<T, T>(Fb, Coef<T>(Fb), phi_of<T>(Fb), rhs_of<T>(Fb), Cb, Coef<T>(Cb), phi_of<T>(Cb),
                              rhs_of<T>(Cb), I, J, (int)K);
        else
          prolong_group<T, T>(Fb, phi_of<T>(Fb), Cb, phi_of<T>(Cb), I, J, (int)K);
      }
    }
    if (p + 1 < nph && !mid_barrier(bar, err)) return;  // (its __syncthreads also frees the shared tables)
  }
}

}  // namespace mf3d
