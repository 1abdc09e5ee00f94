/*
 * mf3d.h - C ABI of the B200 pressure-Poisson multigrid library.
 *
 * The library replaces MultiFlow3D's projection step: `newsolv_mg`
 * (newsolv_mg.for:2-102) with the V-cycle it drives (`coeff`, `mgkcyc`,
 * `mgrelax`, `mgrestr`, `mgcorr`, `mgbound` in mgsolver.for:2-992), the
 * multigrid halo copies (`exchangepp`, `exchbc_mgpp` in exchangepp.for), and
 * the FP64 projection kernels `calvel`, `calmas`, `pbound` (press.for:2-200)
 * with the field halos `exchange(1..4)` (exchange.for, exchange_bc.for).
 *
 * All blocks of one solve live on one GPU.  Plain pointers and sizes only:
 * no CUDA or torch types cross this boundary.  Every function returns an
 * `int` status (enum mf3d_status); the library never exits the process
 * (the reference `stop`s at newsolv_mg.for:82 and localparameters.for:205).
 *
 * Array layout of the field arguments (`mf3d_fields`): Fortran column-major
 * `(ttc_i, ttc_j, ttc_k)`, i fastest, with `pl` ghost layers on each side,
 * ttc_i = nx + 2*pl (localparameters.for:138-140).  Cell (i,j,k) of the
 * reference (1-based) is element (i-1) + ttc_i*((j-1) + ttc_j*(k-1)).
 * The staggered velocity u(i,j,k) sits on the east face of cell (i,j,k).
 */
#ifndef MF3D_H
#define MF3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MF3D_ABI_VERSION 1

/* Status codes.  Non-negative = the solve ran; negative = it did not. */
enum mf3d_status {
  MF3D_OK = 0,
  MF3D_NOT_CONVERGED = 1, /* maxcy exhausted (newsolv_mg.for:59-60 prints) */
  MF3D_DIVERGED = 2,      /* rmax > 100 (newsolv_mg.for:64-83 stops)      */
  MF3D_PENDING = 3,       /* server: the request has not finished yet       */
  MF3D_E_INVALID = -1,    /* bad config (localparameters.for:84-98,201-206)*/
  MF3D_E_CUDA = -2,       /* a CUDA runtime call failed                     */
  MF3D_E_OOM = -3,        /* device allocation failed or over the cap       */
  MF3D_E_TIMEOUT = -4,    /* a bounded device wait gave up                  */
  MF3D_E_NONFINITE = -5,  /* NaN/Inf met in the residual                     */
  MF3D_E_UNSUPPORTED = -6 /* a reference feature outside this build (LMR
                             in the outer loop) or an unsupported
                             combination                                   */
};

/* Boundary-condition code meaning "periodic" (control.cin:17-22). Any other
 * code on a face with no neighbour block is a homogeneous Neumann face for
 * the pressure (mgbound, mgsolver.for:931-986; pbound, press.for:90-133). */
#define MF3D_BC_PERIODIC 5

/* Precision of the multigrid V-cycle.  The outer defect-correction loop
 * (calvel / calmas / p += pp) is always FP64. */
enum mf3d_precision {
  MF3D_PREC_FP64 = 0, /* the reference's arithmetic, bit-exact              */
  MF3D_PREC_FP32 = 1, /* FP32 smoother/transfer, FP32 correction storage    */
  MF3D_PREC_BF16 = 2  /* FP32 arithmetic, BF16 storage of the correction    */
};

/* One block (reference `type multidom`, module_multidata.for:15-122): the
 * fields the projection path reads.  Neighbour ids are block ids (dom_id),
 * -1 = none, exactly as alloc_dom.for:456-1150 sets them. */
typedef struct mf3d_block_desc {
  int id;                  /* dom_id, 0-based, unique                       */
  int nx, ny, nz;          /* interior cells: iep-isp+1, jep-jsp+1, kep-ksp+1 */
  double dx, dy, dz;       /* uniform spacing (localparameters.for:245-247) */
  double xsl, xel, ysl, yel, zsl, zel; /* block extents (infodom.cin)       */
  int iprev, inext, jprev, jnext, kprev, knext;   /* face neighbours      */
  int corprev[4], cornext[4];                     /* corner neighbours    */
  int edgprev[6], edgnext[6];                     /* edge neighbours      */
  int per_ip, per_in, per_jp, per_jn, per_kp, per_kn; /* periodic partners */
  int bc_west, bc_east, bc_south, bc_north, bc_bottom, bc_top;
  /* Optional non-uniform cell widths (length nx / ny / nz).  NULL = uniform
   * spacing dx/dy/dz.  This is an extension with no reference counterpart:
   * the reference grid is uniform per block (localparameters.for:245-247). */
  const double *hx, *hy, *hz;
} mf3d_block_desc;

/* Solver parameters: the control.cin fields the projection path reads
 * (initial.for:21-26). */
typedef struct mf3d_params {
  int ngrid;        /* multigrid levels ngrd_gl (control.cin:10)             */
  int mg_itrsch;    /* smoother: 1 lexicographic GS, 2 line TDMA, 3 RB GS    */
  int irestr;       /* pre-smoothing sweeps ("restriction iter")             */
  int iproln;       /* post-smoothing sweeps ("prolongation iter")           */
  int maxcy;        /* maximum outer iterations per solve                    */
  double eps;       /* stopping tolerance on rmax (newsolv_mg.for:56)        */
  int eps_relative; /* 0: rmax < eps (reference); 1: rmax < eps * rmax_0     */
  int pl;           /* ghost layers of the field arrays (localparameters.for:17-24) */
  int differencing; /* control.cin differencing: 1 (2nd-order CDS) or 3 (WENO,
                       which L_LSM requires, initial.for:133-135) - calmas
                       takes its 2nd-order divergence for both
                       (press.for:38-67); 2 (4th-order CDS): calmas' 4th-order
                       divergence (press.for:13-35), which reads u(i-2) and
                       u(i+1): needs pl >= 2, uniform spacing, no lsm          */
  int precision;    /* enum mf3d_precision                                   */
  int device;       /* CUDA device ordinal                                   */
  int pl_ex;        /* extra ghost planes (control.cin pl_ex; pl = LMR + pl_ex,
                       localparameters.for:17-24): the final exchange(1..3)
                       refreshes ghost layers 0..pl_ex of u, v, w
                       (exchange.for:16-20).  0 <= pl_ex < pl, and every block
                       edge must exceed pl_ex.                                */
  int lsm;          /* L_LSM (control.cin): variable density.  coeff runs at
                       every solve from mf3d_fields.dens (newsolv_mg.for:12-14,
                       mgsolver.for:69-182), calvel divides by the face
                       density (press.for:152-190) and the rhs is sup =
                       div(u)*dx*dy*dz/dt (press.for:51-53).  FP64 only,
                       uniform spacing, mf3d_create contexts only.            */
  int bounds;       /* 1: after the loop, boundu/boundv/boundw (newsolv_mg.for:
                       86-88, bounds.for:2-916) on the device: the periodic
                       exchange_bc of u, v, w, then every face without a
                       neighbour by its code - 1 inflow (west: u = ubulk,
                       v = w = 0; bottom: u = v = 0, w = 1.1), 2 outflow
                       (east, alfabc = 1: copy of the last face), 3 symmetry,
                       4 wall, 5 periodic, and the west inlets 7, 8 (file
                       values, mf3d_set_inlet), 12, 13 (1/7 power law); a
                       code with no branch for a face writes nothing there,
                       as in the reference; 21 on the east (convective
                       outflow, alfabc = 1) from the old velocities of
                       mf3d_bind_old_velocity; the wall functions 61 to 65
                       with the Re and fric of mf3d_set_wall_model.  The
                       codes that need data the library does not hold -
                       above 65 (no branch), 61 to 65 and 1 / 2 with lsm
                       (mu, dens, phi) - return MF3D_E_UNSUPPORTED.  Also
                       refreshes the
                       full periodic ghost planes of the final exchange(1..3).
                       Skipped when the solve diverged (the reference stops).
                       mf3d_create contexts only.  0: u, v, w face ghosts as
                       documented at mf3d_fields.                             */
  int solver;       /* control.cin solver: 2 (or 0) multigrid newsolv_mg; 1
                       pressure_1sweep with Stone's SIP (press.for:274-420,
                       sipsol.for:2-206), maxcy playing niter.  FP64,
                       mf3d_create contexts, no lsm.                          */
  int nswp;         /* solver 1: SIP sweeps per call (control.cin nswp(4))    */
  int alfabc;       /* control.cin alfabc: 1 = bounds applies the outflow
                       faces (code 2, bounds.for:136-170)                     */
  double ubulk;     /* control.cin ubulk: the inflow velocity of code-1 west
                       faces under bounds (bounds.for:42-53)                  */
} mf3d_params;

/* Field pointers of one block, each a (ttc_i,ttc_j,ttc_k) array.
 * ustar/vstar/wstar: in.  p: in/out (interior and every ghost that
 * p = p + pp, exchange(4) and pbound write).  u/v/w: in (faces on physical
 * walls, which calvel never writes) and out (all faces calvel writes, and
 * every ghost exchange(1..3) writes: in mf3d_create contexts its periodic
 * planes, face layers 0..pl_ex and the ghost edges and corners of its
 * corner and edge neighbours, exchange.for:343-2498; in batch and server
 * contexts the face layers 0..pl_ex over the interior tangential range
 * alone, other ghosts left as given).  For the host
 * entry point these are host pointers; for the `_device` one, device pointers.
 * `su` may be NULL; if set it receives the final RHS div(u)/dt (calmas;
 * sup under lsm).  `dens` (in, lsm only, else ignored): cell densities, ghost
 * layers included - calvel reads the first ghost layer. */
typedef struct mf3d_fields {
  double *ustar, *vstar, *wstar;
  double *u, *v, *w;
  double *p;
  double *su;
  double *dens;
} mf3d_fields;

typedef struct mf3d_ctx mf3d_ctx;

/* Result of one projection call. */
typedef struct mf3d_solve_info {
  double rmax;       /* final rmax (module vars `rmax`)                        */
  double rmax0;      /* rmax after the initial calvel/calmas                   */
  int iter;          /* outer iterations run (module vars `iter`)              */
  int status;        /* same as the return value                               */
  double ms_device;  /* device time of the solve in milliseconds               */
} mf3d_solve_info;

/* ---------------------------------------------------------------------- */
/* Set-up.                                                                  */
/* ---------------------------------------------------------------------- */

/* Neighbour search of alloc_dom.for:456-1150 (faces 465-628, corners
 * 632-750, edges 752-968, periodic partners 971-1150) over block extents.
 * `extents` holds 6 doubles per block (xsl,xel,ysl,yel,zsl,zel); `bc6` the
 * six global BC codes (W,E,S,N,B,T); dx,dy,dz the uniform spacing.  Fills
 * ids, nx/ny/nz, spacing and all neighbour fields of `out[nblocks]`. */
int mf3d_build_topology(int nblocks, const double *extents, const int *bc6,
                        double dx, double dy, double dz,
                        mf3d_block_desc *out);

/* Allocate device state for a solve over `nblocks` blocks: the multigrid
 * hierarchy (replaces `coeff`, mgsolver.for:2-222, and the `cof` storage of
 * localparameters.for:208-237), halo maps, field mirrors and streams.
 * Checks the divisibility rule of localparameters.for:200-206.
 *
 * LMR (2:1 refinement, localparameters.for:26-102): blocks whose spacings
 * differ by powers of two.  A block's rdiv is the coarsest block's dx over
 * its own; a refined block is given with rdiv times the cells over the
 * same extents.  params.ngrid is then ngrd_gl = ngrid_input + log2(max
 * rdiv); a block keeps ngrid_input + log2(rdiv) levels of its own size and
 * must be divisible by 2^(that - 1).  Neighbours may differ by 2:1 at most
 * and periodic partners not at all (alloc_dom.for:12-230).  FP64 or FP32
 * (the FP32 V-cycle keeps its coarsest level in FP64), uniform spacing, no
 * lsm, bounds or solver 1 (MF3D_E_UNSUPPORTED otherwise).  Such
 * a context runs mf3d_mgkcyc_device only: the outer loop's field exchanges
 * at refinement interfaces are not restated, and the other entry points
 * return MF3D_E_UNSUPPORTED. */
int mf3d_create(const mf3d_block_desc *blocks, int nblocks,
                const mf3d_params *params, mf3d_ctx **ctx);

int mf3d_destroy(mf3d_ctx *ctx);

/* ---------------------------------------------------------------------- */
/* The projection (newsolv_mg.for:2-102).                                  */
/* ---------------------------------------------------------------------- */

/* Host-array entry point: the drop-in for `newsolv_mg`.  `fields[nblocks]`
 * hold host pointers in the ttc layout; they are borrowed for the call.
 * Runs calvel/calmas, then up to maxcy x (V-cycle, p += pp, p halo, pbound,
 * calvel, calmas) until rmax < eps and iter > 1, then writes p, u, v, w
 * back.  The caller then runs exchange(1..3) and boundu/boundv/boundw as
 * newsolv_mg.for:86-88 does.  `rmax_hist` (may be NULL) receives rmax after
 * each outer iteration, at most `hist_cap` entries. */
int mf3d_newsolv_mg(mf3d_ctx *ctx, const mf3d_fields *fields, double dt,
                    double alfapr, mf3d_solve_info *info, double *rmax_hist,
                    int hist_cap);

/* Same, with `fields` pointing to device memory (a GPU-resident caller). */
int mf3d_newsolv_mg_device(mf3d_ctx *ctx, const mf3d_fields *fields,
                           double dt, double alfapr, mf3d_solve_info *info,
                           double *rmax_hist, int hist_cap);

/* ---------------------------------------------------------------------- */
/* The momentum predictor before the projection (upstream of newsolv_mg).   */
/* ---------------------------------------------------------------------- */

/* Per block, what one Runge-Kutta stage reads besides u, v, w (ttc layout):
 * the velocities at the start of the time step (flosol.for:98-104) and the
 * cell viscosity `vis` (molecular plus eddy; the predictor reads its ghost
 * layer 1 on the high faces). */
typedef struct mf3d_rk_fields {
  const double *uoo, *voo, *woo;
  const double *vis;
} mf3d_rk_fields;

/* One Runge-Kutta stage of the velocity predictor with explicit diffusion
 * (flosol.for:151-172 with diff_sch = 3), by the context's `differencing`:
 * 1 - rungek_conv2nd (rungek.for:314-412) then rungek_diff2nd
 * (rungek.for:584-779); 2 - rungek_conv4th (rungek.for:2-212) then
 * rungek_diff4th (rungek.for:214-312); 3 - rungek_convWENO (rungek.for:
 * 414-582, the HJ_WENO derivatives of weno.for) then rungek_diff2nd.  2 and 3
 * read three ghost layers (pl >= 3, else MF3D_E_INVALID; the reference sets
 * pl_ex = 2 for WENO, initial.for:114-117).  Each convection is boundu, the
 * u predictor, boundv, the v predictor, boundw, the w predictor; the
 * reference's branch without L_LSM, immersed boundaries or wall functions.
 * In: u, v, w (their ghosts
 * are refreshed by boundu/v/w, as in the reference), `rk`; out: ustar,
 * vstar, wstar over the faces calvel later reads (isu..ieu etc.).  `p` must
 * be set as for the projection (not read here; su and dens may be NULL).
 * `alfabc`: 1 on the first stage, 0 after (flosol.for:153-157) - the
 * context's own `alfabc` stays the projection's; `alfapr`: the stage's
 * alfark.  With the start-of-step velocities at hand, the stage's boundu/v/w
 * also restate the convective outflow (code 21, bounds.for:143-170), which
 * the projection's bounds mode refuses.  `pressureforce` adds dt*alfapr*forcn to ustar
 * (rungek.for:642-656).  Device pointers; contexts from mf3d_create with
 * `bounds = 1`, FP64, uniform spacing, no lsm (else MF3D_E_UNSUPPORTED).
 * Between stages the reference runs calvel (flosol.for:171;
 * mf3d_calvel_device), after the last one the projection
 * (mf3d_newsolv_mg_device). */
int mf3d_rungek_2nd_device(mf3d_ctx *ctx, const mf3d_fields *fields, const mf3d_rk_fields *rk,
                           double dt, double alfapr, int alfabc, int pressureforce, double forcn);

/* calvel alone (press.for:139-198, flosol.for:171 between Runge-Kutta
 * stages): u, v, w from ustar, vstar, wstar and p over the faces calvel
 * writes, then its exchange(1..3) (exchange.for:2-23: the periodic planes,
 * the face layers and the corner and edge ghosts of exchange_smlvl), from
 * the ghosts as they stand, without boundu/v/w.  Device pointers;
 * mf3d_create contexts, FP64, no lsm. */
int mf3d_calvel_device(mf3d_ctx *ctx, const mf3d_fields *fields, double dt, double alfapr);

/* The inlet file of a west face of code 7 or 8 (boundu, bounds.for:55-103),
 * for the boundu/v/w of the solve (bounds = 1) and of the velocity
 * predictor.  The reference opens the file itself at every boundu; here the
 * caller reads it and hands the values over, once per file (the library
 * keeps the plane until the next call).
 *   code 7: the values of Inlet/Inlet_<dom>_<n>.dat, one u per line, k
 *           outer, j inner over j = js-1..je+1, k = ks-1..ke+1:
 *           n = (ny+2)*(nz+2);
 *   code 8: the first column ("up") of inflow/Inlet_<dom>_<n>.dat after its
 *           two header lines, over j = js-1..je, k = ks-1..ke (the rows the
 *           reference reads, k outer): n = (ny+1)*(nz+1); u = up + ubulk, or
 *           up + the 1/7 power-law profile when uprof_sem = 12 (UPROF_SEM,
 *           initial.for:37).
 * Every ghost layer 0..pl_ex of u takes the plane; v and w are left as the
 * reference leaves them.  The power-law inlets (codes 12, 13,
 * bounds.for:105-135) need no call: the library forms them at create from
 * ubulk, the cell centres and the extents of all blocks.  Host values;
 * mf3d_create contexts with bounds = 1; a solve or predictor stage with a
 * code-7/8 face whose values were never set returns MF3D_E_INVALID. */
int mf3d_set_inlet(mf3d_ctx *ctx, int block_id, int code, int uprof_sem, const double *values, long long n);

/* The velocities at the start of the time step (uoo, voo, woo of `rk`, one
 * entry per block; vis is not read) for the convective outflow of the
 * solve's boundu/v/w: an east face of code 21 with alfabc = 1 sets
 *   u(ie+1+ly) = uoo(ie+1+ly) - dt*alfapr*(uoo(ie+1+ly) - uoo(ie))/dx
 * and the same for v and w (bounds.for:141-170, 449-474, 743-768), with the
 * solve's dt and alfapr.  The reference reaches that branch when the last
 * Runge-Kutta stage left alfabc = 1 (one stage, flosol.for:151-157).
 * Device pointers, borrowed until the next call; NULL unbinds.  A solve of
 * a bounds context with such a face and nothing bound returns
 * MF3D_E_INVALID.  mf3d_create contexts. */
int mf3d_bind_old_velocity(mf3d_ctx *ctx, const mf3d_rk_fields *rk);

/* Re and fric (control.cin) for the wall functions of boundu/v/w: codes 61
 * (smooth wall, log law), 62 (rough wall, log law with the roughness fric),
 * 63, 64, 65 (the Werner-Wengle 1/6, 1/7, 1/8 power laws) on faces without a
 * neighbour (bounds.for:187-206 and the matching branches; log_law.for,
 * wall_function.for).  At layer 0 a face's law gives the wall stress tau2
 * per face cell from the first cell layer's tangential speed; the
 * tangential component's first cell c takes c += sign(tau2*c/h, -c)*alfapr*dt
 * and its ghost -c; deeper layers mirror; the normal component is 0.  The
 * stresses stay in the context across calls (log_law keeps tau2 where y+ is
 * below 11.067) and this call clears them.  The laws take CUDA's sqrt, log
 * and pow, so the velocities they touch agree with the reference's libm to
 * rounding, not bit for bit.  A smooth-wall law that does not converge in
 * 10 steps (the reference stops) fails the call with MF3D_E_INVALID.  The
 * reference sets the power laws' constants with DATA statements inside the
 * CASE arms (wall_function.for:34-49); the library takes each arm's own
 * pair.  Needs uniform spacing and two or more cells along the face
 * normal; no lsm (the laws would read mu/dens). */
int mf3d_set_wall_model(mf3d_ctx *ctx, double re, double fric);

/* boundu, boundv, boundw alone (bounds.for:2-916) on device arrays u, v, w
 * of `fields` (the other pointers must be set as for a solve), with the
 * caller's dt, alfapr and alfabc: each component's periodic copy, then its
 * faces W, E, S, N, B, T per ghost layer 0..pl_ex, every code the bounds
 * mode of the solve handles.  mf3d_create contexts with bounds = 1, FP64. */
int mf3d_bounds_device(mf3d_ctx *ctx, const mf3d_fields *fields, double dt, double alfapr, int alfabc);

/* ---------------------------------------------------------------------- */
/* Batches of independent domains (no counterpart in the reference, which   */
/* solves one problem per call).                                            */
/* ---------------------------------------------------------------------- */

/* One independent single-block domain: its own size, spacing, boundary
 * conditions and multigrid depth. */
typedef struct mf3d_domain_desc {
  int nx, ny, nz;          /* interior cells                                    */
  double dx, dy, dz;       /* uniform spacing                                   */
  int bc[3];               /* per axis x, y, z: MF3D_BC_PERIODIC or a wall code */
  int ngrid;               /* levels; <= 0: the deepest mf3d_max_levels allows  */
  const double *hx, *hy, *hz; /* optional widths as in mf3d_block_desc         */
} mf3d_domain_desc;

/* Deepest level count for an nx x ny x nz block: every edge divisible by
 * 2^(L-1) and the coarsest edge at least 4 cells (minimum 1). */
int mf3d_max_levels(int nx, int ny, int nz);

/* A context over `ndomains` independent domains.  One launch per phase
 * covers every domain; each domain runs exactly its own V-cycles (its own
 * depth) and stops on its own convergence test, so its result is the same
 * alone or in the batch. */
int mf3d_batch_create(const mf3d_domain_desc *domains, int ndomains,
                      const mf3d_params *params, mf3d_ctx **ctx);

/* Solve every domain of a batch context: `fields[d]` (device arrays),
 * `dt[d]`, `alfapr[d]`; `infos[d]` and rows of `rmax_hist` (ndomains x
 * hist_cap, may be NULL) per domain.  Returns the worst status. */
int mf3d_batch_solve_device(mf3d_ctx *ctx, const mf3d_fields *fields,
                            const double *dt, const double *alfapr,
                            mf3d_solve_info *infos, double *rmax_hist,
                            int hist_cap);

/* One V-cycle (mgkcyc, mgsolver.for:224-369) on device arrays: reads the
 * RHS `su` and writes the correction `pp` of each block, both in the ttc
 * layout (pp including its first ghost layer, mgsolver.for:351-364). The
 * V-cycle starts from pp = 0 as newsolv_mg.for:19-21 and :44 leave it.
 * On an LMR context it runs the reference's LMR branches: levels past a
 * block's own keep its size (injection in mgrestr, whole-array addition in
 * mgcorr), and exchangepp's fine/coarse cases across refinement interfaces;
 * the entries of a refined block's face buffer that no coarse sender
 * writes (the reference leaves them to earlier exchanges) read as 0. */
int mf3d_mgkcyc_device(mf3d_ctx *ctx, double *const *su, double *const *pp);

/* mf3d_mgkcyc_device that allocates nothing: no cudaMalloc, no cudaFree,
 * no allocating library.  It runs the same V-cycle on the same context, but
 * the per-call tables of the su and pp pointers (which mf3d_mgkcyc_device
 * keeps in a buffer the context allocates on first use) live in a fixed
 * device array inside the library, sized for MF3D_NOALLOC_MAX_BLOCKS blocks
 * (2 x 512 pointers, 8 KiB).  All other device memory the call touches was
 * allocated by mf3d_create.  No counterpart in the reference (it has no GPU).
 *
 * For callers that must not allocate device memory while they run: a time
 * loop that shares the device with other streams (cudaMalloc/cudaFree may
 * synchronise the whole device), or a process whose device memory is held
 * by another allocator's pool.
 *
 * - More than MF3D_NOALLOC_MAX_BLOCKS blocks: MF3D_E_INVALID, nothing runs.
 * - Nothing has to start at zero: both tables are written in full before
 *   each use.  pp starts from 0 as in mf3d_mgkcyc_device.
 * - The array is shared by every context on a device: calls on one device
 *   must not overlap (from several threads, or on several contexts whose
 *   streams run concurrently); overlapping calls race on the tables.
 * - The set-up happens when the context is created: mf3d_create looks up
 *   the array's device address (cudaGetSymbolAddress) with the context's
 *   device current, keeps it in the context, and loads every kernel the
 *   V-cycle can launch, so that no call makes the driver load code on first
 *   use.  A context created after a device reset looks the address up anew. */
#define MF3D_NOALLOC_MAX_BLOCKS 512
int mf3d_mgkcyc_device_noalloc(mf3d_ctx *ctx, double *const *su, double *const *pp);

/* ---------------------------------------------------------------------- */
/* Introspection.                                                           */
/* ---------------------------------------------------------------------- */

/* Message of the last error on this thread ("" if none). */
const char *mf3d_last_error(void);
const char *mf3d_status_string(int status);
int mf3d_abi_version(void);

/* Number of device kernel launches issued by the last solve on `ctx`. */
long long mf3d_last_launch_count(const mf3d_ctx *ctx);

/* Kernel timing.  `kind` selects one kernel class whose every launch the
 * library then brackets with CUDA events on its own stream; 0 turns timing
 * off.  mf3d_profile_read returns, for the launches since the last
 * mf3d_profile call: total device milliseconds, launch count and the
 * algorithmic bytes those launches had to move (compulsory traffic). */
enum mf3d_profile_kind {
  MF3D_PROF_OFF = 0,
  MF3D_PROF_SMOOTH_L1 = 1,   /* red-black half-sweeps on the finest level */
  MF3D_PROF_CALMAS = 2,      /* fused calvel + calmas                      */
  MF3D_PROF_RESTRICT_L1 = 3, /* residual + restriction from the finest level */
  MF3D_PROF_PROLONG_L1 = 4   /* prolongation + correction onto the finest level */
};
int mf3d_profile(mf3d_ctx *ctx, int kind);
int mf3d_profile_read(mf3d_ctx *ctx, double *total_ms, long long *launches,
                      double *algorithmic_bytes);

/* Launch shapes the library chose for level `level` (1-based) of `ctx` -
 * by its autotuner (timed at mf3d_create / mf3d_batch_create, cached per
 * process by device, precision, smoother and block shapes; MF3D_AUTOTUNE=0
 * turns it off) or by default: the red-black sweep schedule (0..3), 1 when
 * the level sweeps with the plain-load kernel, the planes per CTA of the
 * TMA restriction into the level (-1: the plain-load restriction), and the
 * CTAs per block of the line or
 * lexicographic relaxation.  Any of the outputs may be NULL.  No
 * counterpart in the reference. */
int mf3d_tuning(const mf3d_ctx *ctx, int level, int *sweep_schedule, int *small_sweep, int *restrict_planes,
                int *cluster_ctas);

/* Host-only view of a field exchange: exchange(op) of exchange.for:2-23
 * (exchange_bc on the periodic faces, then exchange_smlvl with its corners,
 * edges and faces), followed by pbound for op 4 (press.for:77-137), as
 * (destination, source) cell pairs against the state before the exchange.
 * op 1, 2, 3: u, v, w with layers 0..pl_ex; op 4: p with one layer.  Cell
 * number = base(b) + (i-1) + ttc_i*((j-1) + ttc_j*(k-1)), 1-based field
 * indices, base(b) the sum of the ttc volumes of the blocks before b.  With
 * dst == NULL returns the pair count; -1 on bad arguments.  Needs no GPU. */
long long mf3d_field_exchange_map(const mf3d_block_desc *blocks, int nblocks, int pl, int pl_ex, int op,
                                  long long *dst, long long *src);

/* Testing aids for the failure paths (no counterpart in the reference, which
 * prints and stops).  Neither faults the device.
 * mf3d_test_fail_alloc: the device allocation `after` allocations from now
 * (0 = the next one) fails as if the device were out of memory, so the call
 * making it returns MF3D_E_OOM; -1 turns the injection off.  Process-wide.
 * mf3d_test_stall_copy: on `device`, the next red-black half-sweep declares
 * `bytes` (1..65536) more on one CTA's first copy barrier than its copies
 * deliver; that CTA's bounded wait gives up after 2 s and the call returns
 * MF3D_E_TIMEOUT.  The copies themselves complete; 0 clears it. */
int mf3d_test_fail_alloc(long long after);
int mf3d_test_stall_copy(int device, int bytes);

/* Host-only view of the multigrid halo refresh of level `level` (1-based)
 * that follows every smoothing sweep: the composition of mgbound,
 * exchangepp (with its trailing mgbound and exchbc_mgpp) - mgsolver.for:
 * 610-611, exchangepp.for:43-4763 - as (destination, source) cell pairs
 * against the state before the refresh.  Cell number = base(b) +
 * (k*(ny+2) + j)*(nx+2) + i, with 0-based ghost-inclusive local indices of
 * the level and base(b) the sum of the ghost-inclusive volumes of the
 * blocks before b (in argument order).  With dst == NULL returns the pair
 * count.  Needs no GPU. */
long long mf3d_halo_map(const mf3d_block_desc *blocks, int nblocks, int ngrid,
                        int level, long long *dst, long long *src);

/* Host-only: the same refresh applied to host arrays, for any layout - LMR
 * included, where a level on which refinements meet (rdv differing,
 * localparameters.for:47-57) takes the weighted sums of exchangepp's
 * fine/coarse branches instead of copies (exchangepp.for:43-4763).  fi[b]
 * holds block b's level-`level` array, ghost-inclusive, i fastest, of the
 * block's level size (an LMR block past its own last level keeps that
 * size).  Same arithmetic, in the same order, as the device's refresh; the
 * entries of a refined block's face buffer that no coarse sender writes
 * are taken as 0.  Needs no GPU.  Returns MF3D_OK or an error status. */
int mf3d_halo_refresh_host(const mf3d_block_desc *blocks, int nblocks, int ngrid,
                           int level, double *const *fi);

/* ---------------------------------------------------------------------- */
/* Serving (no counterpart in the reference): a request loop on one device */
/* that admits independent single-block solves as they arrive, keeps their  */
/* multigrid hierarchies resident, and advances every resident request by   */
/* one outer iteration per cycle in shared launches (continuous batching).  */
/* A request runs exactly its own solve: its result is the same alone and   */
/* in any mix.                                                              */
/* ---------------------------------------------------------------------- */
typedef struct mf3d_server mf3d_server;

/* Result and timeline of one request; times in seconds on the server's
 * steady clock (mf3d_server_clock). */
typedef struct mf3d_request_info {
  mf3d_solve_info info;
  double t_submit, t_admit, t_done;
} mf3d_request_info;

/* A server for `params` (precision, smoother, sweeps, tolerance, maxcy,
 * device; params->ngrid is ignored: each request brings its own depth).
 * Admission: requests enter in arrival order while the resident
 * hierarchies stay within `mem_cap_bytes` (and the device's free memory)
 * and at most `max_resident` requests are resident.  A worker thread owns
 * the device work; submit and poll are thread-safe.  In FP32 precision the
 * coarsest levels stay FP32 (resident mixes have mixed depths). */
int mf3d_server_create(const mf3d_params *params, double mem_cap_bytes, int max_resident, mf3d_server **out);

/* Queue one solve: `domain` as for mf3d_batch_create, `fields` device
 * arrays of one block (borrowed until the request completes: p, u, v, w
 * are written), dt, alfapr.  Returns a ticket.  The server's streams do not
 * order after the caller's: the fields' contents must be complete on the
 * device when this is called (synchronise the stream that produced them). */
int mf3d_server_submit(mf3d_server *srv, const mf3d_domain_desc *domain, const mf3d_fields *fields, double dt,
                       double alfapr, long long *ticket);

/* MF3D_PENDING while the request runs (waiting up to wait_ms for it), else
 * its final status with `info` filled; a finished ticket is then released. */
int mf3d_server_poll(mf3d_server *srv, long long ticket, mf3d_request_info *info, int wait_ms);

/* Counters since creation (any pointer may be NULL). */
int mf3d_server_stats(mf3d_server *srv, long long *submitted, long long *completed, long long *resident,
                      long long *queued, double *resident_bytes, long long *cycles);

/* Worker seconds spent (summed over the lanes) building hierarchies,
 * rebuilding the launch tables for a new mix, running cycles (launch to
 * completion check) and finishing requests; counts of builds and rebuilds. */
int mf3d_server_profile(mf3d_server *srv, double *build_s, double *rebuild_s, double *cycle_s, double *finish_s,
                        long long *builds, long long *rebuilds);

/* Seconds on the steady clock the server stamps requests with. */
double mf3d_server_clock(void);

/* Stops the worker after the cycle in flight; unfinished requests are
 * dropped (their fields are left as they are). */
int mf3d_server_destroy(mf3d_server *srv);

/* Self-test of the quotient the TMA calvel/calmas kernel forms on axes that
 * are not uniform powers of two: for n pairs (x[i], b[i]) in host memory,
 * q[i] = x[i]/b[i] from the reciprocal RN(1/b[i]) (Markstein's correction)
 * and qref[i] = the device's IEEE division, both computed on `device`.  The
 * two agree bit for bit.  No counterpart in the reference (a test hook of
 * this implementation). */
int mf3d_selftest_divide(const double *x, const double *b, long long n, double *q, double *qref, int device);

/* ---------------------------------------------------------------------- */
/* Restart files `tecbin<id>.bin` (the writer post.for:496-548 `tecbin`,   */
/* the reader initial.for:689-760), decoded and encoded on the device.     */
/* A file is gfortran unformatted sequential: each record framed by its    */
/* byte length as a 4-byte integer before and after; records (toti, totj,  */
/* totk), (pl), (inind, jnind, knind), then one record of 19 doubles per   */
/* ttc cell, i fastest: x(i), y(j), z(k), p, pm, ppm, vis, u, um, uum, v,  */
/* vm, vvm, w, wm, wwm, uvm, uwm, vwm.                                     */
/* ---------------------------------------------------------------------- */
typedef struct mf3d_tecbin_info {
  int toti, totj, totk;      /* ttc extents                                */
  int pl;                    /* ghost layers it was written with (the reader
                                stops when they differ, initial.for:714-719) */
  int inind, jnind, knind;   /* -1 where the block ends on a wall          */
  long long records;         /* toti*totj*totk                             */
  long long data_offset;     /* byte offset of the first cell record (52)  */
} mf3d_tecbin_info;

/* Checks the three header records of a file image (host memory, `nbytes`
 * long) and that its size is exactly the cell records they announce. */
int mf3d_tecbin_info_of(const void *image, size_t nbytes, mf3d_tecbin_info *info);

/* Bytes of the file image for these extents (-1 if an extent is < 1). */
long long mf3d_tecbin_size(int toti, int totj, int totk);

/* The reader: `image` is a whole file image in device memory; out[16] are
 * device arrays of info->records doubles receiving p, pm, ppm, vis, u, um,
 * uum, v, vm, vvm, w, wm, wwm, uvm, uwm, vwm (initial.for:718-733), a NULL
 * entry skipping its field.  Every cell record's framing is checked:
 * MF3D_E_INVALID names the first bad record.  Synchronous on `device`. */
int mf3d_tecbin_decode_device(const void *image, const mf3d_tecbin_info *info, double *const *out, int device);

/* The writer: the file image of mf3d_tecbin_size bytes into device memory
 * `image` from the node coordinates x[toti], y[totj], z[totk] and the 16
 * fields in the reader's order (device arrays, NULL = zeros). */
int mf3d_tecbin_encode_device(int toti, int totj, int totk, int pl, int inind, int jnind, int knind,
                              const double *x, const double *y, const double *z, const double *const *fields,
                              void *image, int device);

#ifdef __cplusplus
}
#endif

#endif /* MF3D_H */
