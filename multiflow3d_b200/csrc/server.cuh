// Serving: a request loop that admits independent single-block solves as
// they arrive, keeps their hierarchies resident on the device, and advances
// every resident request by one outer iteration per cycle in shared launches
// (continuous batching).  Included at the end of mf3d.cu (one translation
// unit with the engine it drives).
//
// Each request is a domain of its own: its DomState (iteration count,
// thresholds, rmax) lives on the device and travels with it when the view is
// rebuilt for a new mix, so it runs exactly the operation sequence of its own
// solve and its result does not depend on what else is resident.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>

namespace mf3d {

static double steady_now() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct SrvReq {
  long long ticket = 0;
  mf3d_domain_desc desc{};
  mf3d_fields fields{};
  double dt = 1.0, alfapr = 1.0;
  int ngrid = 1;
  double est = 0.0;            // device bytes the request holds while resident
  int state = 0;               // 0 queued, 1 resident, 2 finished
  int status = MF3D_PENDING;
  int vidx = -1;               // index in the current view (-1: not yet in one)
  int lane = 0;
  mf3d_request_info info{};
  std::unique_ptr<DomainStore> dom;
};

// Device bytes of one domain's resident storage (build_block's sizes) plus
// the launch tables a view spends on it.
static double domain_bytes(const mf3d_domain_desc &d, int ngrid, int elem) {
  double b = 0.0;
  for (int g = 1; g <= ngrid; ++g) {
    const int nx = d.nx >> (g - 1), ny = d.ny >> (g - 1), nz = d.nz >> (g - 1);
    const long long cstr = ((long long)(nz + 2) * (ny + 2) * hp_of(nx, elem) + 31) / 32 * 32;
    b += 4.0 * cstr * elem + 9.0 * (nx + ny + nz + 6) * elem + 4 * sizeof(CUtensorMap);
    // tiles of the sweep, restriction, prolongation and cell lists
    b += 4.0 * sizeof(Tile) * ((double)(nx + 2) * (ny + 2) * (nz + 2) / 2048.0 + 4.0);
  }
  b += 8.0 * 5.0 * (d.nx + d.ny + d.nz + 6);                                            // level-1 geometry
  b += 16.0 * ((double)d.ny * d.nz + (double)d.nx * d.nz + (double)d.nx * d.ny);        // face planes
  b += 8.0 * ((double)(d.nx + 2) * (d.ny + 2) + (d.nx + 2) * (d.nz + 2) + (d.ny + 2) * (d.nz + 2));  // halo pairs
  return b;
}

// Shape key of a domain whose storage can be reused by a later request
// (uniform spacing only: stretched widths are caller arrays); "" otherwise.
static std::string shape_key(const mf3d_domain_desc &d, int ngrid) {
  if (d.hx || d.hy || d.hz) return std::string();
  char buf[256];
  std::snprintf(buf, sizeof buf, "%d,%d,%d,%d,%d,%d,%d,%a,%a,%a", d.nx, d.ny, d.nz, d.bc[0], d.bc[1], d.bc[2], ngrid,
                d.dx, d.dy, d.dz);
  return buf;
}

}  // namespace mf3d

// Requests run in two lanes by size, each with its own worker thread,
// stream and view: the cycle of a lane costs about the work of its largest
// resident domains, so small requests do not advance at the pace of large
// ones; the lanes' kernels share the device concurrently.
namespace mf3d {
constexpr int kSrvLanes = 2;
constexpr double kSrvLargeCells = 8.0e6;  // a request of at least this many cells runs in lane 1
// Lane 1 holds one request at a time: a request that size fills the device
// alone, so two resident together each advance at half the pace and both
// finish late; one at a time they finish in arrival order at full pace.
constexpr int kSrvLargeResident = 1;
constexpr int kSrvIters = 8;              // outer iterations per cycle at most (fewer when a request stops)
}  // namespace mf3d

struct mf3d_server {
  std::unique_ptr<mf3d_ctx> C[mf3d::kSrvLanes];
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<mf3d::SrvReq *> queue[mf3d::kSrvLanes];
  std::unordered_map<long long, std::unique_ptr<mf3d::SrvReq>> reqs;
  long long next_ticket = 1;
  double cap = 0.0;
  int max_resident = 1;
  double used = 0.0;            // estimated bytes of resident requests
  double pooled = 0.0;          // bytes of retired storage kept for reuse
  long long submitted = 0, completed = 0, resident = 0, cycles = 0;
  int lane_resident[mf3d::kSrvLanes] = {};  // resident requests per lane
  double t_build = 0.0, t_rebuild = 0.0, t_cycle = 0.0, t_finish = 0.0;  // worker seconds, all lanes
  long long builds = 0, rebuilds = 0;
  bool stop = false;
  std::thread worker[mf3d::kSrvLanes];
};

namespace mf3d {

// Record the end of a request (under the server lock).  `release`: its
// device bytes are given back now (else when its storage leaves the view).
static void srv_finish(mf3d_server *S, SrvReq *r, int status, bool release = true) {
  std::lock_guard<std::mutex> lk(S->mu);
  if (r->state == 1) {
    S->resident--;
    S->lane_resident[r->lane]--;
  }
  r->state = 2;
  r->status = status;
  r->info.info.status = status;
  r->info.t_done = steady_now();
  if (release) S->used -= r->est;
  S->completed++;
  S->cv_done.notify_all();
}

// Rebuild the view over the resident requests `res` (those with vidx >= 0,
// a prefix, keep their device state; the rest are new and are initialised:
// face planes, the initial calvel/calmas, rmax0 and thresholds).
template <typename T>
static int srv_rebuild(mf3d_ctx *C, View &V, std::vector<SrvReq *> &res) {
  cudaStream_t s = C->stream;
  std::vector<DomState> old(V.ds.n);
  if (!old.empty()) CK(cudaMemcpy(old.data(), V.ds.p, old.size() * sizeof(DomState), cudaMemcpyDeviceToHost));
  const int nd = (int)res.size();
  int ncont = 0;
  while (ncont < nd && res[ncont]->vidx >= 0) ++ncont;
  std::vector<DomainStore *> doms(nd);
  std::vector<mf3d_fields> fields(nd);
  for (int d = 0; d < nd; ++d) {
    doms[d] = res[d]->dom.get();
    fields[d] = res[d]->fields;
  }
  int st;
  if ((st = build_view(C, V, doms, 1))) return st;
  // tuned schedules of levels seen before; a miss keeps the defaults (no
  // timing inside a serving cycle)
  if ((st = autotune_view(C, V, false))) return st;
  std::vector<DomState> hs(nd);
  std::vector<int> fresh(nd, 0);
  for (int d = 0; d < nd; ++d) {
    SrvReq *r = res[d];
    if (d < ncont) {
      hs[d] = old[r->vidx];
    } else {
      std::memset(&hs[d], 0, sizeof(DomState));
      hs[d].dt = r->dt;
      hs[d].dtinv = pow2_inverse(r->dt);
      hs[d].rdt = div_reciprocal(r->dt);
      hs[d].alfapr = r->alfapr;
      hs[d].tol = C->prm.eps;
      hs[d].eps_relative = C->prm.eps_relative;
      hs[d].maxcy = std::max(C->prm.maxcy, 0);
      fresh[d] = 1;
    }
    r->vidx = d;
  }
  CK(cudaMemcpyAsync(V.ds.p, hs.data(), nd * sizeof(DomState), cudaMemcpyHostToDevice, s));
  if ((st = bind_fields(C, V, fields.data()))) return st;
  if (ncont < nd) {
    DevBuf<int> fmask;
    if ((st = fmask.upload(fresh, s))) return st;
    launch(k_face_planes, V.n_planes, kTile, 0, s, V.df.p, V.t_planes.p, 0);
    calvel_calmas<T>(C, V, fmask.p, V.rmax.p, 0);
    launch(k_dom_init, 1, 256, 0, s, V.ds.p + ncont, nd - ncont, V.rmax.p + ncont, V.act.p + ncont);
    CK(cudaStreamSynchronize(s));  // fmask and the host vectors are locals
  } else {
    CK(cudaStreamSynchronize(s));
  }
  CK(cudaGetLastError());
  return MF3D_OK;
}

// Status of a finished domain from its device state (as collect does).
static int srv_status(const DomState &D) {
  int status = MF3D_OK;
  if (D.done == 2) status = MF3D_E_NONFINITE;
  else if (D.done != 1) status = MF3D_NOT_CONVERGED;
  const double rmax = D.iter > 0 ? D.rmax : D.rmax0;
  if (status >= 0 && rmax > 100.0) status = MF3D_DIVERGED;  // newsolv_mg.for:64
  return status;
}

// A position in the current view: a running request, or the storage of one
// that finished and has been handed back (kept until the next rebuild, since
// the view's tables still point at it; its domain is inactive meanwhile).
struct SrvSlot {
  SrvReq *r = nullptr;
  std::unique_ptr<DomainStore> dead;
  std::string key;
  double est = 0.0;
};

template <typename T>
static void srv_loop(mf3d_server *S, int lane) {
  mf3d_ctx *C = S->C[lane].get();
  std::deque<SrvReq *> &queue = S->queue[lane];
  cudaSetDevice(C->device);
  cudaStream_t s = C->stream;
  AllocScope scope(s);  // the lane's device memory is ordered on its own stream
  View V;
  std::vector<SrvSlot> slots;     // view order
  std::vector<SrvReq *> pending;  // built, waiting for the next rebuild
  std::vector<int> act;
  // Retired hierarchies kept for later requests of the same shape (they end
  // a solve with the invariants a fresh one starts with: zero ghost shell of
  // the level-1 correction, coarse levels rewritten before use).  Oldest
  // first; evicted when admission needs the memory.
  std::vector<std::pair<std::string, std::unique_ptr<DomainStore>>> pool;
  std::vector<double> pool_est;
  // rebuild pacing: a rebuild (host tables, uploads) costs several cycles
  // when many domains are resident, so joins and leaves are gathered until
  // the cycles since the last rebuild have taken about as long as one
  double rebuild_s = 0.0, cycle_s = 1e-3, since_rebuild_s = 0.0;
  auto evict_oldest = [&]() {
    if (pool.empty()) return;
    pool.erase(pool.begin());
    const double b = pool_est.front();
    pool_est.erase(pool_est.begin());
    std::lock_guard<std::mutex> lk(S->mu);
    S->pooled -= b;
  };
  auto fail_all = [&](int st) {
    for (SrvSlot &x : slots)
      if (x.r) {
        x.r->dom.reset();
        srv_finish(S, x.r, st);
      } else if (x.dead) {
        x.dead.reset();
        std::lock_guard<std::mutex> lk(S->mu);
        S->used -= x.est;
      }
    for (SrvReq *r : pending) {
      r->dom.reset();
      srv_finish(S, r, st);
    }
    slots.clear();
    pending.clear();
    V.drop_graphs();
  };
  for (;;) {
    int live = 0, dead = 0;
    for (const SrvSlot &x : slots) (x.r ? live : dead) += 1;
    std::vector<SrvReq *> admit;
    std::vector<int> reuse;  // pool index per admitted request, -1: build
    bool need_room = false;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      if (live == 0 && pending.empty() && queue.empty() && !S->stop)
        S->cv_work.wait_for(lk, std::chrono::milliseconds(20));
      if (S->stop) break;
      // arrival order; a request waits at the head until memory frees up,
      // unless nothing else is resident (then it is admitted and may fail on OOM)
      std::vector<char> taken(pool.size(), 0);
      while (!queue.empty() && S->resident < S->max_resident &&
             (lane == 0 || S->lane_resident[lane] < kSrvLargeResident)) {
        SrvReq *r = queue.front();
        const std::string key = shape_key(r->desc, r->ngrid);
        int hit = -1;
        for (size_t q = 0; q < pool.size() && !key.empty(); ++q)
          if (!taken[q] && pool[q].first == key) { hit = (int)q; break; }
        const double extra = hit >= 0 ? 0.0 : r->est;  // a pooled store is already counted
        const bool alone = S->resident == 0;  // nothing resident in any lane
        if (!alone && S->used + S->pooled + extra > S->cap) {
          need_room = !pool.empty();
          break;
        }
        queue.pop_front();
        if (hit >= 0) {
          taken[hit] = 1;
          S->pooled -= pool_est[hit];
        }
        S->used += r->est;
        r->state = 1;
        S->resident++;
        S->lane_resident[lane]++;
        admit.push_back(r);
        reuse.push_back(hit);
      }
    }
    // take the reused stores out of the pool (highest index first)
    std::vector<std::unique_ptr<DomainStore>> got(admit.size());
    {
      std::vector<std::pair<int, int>> order;
      for (size_t a = 0; a < admit.size(); ++a)
        if (reuse[a] >= 0) order.push_back({reuse[a], (int)a});
      std::sort(order.rbegin(), order.rend());
      for (auto &o : order) {
        got[o.second] = std::move(pool[o.first].second);
        pool.erase(pool.begin() + o.first);
        pool_est.erase(pool_est.begin() + o.first);
      }
    }
    if (need_room && admit.empty()) evict_oldest();
    for (size_t a = 0; a < admit.size(); ++a) {
      SrvReq *r = admit[a];
      int st = MF3D_OK;
      if (got[a]) {
        r->dom = std::move(got[a]);
      } else {
        const double tb = steady_now();
        r->dom.reset(new DomainStore());
        mf3d_block_desc b = lone_block(r->desc);
        st = build_domain(*r->dom, &b, 1, r->ngrid, C->elem, C->elem, C->prm.pl, s);
        std::lock_guard<std::mutex> lk(S->mu);
        S->t_build += steady_now() - tb;
        S->builds++;
      }
      if (st) {
        r->dom.reset();
        srv_finish(S, r, st);
        continue;
      }
      r->info.t_admit = steady_now();
      r->vidx = -1;
      pending.push_back(r);
    }
    // rebuild the view when requests wait to join or finished ones can leave
    const bool want = !pending.empty() || dead > 0;
    const bool due = live == 0 || since_rebuild_s >= rebuild_s || 2 * dead >= (int)slots.size();
    if (want && due) {
      const double t0 = steady_now();
      std::vector<SrvReq *> res;
      std::vector<SrvSlot> next;
      for (SrvSlot &x : slots) {
        if (x.r) {
          res.push_back(x.r);
          continue;
        }
        // storage of a finished request leaves the view: reuse or free it
        std::lock_guard<std::mutex> lk(S->mu);
        S->used -= x.est;
        if (!x.key.empty()) {
          pool.emplace_back(x.key, std::move(x.dead));
          pool_est.push_back(x.est);
          S->pooled += x.est;
        }
      }
      for (SrvReq *r : pending) res.push_back(r);
      pending.clear();
      for (SrvReq *r : res) {
        SrvSlot x;
        x.r = r;
        next.push_back(std::move(x));
      }
      const int st = res.empty() ? MF3D_OK : srv_rebuild<T>(C, V, res);
      slots.swap(next);
      next.clear();  // frees the storage of finished requests that was not pooled
      if (st) { fail_all(st); continue; }
      rebuild_s = steady_now() - t0;
      since_rebuild_s = 0.0;
      {
        std::lock_guard<std::mutex> lk(S->mu);
        S->t_rebuild += rebuild_s;
        S->rebuilds++;
      }
      live = (int)slots.size();
    }
    if (live == 0) continue;
    // outer iterations of every running request, as one graph launch that
    // returns when a request stops or after kSrvIters iterations
    const double c0 = steady_now();
    if (!V.x_loop && build_server_graph<T>(C, V)) {
      fail_all(MF3D_E_CUDA);
      continue;
    }
    const int nd = (int)slots.size();
    act.assign(nd, 0);
    if (cudaMemcpyAsync(V.budget.p, &kSrvIters, sizeof(int), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaGraphLaunch(V.x_loop, s) != cudaSuccess ||
        cudaMemcpyAsync(act.data(), V.act.p, nd * sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      set_error(std::string("server cycle: ") + cudaGetErrorString(cudaGetLastError()));
      fail_all(MF3D_E_CUDA);
      continue;
    }
    const double dc = steady_now() - c0;
    cycle_s = 0.8 * cycle_s + 0.2 * dc;
    since_rebuild_s += dc;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->cycles++;
      S->t_cycle += dc;
    }
    std::vector<int> fin(nd, 0);
    bool any = false;
    for (int d = 0; d < nd; ++d) any |= (fin[d] = slots[d].r != nullptr && act[d] == 0);
    if (!any) continue;
    // final calvel of the finished requests, then hand them back
    const double tf = steady_now();
    std::vector<DomState> hs(nd);
    DevBuf<int> fmask;
    int st = fmask.upload(fin, s);
    if (!st) {
      launch(k_calvel, V.n_int, dim3(RW_TX, RW_RJ), 0, s, V.df.p, V.t_int.p, V.ds.p, fmask.p);
      launch(k_vel_faces, V.n_vfaces, kTile, 0, s, V.df.p, V.t_vfaces.p, fmask.p, C->prm.pl_ex);
      if (cudaMemcpyAsync(hs.data(), V.ds.p, nd * sizeof(DomState), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        st = MF3D_E_CUDA;
    }
    if (!st) st = check_device_error(V);
    if (st) { fail_all(st); continue; }
    for (int d = 0; d < nd; ++d) {
      if (!fin[d]) continue;
      SrvSlot &x = slots[d];
      SrvReq *r = x.r;
      const DomState &D = hs[d];
      r->info.info.rmax = D.iter > 0 ? D.rmax : D.rmax0;
      r->info.info.rmax0 = D.rmax0;
      r->info.info.iter = D.iter;
      r->info.info.ms_device = 0.f;
      const int status = srv_status(D);
      x.key = status >= 0 ? shape_key(r->desc, r->ngrid) : std::string();
      x.est = r->est;
      x.dead = std::move(r->dom);
      x.r = nullptr;
      srv_finish(S, r, status, false);  // r may be released by a poll from here on
    }
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->t_finish += steady_now() - tf;
    }
  }
  fail_all(MF3D_E_INVALID);  // stopped: drop what is resident
}

}  // namespace mf3d

extern "C" {

double mf3d_server_clock(void) { return mf3d::steady_now(); }

int mf3d_server_profile(mf3d_server *S, double *build_s, double *rebuild_s, double *cycle_s, double *finish_s,
                        long long *builds, long long *rebuilds) {
  if (!S) { mf3d::set_error("mf3d_server_profile: bad arguments"); return MF3D_E_INVALID; }
  std::lock_guard<std::mutex> lk(S->mu);
  if (build_s) *build_s = S->t_build;
  if (rebuild_s) *rebuild_s = S->t_rebuild;
  if (cycle_s) *cycle_s = S->t_cycle;
  if (finish_s) *finish_s = S->t_finish;
  if (builds) *builds = S->builds;
  if (rebuilds) *rebuilds = S->rebuilds;
  return MF3D_OK;
}

int mf3d_server_create(const mf3d_params *prm, double mem_cap_bytes, int max_resident, mf3d_server **out) {
  using namespace mf3d;
  if (!prm || !out || max_resident < 1 || !(mem_cap_bytes > 0)) {
    set_error("mf3d_server_create: bad arguments");
    return MF3D_E_INVALID;
  }
  if (prm->lsm || prm->bounds || prm->solver == 1) {
    set_error("lsm, bounds and solver 1: single-problem contexts (mf3d_create) only");
    return MF3D_E_UNSUPPORTED;
  }
  mf3d_params p = *prm;
  p.ngrid = std::max(p.ngrid, 1);
  int st = check_params(&p);
  if (st) return st;
  auto S = std::make_unique<mf3d_server>();
  for (int l = 0; l < kSrvLanes; ++l) {
    S->C[l] = std::make_unique<mf3d_ctx>();
    // lane 0 (small requests, latency-bound cycles) gets the high-priority
    // stream: its CTAs are scheduled ahead of lane 1's queued ones
    if ((st = ctx_init(S->C[l].get(), &p, true, l == 0))) return st;
    S->C[l]->use_graph = false;
  }
  S->cap = mem_cap_bytes;
  S->max_resident = max_resident;
  mf3d_server *raw = S.get();
  for (int l = 0; l < kSrvLanes; ++l) {
    if (S->C[l]->elem == 8) S->worker[l] = std::thread(srv_loop<double>, raw, l);
    else S->worker[l] = std::thread(srv_loop<float>, raw, l);
  }
  *out = S.release();
  return MF3D_OK;
}

int mf3d_server_submit(mf3d_server *S, const mf3d_domain_desc *dom, const mf3d_fields *f, double dt, double alfapr,
                       long long *ticket) {
  using namespace mf3d;
  if (!S || !dom || !f || !ticket) { set_error("mf3d_server_submit: bad arguments"); return MF3D_E_INVALID; }
  if (!f->ustar || !f->vstar || !f->wstar || !f->u || !f->v || !f->w || !f->p) {
    set_error("mf3d_server_submit: a required field pointer is NULL");
    return MF3D_E_INVALID;
  }
  const int ngrid = domain_ngrid(*dom);
  if (ngrid < 1) { set_error("mf3d_server_submit: sizes not divisible by 2^(ngrid-1)"); return MF3D_E_INVALID; }
  if (!edges_exceed(*dom, S->C[0]->prm.pl_ex)) {
    set_error("mf3d_server_submit: an edge does not exceed pl_ex");
    return MF3D_E_INVALID;
  }
  if (S->C[0]->prm.differencing == 2 && (dom->hx || dom->hy || dom->hz)) {
    set_error("mf3d_server_submit: differencing = 2 needs uniform spacing");
    return MF3D_E_UNSUPPORTED;
  }
  auto r = std::make_unique<SrvReq>();
  r->desc = *dom;
  r->fields = *f;
  r->fields.su = nullptr;
  r->dt = dt;
  r->alfapr = alfapr;
  r->ngrid = ngrid;
  r->est = domain_bytes(*dom, ngrid, S->C[0]->elem);
  r->info.t_submit = steady_now();
  const int lane = (double)dom->nx * dom->ny * dom->nz >= kSrvLargeCells ? 1 : 0;
  r->lane = lane;
  std::lock_guard<std::mutex> lk(S->mu);
  r->ticket = S->next_ticket++;
  *ticket = r->ticket;
  S->queue[lane].push_back(r.get());
  S->reqs[r->ticket] = std::move(r);
  S->submitted++;
  S->cv_work.notify_all();
  return MF3D_OK;
}

int mf3d_server_poll(mf3d_server *S, long long ticket, mf3d_request_info *info, int wait_ms) {
  using namespace mf3d;
  if (!S) { set_error("mf3d_server_poll: bad arguments"); return MF3D_E_INVALID; }
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) { set_error("mf3d_server_poll: unknown ticket"); return MF3D_E_INVALID; }
  SrvReq *r = it->second.get();
  if (r->state != 2 && wait_ms > 0)
    S->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return r->state == 2; });
  if (r->state != 2) return MF3D_PENDING;
  const int status = r->status;
  if (info) *info = r->info;
  S->reqs.erase(it);
  return status;
}

int mf3d_server_stats(mf3d_server *S, long long *submitted, long long *completed, long long *resident,
                      long long *queued, double *resident_bytes, long long *cycles) {
  if (!S) { mf3d::set_error("mf3d_server_stats: bad arguments"); return MF3D_E_INVALID; }
  std::lock_guard<std::mutex> lk(S->mu);
  if (submitted) *submitted = S->submitted;
  if (completed) *completed = S->completed;
  if (resident) *resident = S->resident;
  if (queued) *queued = (long long)(S->queue[0].size() + S->queue[1].size());
  if (resident_bytes) *resident_bytes = S->used;
  if (cycles) *cycles = S->cycles;
  return MF3D_OK;
}

int mf3d_server_destroy(mf3d_server *S) {
  if (!S) return MF3D_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
    S->cv_work.notify_all();
  }
  for (auto &w : S->worker)
    if (w.joinable()) w.join();
  mf3d_ctx *C[kSrvLanes];
  for (int l = 0; l < kSrvLanes; ++l) C[l] = S->C[l].release();
  S->reqs.clear();
  delete S;
  for (int l = 0; l < kSrvLanes; ++l) mf3d_destroy(C[l]);
  return MF3D_OK;
}

}  // extern "C"
