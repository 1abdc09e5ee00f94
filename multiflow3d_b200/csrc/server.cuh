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

}  // namespace mf3d

struct mf3d_server {
  std::unique_ptr<mf3d_ctx> C;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<mf3d::SrvReq *> queue;
  std::unordered_map<long long, std::unique_ptr<mf3d::SrvReq>> reqs;
  long long next_ticket = 1;
  double cap = 0.0;
  int max_resident = 1;
  double used = 0.0;
  long long submitted = 0, completed = 0, resident = 0, cycles = 0;
  bool stop = false;
  std::thread worker;
};

namespace mf3d {

// Record the end of a request (under the server lock).
static void srv_finish(mf3d_server *S, SrvReq *r, int status) {
  std::lock_guard<std::mutex> lk(S->mu);
  if (r->state == 1) S->resident--;
  r->state = 2;
  r->status = status;
  r->info.info.status = status;
  r->info.t_done = steady_now();
  S->used -= r->est;
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
    k_face_planes<<<V.n_planes, kTile, 0, s>>>(V.df.p, V.t_planes.p);
    calvel_calmas<T>(C, V, fmask.p, V.rmax.p, 0);
    k_dom_init<<<1, 256, 0, s>>>(V.ds.p + ncont, nd - ncont, V.rmax.p + ncont, V.act.p + ncont);
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

template <typename T>
static void srv_loop(mf3d_server *S) {
  mf3d_ctx *C = S->C.get();
  cudaSetDevice(C->device);
  cudaStream_t s = C->stream;
  View V;
  std::vector<SrvReq *> res;
  std::vector<int> act;
  bool dirty = false;
  auto fail_all = [&](int st) {
    for (SrvReq *r : res) {
      r->dom.reset();
      srv_finish(S, r, st);
    }
    res.clear();
    V.drop_graphs();
  };
  for (;;) {
    std::vector<SrvReq *> admit;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      if (res.empty() && S->queue.empty() && !S->stop) S->cv_work.wait_for(lk, std::chrono::milliseconds(20));
      if (S->stop) break;
      // arrival order; a request waits at the head until memory frees up,
      // unless nothing is resident (then it is admitted and may fail on OOM)
      while (!S->queue.empty() && (int)(res.size() + admit.size()) < S->max_resident) {
        SrvReq *r = S->queue.front();
        if (!(res.empty() && admit.empty()) && S->used + r->est > S->cap) break;
        S->queue.pop_front();
        S->used += r->est;
        r->state = 1;
        S->resident++;
        admit.push_back(r);
      }
    }
    for (SrvReq *r : admit) {
      r->dom.reset(new DomainStore());
      mf3d_block_desc b = lone_block(r->desc);
      const int st = build_domain(*r->dom, &b, 1, r->ngrid, C->elem, C->elem, C->prm.pl, s);
      if (st) {
        r->dom.reset();
        srv_finish(S, r, st);
        continue;
      }
      r->info.t_admit = steady_now();
      r->vidx = -1;
      res.push_back(r);
      dirty = true;
    }
    if (res.empty()) continue;
    if (dirty) {
      const int st = srv_rebuild<T>(C, V, res);
      if (st) { fail_all(st); continue; }
      dirty = false;
    }
    // one outer iteration of every resident request
    iteration_body<T>(C, V, false);
    const int nd = (int)res.size();
    act.assign(nd, 0);
    if (cudaMemcpyAsync(act.data(), V.act.p, nd * sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      set_error(std::string("server cycle: ") + cudaGetErrorString(cudaGetLastError()));
      fail_all(MF3D_E_CUDA);
      continue;
    }
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->cycles++;
    }
    std::vector<int> fin(nd, 0);
    bool any = false;
    for (int d = 0; d < nd; ++d) any |= (fin[d] = act[d] == 0);
    if (!any) continue;
    // final calvel of the finished requests, then hand them back
    std::vector<DomState> hs(nd);
    DevBuf<int> fmask;
    int st = fmask.upload(fin, s);
    if (!st) {
      k_calvel<<<V.n_int, dim3(RW_TX, RW_RJ), 0, s>>>(V.df.p, V.t_int.p, V.ds.p, fmask.p);
      if (cudaMemcpyAsync(hs.data(), V.ds.p, nd * sizeof(DomState), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        st = MF3D_E_CUDA;
    }
    if (!st) st = check_device_error(V);
    if (st) { fail_all(st); continue; }
    std::vector<SrvReq *> keep;
    for (int d = 0; d < nd; ++d) {
      SrvReq *r = res[d];
      if (!fin[d]) { keep.push_back(r); continue; }
      const DomState &D = hs[d];
      r->info.info.rmax = D.iter > 0 ? D.rmax : D.rmax0;
      r->info.info.rmax0 = D.rmax0;
      r->info.info.iter = D.iter;
      r->info.info.ms_device = 0.f;
      r->dom.reset();
      srv_finish(S, r, srv_status(D));
    }
    res.swap(keep);
    dirty = true;
  }
  fail_all(MF3D_E_INVALID);  // stopped: drop what is resident
}

}  // namespace mf3d

extern "C" {

double mf3d_server_clock(void) { return mf3d::steady_now(); }

int mf3d_server_create(const mf3d_params *prm, double mem_cap_bytes, int max_resident, mf3d_server **out) {
  using namespace mf3d;
  if (!prm || !out || max_resident < 1 || !(mem_cap_bytes > 0)) {
    set_error("mf3d_server_create: bad arguments");
    return MF3D_E_INVALID;
  }
  mf3d_params p = *prm;
  p.ngrid = std::max(p.ngrid, 1);
  int st = check_params(&p);
  if (st) return st;
  auto S = std::make_unique<mf3d_server>();
  S->C = std::make_unique<mf3d_ctx>();
  if ((st = ctx_init(S->C.get(), &p))) return st;
  S->C->use_graph = false;
  S->cap = mem_cap_bytes;
  S->max_resident = max_resident;
  mf3d_server *raw = S.get();
  if (S->C->elem == 8) S->worker = std::thread(srv_loop<double>, raw);
  else S->worker = std::thread(srv_loop<float>, raw);
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
  auto r = std::make_unique<SrvReq>();
  r->desc = *dom;
  r->fields = *f;
  r->fields.su = nullptr;
  r->dt = dt;
  r->alfapr = alfapr;
  r->ngrid = ngrid;
  r->est = domain_bytes(*dom, ngrid, S->C->elem);
  r->info.t_submit = steady_now();
  std::lock_guard<std::mutex> lk(S->mu);
  r->ticket = S->next_ticket++;
  *ticket = r->ticket;
  S->queue.push_back(r.get());
  S->reqs[r->ticket] = std::move(r);
  S->submitted++;
  S->cv_work.notify_one();
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
  if (queued) *queued = (long long)S->queue.size();
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
  if (S->worker.joinable()) S->worker.join();
  mf3d_ctx *C = S->C.release();
  S->reqs.clear();
  delete S;
  return mf3d_destroy(C);
}

}  // extern "C"
