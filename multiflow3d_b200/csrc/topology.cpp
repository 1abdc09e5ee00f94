// Host-side set-up of libmf3d: neighbour search, multigrid halo copy maps
// and field face rules.  Pure C++, no CUDA.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <unordered_map>

#include "mf3d_internal.h"

namespace mf3d {

// ---------------------------------------------------------------------------
// Neighbour search (alloc_dom.for:456-1150).  Two blocks touch when their
// face coordinates agree within 1e-8 (the reference's tolerance); face
// neighbours must share both tangential extents, edge neighbours the one
// extent along the edge, corner neighbours only the corner point.  Periodic
// partners are searched against the domain's bounding box (xst..zen).
// ---------------------------------------------------------------------------
int build_topology(int nb, const double *ext, const int *bc6, double dx, double dy,
                   double dz, mf3d_block_desc *out) {
  if (nb <= 0 || !ext || !bc6 || !out) {
    set_error("build_topology: bad arguments");
    return MF3D_E_INVALID;
  }
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int b = 0; b < nb; ++b)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], ext[6 * b + 2 * a]);
      hi[a] = std::max(hi[a], ext[6 * b + 2 * a + 1]);
    }
  auto S = [&](int b, int a) { return ext[6 * b + 2 * a]; };      // start along axis a
  auto E = [&](int b, int a) { return ext[6 * b + 2 * a + 1]; };  // end along axis a
  auto eq = [](double x, double y) { return std::fabs(x - y) < 1e-8; };
  auto same = [&](int b, int o, int a) { return eq(S(b, a), S(o, a)) && eq(E(b, a), E(o, a)); };
  // Relation of block o to block b along axis a: -1 = o ends where b starts,
  // +1 = o starts where b ends, 0 = same extent, 2 = none.
  auto rel = [&](int b, int o, int a) -> int {
    if (eq(S(b, a), E(o, a))) return -1;
    if (eq(E(b, a), S(o, a))) return +1;
    return same(b, o, a) ? 0 : 2;
  };
  const double h[3] = {dx, dy, dz};
  // offsets of the reference's numbered corner / edge neighbours
  const int corp[4][2] = {{-1, -1}, {-1, +1}, {+1, +1}, {+1, -1}};  // (x,y) at z-1
  const int corn[4][2] = {{+1, +1}, {+1, -1}, {-1, -1}, {-1, +1}};  // (x,y) at z+1
  // edges: (dx, dy, dz) with 0 meaning "same extent"
  const int edp[6][3] = {{-1, 0, -1}, {0, +1, -1}, {+1, 0, -1}, {0, -1, -1}, {-1, -1, 0}, {-1, +1, 0}};
  const int edn[6][3] = {{+1, 0, +1}, {0, -1, +1}, {-1, 0, +1}, {0, +1, +1}, {+1, +1, 0}, {+1, -1, 0}};
  for (int b = 0; b < nb; ++b) {
    mf3d_block_desc &d = out[b];
    std::memset(&d, 0, sizeof d);
    d.id = b;
    d.dx = dx; d.dy = dy; d.dz = dz;
    d.xsl = S(b, 0); d.xel = E(b, 0); d.ysl = S(b, 1); d.yel = E(b, 1); d.zsl = S(b, 2); d.zel = E(b, 2);
    int n[3];
    for (int a = 0; a < 3; ++a) {
      double c = (E(b, a) - S(b, a)) / h[a];
      if (std::fabs(c - std::nearbyint(c)) > 1e-8 || c < 1) {  // localparameters.for:84-98
        set_error("block " + std::to_string(b) + ": extent is not a whole number of cells");
        return MF3D_E_INVALID;
      }
      n[a] = (int)std::nearbyint(c);
    }
    d.nx = n[0]; d.ny = n[1]; d.nz = n[2];
    d.bc_west = bc6[0]; d.bc_east = bc6[1]; d.bc_south = bc6[2];
    d.bc_north = bc6[3]; d.bc_bottom = bc6[4]; d.bc_top = bc6[5];
    int face[6];
    for (int f = 0; f < 6; ++f) face[f] = -1;
    for (int q = 0; q < 4; ++q) d.corprev[q] = d.cornext[q] = -1;
    for (int q = 0; q < 6; ++q) d.edgprev[q] = d.edgnext[q] = -1;
    int count_face[6] = {0};
    for (int o = 0; o < nb; ++o) {
      if (o == b) continue;
      int r[3] = {rel(b, o, 0), rel(b, o, 1), rel(b, o, 2)};
      for (int a = 0; a < 3; ++a) {
        int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
        if ((r[a] == -1 || r[a] == 1) && r[t1] == 0 && r[t2] == 0) {
          int f = 2 * a + (r[a] == 1);
          face[f] = o;
          ++count_face[f];
        }
      }
      // corners: only the corner point must coincide
      auto corner = [&](int sx, int sy, int sz) {
        bool x = sx < 0 ? eq(S(b, 0), E(o, 0)) : eq(E(b, 0), S(o, 0));
        bool y = sy < 0 ? eq(S(b, 1), E(o, 1)) : eq(E(b, 1), S(o, 1));
        bool z = sz < 0 ? eq(S(b, 2), E(o, 2)) : eq(E(b, 2), S(o, 2));
        return x && y && z;
      };
      for (int q = 0; q < 4; ++q) {
        if (corner(corp[q][0], corp[q][1], -1)) d.corprev[q] = o;
        if (corner(corn[q][0], corn[q][1], +1)) d.cornext[q] = o;
      }
      auto edge = [&](const int *e) {
        for (int a = 0; a < 3; ++a) {
          if (e[a] == 0) { if (!same(b, o, a)) return false; }
          else if (e[a] < 0) { if (!eq(S(b, a), E(o, a))) return false; }
          else if (!eq(E(b, a), S(o, a))) return false;
        }
        return true;
      };
      for (int q = 0; q < 6; ++q) {
        if (edge(edp[q])) d.edgprev[q] = o;
        if (edge(edn[q])) d.edgnext[q] = o;
      }
    }
    for (int f = 0; f < 6; ++f)
      if (count_face[f] > 1) {  // alloc_dom.for:483-487 and alike
        set_error("block " + std::to_string(b) + " has more than one neighbour on a face");
        return MF3D_E_INVALID;
      }
    d.iprev = face[0]; d.inext = face[1]; d.jprev = face[2];
    d.jnext = face[3]; d.kprev = face[4]; d.knext = face[5];
    // periodic partners: the block at the far end of the box, same tangential extents
    int *per[6] = {&d.per_ip, &d.per_in, &d.per_jp, &d.per_jn, &d.per_kp, &d.per_kn};
    for (int f = 0; f < 6; ++f) {
      *per[f] = -1;
      int a = f / 2;
      bool is_prev = (f % 2) == 0;
      if (bc6[f] != MF3D_BC_PERIODIC || face[f] >= 0) continue;
      for (int o = 0; o < nb; ++o) {
        if (o == b) continue;
        int t1 = (a + 1) % 3, t2 = (a + 2) % 3;
        if (!same(b, o, t1) || !same(b, o, t2)) continue;
        if (is_prev ? eq(hi[a], E(o, a)) : eq(lo[a], S(o, a))) *per[f] = o;
      }
    }
  }
  return MF3D_OK;
}

// ---------------------------------------------------------------------------
// Halo copy map.  Every cell of the level carries a token (the id of the
// cell whose pre-exchange value it holds); the reference's sequence of
// copies is replayed on tokens, each pack/unpack phase reading from the
// state at the start of its phase.
// ---------------------------------------------------------------------------
namespace {

struct TokenLevel {
  const std::vector<mf3d_block_desc> &blk;
  const std::vector<LevelGeom> &geom;
  const std::vector<long long> &base;
  std::unordered_map<int, int> pos;  // block id -> position
  // Only ghost cells are ever written (and interior cells keep their own
  // token), so tokens are stored for the ghost shell of each block alone:
  // the work and memory grow with the block surfaces, not their volumes.
  std::vector<std::vector<long long>> shell;
  std::vector<int> order;  // block positions by increasing base

  TokenLevel(const std::vector<mf3d_block_desc> &b, const std::vector<LevelGeom> &g,
             const std::vector<long long> &bs)
      : blk(b), geom(g), base(bs) {
    shell.resize(b.size());
    for (size_t q = 0; q < b.size(); ++q) {
      pos[b[q].id] = (int)q;
      const LevelGeom &G = g[q];
      shell[q].resize((size_t)(G.cells() - (long long)G.nx * G.ny * G.nz));
      order.push_back((int)q);
    }
    std::sort(order.begin(), order.end(), [&](int x, int y) { return bs[x] < bs[y]; });
    for (size_t q = 0; q < b.size(); ++q) {
      const LevelGeom &G = g[q];
      for (int k = 0; k <= G.nz + 1; ++k)
        for (int j = 0; j <= G.ny + 1; ++j)
          for (int i = 0; i <= G.nx + 1; ++i) {
            if (!on_shell(G, i, j, k)) {
              i = G.nx;  // skip the interior of the row
              continue;
            }
            shell[q][sidx(G, i, j, k)] = id((int)q, i, j, k);
          }
    }
  }
  static bool on_shell(const LevelGeom &G, int i, int j, int k) {
    return i == 0 || j == 0 || k == 0 || i == G.nx + 1 || j == G.ny + 1 || k == G.nz + 1;
  }
  // index of a shell cell: the two z planes, then per interior plane the two
  // y rows, then per interior row the two x ends
  static long long sidx(const LevelGeom &G, int i, int j, int k) {
    const long long W = G.nx + 2, H = G.ny + 2;
    if (k == 0) return (long long)j * W + i;
    if (k == G.nz + 1) return W * H + (long long)j * W + i;
    const long long pl = 2 * W + 2LL * G.ny;  // shell cells of one interior plane
    long long o = 2 * W * H + (long long)(k - 1) * pl;
    if (j == 0) return o + i;
    if (j == G.ny + 1) return o + W + i;
    return o + 2 * W + 2LL * (j - 1) + (i == 0 ? 0 : 1);
  }
  long long id(int p, int i, int j, int k) const { return base[p] + geom[p].lin(i, j, k); }
  int P(int block_id) const {
    auto it = pos.find(block_id);
    return it == pos.end() ? -1 : it->second;
  }
  // the block and (i, j, k) of a cell id
  void decode(long long c, int &p, int &i, int &j, int &k) const {
    int lo = 0, hi = (int)order.size() - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (base[order[mid]] <= c) lo = mid;
      else hi = mid - 1;
    }
    p = order[lo];
    const LevelGeom &G = geom[p];
    long long r = c - base[p];
    i = (int)(r % (G.nx + 2));
    r /= (G.nx + 2);
    j = (int)(r % (G.ny + 2));
    k = (int)(r / (G.ny + 2));
  }
  long long get(long long c) const {
    int p, i, j, k;
    decode(c, p, i, j, k);
    const LevelGeom &G = geom[p];
    return on_shell(G, i, j, k) ? shell[p][sidx(G, i, j, k)] : c;
  }
  void set(long long c, long long v) {
    int p, i, j, k;
    decode(c, p, i, j, k);
    shell[p][sidx(geom[p], i, j, k)] = v;  // destinations are ghost cells
  }
};

// A phase: ordered (dst, src) pairs read from the phase-start state; later
// pairs override earlier ones on the same dst.
struct Phase {
  std::vector<HaloPair> pairs;
  void add(long long d, long long s) { pairs.push_back({d, s}); }
  void apply(TokenLevel &T) const {
    std::vector<long long> v(pairs.size());
    for (size_t q = 0; q < pairs.size(); ++q) v[q] = T.get(pairs[q].src);
    for (size_t q = 0; q < pairs.size(); ++q) T.set(pairs[q].dst, v[q]);
  }
};

// Cell at index `a` along axis `ax` and (s,t) along the other two axes.
struct AxisView {
  int ax;
  long long at(const TokenLevel &T, int p, int a, int s, int t) const {
    if (ax == 0) return T.id(p, a, s, t);
    if (ax == 1) return T.id(p, s, a, t);
    return T.id(p, s, t, a);  // z: s = i, t = j
  }
};

void mgbound_tokens(TokenLevel &T) {
  for (size_t p = 0; p < T.blk.size(); ++p) {
    const auto &d = T.blk[p];
    const LevelGeom &g = T.geom[p];
    int nx = g.nx, ny = g.ny, nz = g.nz;
    auto cp = [&](long long dst, long long src) { T.set(dst, T.get(src)); };
    if (d.iprev < 0 && d.bc_west != MF3D_BC_PERIODIC)
      for (int k = 0; k <= nz + 1; ++k) for (int j = 0; j <= ny + 1; ++j) cp(T.id(p, 0, j, k), T.id(p, 1, j, k));
    if (d.inext < 0 && d.bc_east != MF3D_BC_PERIODIC)
      for (int k = 0; k <= nz + 1; ++k) for (int j = 0; j <= ny + 1; ++j) cp(T.id(p, nx + 1, j, k), T.id(p, nx, j, k));
    if (d.jprev < 0 && d.bc_south != MF3D_BC_PERIODIC)
      for (int k = 0; k <= nz + 1; ++k) for (int i = 0; i <= nx + 1; ++i) cp(T.id(p, i, 0, k), T.id(p, i, 1, k));
    if (d.jnext < 0 && d.bc_north != MF3D_BC_PERIODIC)
      for (int k = 0; k <= nz + 1; ++k) for (int i = 0; i <= nx + 1; ++i) cp(T.id(p, i, ny + 1, k), T.id(p, i, ny, k));
    if (d.kprev < 0 && d.bc_bottom != MF3D_BC_PERIODIC)
      for (int j = 0; j <= ny + 1; ++j) for (int i = 0; i <= nx + 1; ++i) cp(T.id(p, i, j, 0), T.id(p, i, j, 1));
    if (d.knext < 0 && d.bc_top != MF3D_BC_PERIODIC)
      for (int j = 0; j <= ny + 1; ++j) for (int i = 0; i <= nx + 1; ++i) cp(T.id(p, i, j, nz + 1), T.id(p, i, j, nz));
  }
}

// exchbc_mgpp (exchangepp.for:4768-5383) on tokens: x, y, z; in-block wraps
// are immediate, partner copies are packed from the axis-start state and
// unpacked afterwards.
void exchbc_tokens(TokenLevel &T) {
  const std::vector<mf3d_block_desc> &blocks = T.blk;
  const std::vector<LevelGeom> &geom = T.geom;
  const int nb = (int)blocks.size();
  // exchbc_mgpp: x, y, z; in-block wraps are immediate, partner copies
  // are packed from the axis-start state and unpacked afterwards.
  for (int ax = 0; ax < 3; ++ax) {
    AxisView V{ax};
    Phase ph;
    for (int p = 0; p < nb; ++p) {
      const auto &d = blocks[p];
      int bcp = ax == 0 ? d.bc_west : ax == 1 ? d.bc_south : d.bc_bottom;
      int bcn = ax == 0 ? d.bc_east : ax == 1 ? d.bc_north : d.bc_top;
      if (!(bcp == 5 || bcn == 5)) continue;
      const LevelGeom &g = geom[p];
      int nA = ax == 0 ? g.nx : ax == 1 ? g.ny : g.nz;
      int n1 = ax == 0 ? g.ny : g.nx, n2 = ax == 2 ? g.ny : g.nz;
      int prev = ax == 0 ? d.iprev : ax == 1 ? d.jprev : d.kprev;
      int next = ax == 0 ? d.inext : ax == 1 ? d.jnext : d.knext;
      int perp = ax == 0 ? d.per_ip : ax == 1 ? d.per_jp : d.per_kp;
      int pern = ax == 0 ? d.per_in : ax == 1 ? d.per_jn : d.per_kn;
      if (prev < 0 && next < 0) {
        for (int t = 0; t <= n2 + 1; ++t) for (int s = 0; s <= n1 + 1; ++s)
          T.set(V.at(T, p, 0, s, t), T.get(V.at(T, p, nA, s, t)));
        for (int t = 0; t <= n2 + 1; ++t) for (int s = 0; s <= n1 + 1; ++s)
          T.set(V.at(T, p, nA + 1, s, t), T.get(V.at(T, p, 1, s, t)));
        continue;
      }
      if (prev < 0 && next >= 0 && perp >= 0) {
        int q = T.P(perp);
        int nAq = ax == 0 ? geom[q].nx : ax == 1 ? geom[q].ny : geom[q].nz;
        for (int t = 0; t <= n2 + 1; ++t) for (int s = 0; s <= n1 + 1; ++s)
          ph.add(V.at(T, p, 0, s, t), V.at(T, q, nAq, s, t));
      }
      if (next < 0 && prev >= 0 && pern >= 0) {
        int q = T.P(pern);
        for (int t = 0; t <= n2 + 1; ++t) for (int s = 0; s <= n1 + 1; ++s)
          ph.add(V.at(T, p, nA + 1, s, t), V.at(T, q, 1, s, t));
      }
    }
    ph.apply(T);
  }
}

}  // namespace

std::vector<HaloPair> build_halo_map(const std::vector<mf3d_block_desc> &blocks,
                                     const std::vector<LevelGeom> &geom,
                                     const std::vector<long long> &base) {
  TokenLevel T(blocks, geom, base);
  const int nb = (int)blocks.size();
  // mgrelax calls mgbound before exchangepp (mgsolver.for:610-611)
  mgbound_tokens(T);
  bool periodic = false;
  for (const auto &d : blocks)
    if (d.bc_west == 5 || d.bc_east == 5 || d.bc_south == 5 || d.bc_north == 5 || d.bc_bottom == 5 || d.bc_top == 5)
      periodic = true;

  // exchangepp: sync_dir x, y, z
  for (int ax = 0; ax < 3; ++ax) {
    Phase ph;
    AxisView V{ax};
    for (int p = 0; p < nb; ++p) {
      const auto &d = blocks[p];
      const LevelGeom &g = geom[p];
      int nA = ax == 0 ? g.nx : ax == 1 ? g.ny : g.nz;
      int n1 = ax == 0 ? g.ny : g.nx;           // s extent (interior)
      int n2 = ax == 2 ? g.ny : g.nz;           // t extent (interior)
      int prev = ax == 0 ? d.iprev : ax == 1 ? d.jprev : d.kprev;
      int next = ax == 0 ? d.inext : ax == 1 ? d.jnext : d.knext;
      // faces: full planes including ghost rows (exchangepp.for:155-160, 4036-4043)
      if (prev >= 0) {
        int q = T.P(prev);
        int nAq = ax == 0 ? geom[q].nx : ax == 1 ? geom[q].ny : geom[q].nz;
        for (int t = 0; t <= n2 + 1; ++t) for (int s = 0; s <= n1 + 1; ++s)
          ph.add(V.at(T, p, 0, s, t), V.at(T, q, nAq, s, t));
      }
      if (next >= 0) {
        int q = T.P(next);
        for (int t = 0; t <= n2 + 1; ++t) for (int s = 0; s <= n1 + 1; ++s)
          ph.add(V.at(T, p, nA + 1, s, t), V.at(T, q, 1, s, t));
      }
      if (ax == 2) {
        // corners and edges, unpacked after the faces (exchangepp.for:4433-4755)
        int nx = g.nx, ny = g.ny, nz = g.nz;
        auto src_last = [&](int q, int a) { return a == 0 ? geom[q].nx : a == 1 ? geom[q].ny : geom[q].nz; };
        // previous corners #1..4: ghost (x,y,0) <- neighbour interior
        const int cx[4] = {0, 0, 1, 1}, cy[4] = {0, 1, 1, 0};  // 0 = low side, 1 = high side
        for (int c = 0; c < 4; ++c)
          if (d.corprev[c] >= 0) {
            int q = T.P(d.corprev[c]);
            int gi = cx[c] ? nx + 1 : 0, gj = cy[c] ? ny + 1 : 0;
            int si = cx[c] ? 1 : src_last(q, 0), sj = cy[c] ? 1 : src_last(q, 1);
            ph.add(T.id(p, gi, gj, 0), T.id(q, si, sj, src_last(q, 2)));
          }
        // previous edges #1..6
        auto edge_prev = [&](int e, int q) {
          int lx = src_last(q, 0), ly = src_last(q, 1), lz = src_last(q, 2);
          switch (e) {
            case 0: for (int j = 1; j <= ny; ++j) ph.add(T.id(p, 0, j, 0), T.id(q, lx, j, lz)); break;
            case 1: for (int i = 1; i <= nx; ++i) ph.add(T.id(p, i, ny + 1, 0), T.id(q, i, 1, lz)); break;
            case 2: for (int j = 1; j <= ny; ++j) ph.add(T.id(p, nx + 1, j, 0), T.id(q, 1, j, lz)); break;
            case 3: for (int i = 1; i <= nx; ++i) ph.add(T.id(p, i, 0, 0), T.id(q, i, ly, lz)); break;
            case 4: for (int k = 1; k <= nz; ++k) ph.add(T.id(p, 0, 0, k), T.id(q, lx, ly, k)); break;
            case 5: for (int k = 1; k <= nz; ++k) ph.add(T.id(p, 0, ny + 1, k), T.id(q, lx, 1, k)); break;
          }
        };
        for (int e = 0; e < 6; ++e)
          if (d.edgprev[e] >= 0) edge_prev(e, T.P(d.edgprev[e]));
        // next corners #1..4: ghost (x,y,nz+1)
        const int nxs[4] = {1, 1, 0, 0}, nys[4] = {1, 0, 0, 1};
        for (int c = 0; c < 4; ++c)
          if (d.cornext[c] >= 0) {
            int q = T.P(d.cornext[c]);
            int gi = nxs[c] ? nx + 1 : 0, gj = nys[c] ? ny + 1 : 0;
            int si = nxs[c] ? 1 : src_last(q, 0), sj = nys[c] ? 1 : src_last(q, 1);
            ph.add(T.id(p, gi, gj, nz + 1), T.id(q, si, sj, 1));
          }
        auto edge_next = [&](int e, int q) {
          int lx = src_last(q, 0), ly = src_last(q, 1);
          switch (e) {
            case 0: for (int j = 1; j <= ny; ++j) ph.add(T.id(p, nx + 1, j, nz + 1), T.id(q, 1, j, 1)); break;
            case 1: for (int i = 1; i <= nx; ++i) ph.add(T.id(p, i, 0, nz + 1), T.id(q, i, ly, 1)); break;
            case 2: for (int j = 1; j <= ny; ++j) ph.add(T.id(p, 0, j, nz + 1), T.id(q, lx, j, 1)); break;
            case 3: for (int i = 1; i <= nx; ++i) ph.add(T.id(p, i, ny + 1, nz + 1), T.id(q, i, 1, 1)); break;
            case 4: for (int k = 1; k <= nz; ++k) ph.add(T.id(p, nx + 1, ny + 1, k), T.id(q, 1, 1, k)); break;
            case 5: for (int k = 1; k <= nz; ++k) ph.add(T.id(p, nx + 1, 0, k), T.id(q, 1, ly, k)); break;
          }
        };
        for (int e = 0; e < 6; ++e)
          if (d.edgnext[e] >= 0) edge_next(e, T.P(d.edgnext[e]));
      }
    }
    ph.apply(T);
  }
  mgbound_tokens(T);
  if (periodic) exchbc_tokens(T);
  // changed shell cells, in increasing cell id
  std::vector<HaloPair> out;
  for (int p : T.order) {
    const LevelGeom &G = geom[p];
    for (int k = 0; k <= G.nz + 1; ++k)
      for (int j = 0; j <= G.ny + 1; ++j)
        for (int i = 0; i <= G.nx + 1; ++i) {
          if (!TokenLevel::on_shell(G, i, j, k)) {
            i = G.nx;  // skip the interior of the row
            continue;
          }
          const long long c = T.id(p, i, j, k), v = T.shell[p][TokenLevel::sidx(G, i, j, k)];
          if (v != c) out.push_back({c, v});
        }
  }
  return out;
}

// ---------------------------------------------------------------------------
// The refresh of a level with refinement interfaces (LMR).  Tokens are cell
// ids (the value the cell held before the exchange) or nodes: weighted sums
// of tokens built when a phase starts.  Each sync_dir is one phase: the
// reference packs every block's buffers from the state at the start of the
// phase and unpacks them afterwards, and an unpack formula reads only cells
// that no unpack of the same phase writes (a refined block's interior layers
// next to the face; its ghost rows of the other axes).  So every value of
// the phase is a function of the phase-start state, and later entries win.
// The cases, from the receiving block p and its neighbour q (exchangepp.for
// lines of the sender's pack and the receiver's unpack):
//   rdv equal:            copy of q's cell (as build_halo_map);
//   p finer than q, face: (2 phi_q + 3 phi_p(1 in) - phi_p(2 in)) / 4 on the
//                         whole ghost plane (:174-187, :4046-4056); the
//                         plane's ring rows receive no coarse value - the
//                         buffer entries the coarse sender never writes,
//                         taken as 0 here;
//   p coarser, face:      0.125 * (8 cells of q), q's two layers next to p,
//                         tangential pairs, the buffer's fast axis first and
//                         the normal last (:163-172), on the plane's interior
//                         (:4057-4063);
//   p coarser, corner/edge: (8 cells of q) / 8 in j, i, k order (:448-452,
//                         :652-656);
//   p finer, corner/edge: (27 c + 9 c_j + 9 c_i + 3 c_ij + 9 c_k + 3 c_jk +
//                         3 c_ik + 1 c_ijk) / 64 from q's cell c toward p
//                         (:454-460, :658-669), along an edge toward the fine
//                         cell's half of c.
// ---------------------------------------------------------------------------
namespace {

struct LmrNodeR {
  std::vector<std::pair<long long, double>> t;  // (token, weight)
  double scale;
};

struct LmrReplay {
  TokenLevel &T;
  const std::vector<int> &rdv;
  std::vector<LmrNodeR> nodes;
  static long long node_token(size_t n) { return -2 - (long long)n; }
  long long make(std::vector<std::pair<long long, double>> t, double scale) {
    nodes.push_back(LmrNodeR{std::move(t), scale});
    return node_token(nodes.size() - 1);
  }
  // cell of the face plane of axis ax: a along the axis, (s, t) the
  // reference buffer's axes (ijk = (t-1)*ns1 + s): x (j, k), y (i, k), z (j, i)
  long long fcell(int p, int ax, int a, int s, int t) const {
    if (ax == 0) return T.id(p, a, s, t);
    if (ax == 1) return T.id(p, s, a, t);
    return T.id(p, t, s, a);
  }
  int nax(int p, int a) const { return a == 0 ? T.geom[p].nx : a == 1 ? T.geom[p].ny : T.geom[p].nz; }
};

}  // namespace

LmrProgram build_halo_lmr(const std::vector<mf3d_block_desc> &blocks, const std::vector<LevelGeom> &geom,
                          const std::vector<long long> &base, const std::vector<int> &rdv) {
  TokenLevel T(blocks, geom, base);
  LmrReplay R{T, rdv, {}};
  const int nb = (int)blocks.size();
  mgbound_tokens(T);  // mgrelax's mgbound before exchangepp (mgsolver.for:610-611)
  bool periodic = false;
  for (const auto &d : blocks)
    if (d.bc_west == 5 || d.bc_east == 5 || d.bc_south == 5 || d.bc_north == 5 || d.bc_bottom == 5 || d.bc_top == 5)
      periodic = true;
  using Terms = std::vector<std::pair<long long, double>>;
  for (int ax = 0; ax < 3; ++ax) {
    std::vector<std::pair<long long, long long>> ph;  // (dst, token), in unpack order
    for (int p = 0; p < nb; ++p) {
      const auto &d = blocks[p];
      const int nA = R.nax(p, ax);
      const int n1 = ax == 1 ? geom[p].nx : geom[p].ny;  // s extent
      const int n2 = ax == 2 ? geom[p].nx : geom[p].nz;  // t extent
      const int nbr[2] = {ax == 0 ? d.iprev : ax == 1 ? d.jprev : d.kprev, ax == 0 ? d.inext : ax == 1 ? d.jnext : d.knext};
      for (int side = 0; side < 2; ++side) {
        if (nbr[side] < 0) continue;
        const int q = T.P(nbr[side]);
        const int nAq = R.nax(q, ax);
        const int ga = side ? nA + 1 : 0;         // p's ghost plane
        const int a1 = side ? nA : 1, a2 = side ? nA - 1 : 2;  // p's first two layers inward
        const int qa = side ? 1 : nAq;            // q's layer next to p
        const int qa0 = side ? 1 : nAq - 1;       // the first of q's two layers next to p
        if (rdv[p] == rdv[q]) {
          for (int t = 0; t <= n2 + 1; ++t) for (int s = 0; s <= n1 + 1; ++s)
            ph.push_back({R.fcell(p, ax, ga, s, t), T.get(R.fcell(q, ax, qa, s, t))});
        } else if (rdv[p] > rdv[q]) {
          for (int t = 0; t <= n2 + 1; ++t) for (int s = 0; s <= n1 + 1; ++s) {
            const bool in = s >= 1 && s <= n1 && t >= 1 && t <= n2;
            const long long recv =
                in ? R.make(Terms{{T.get(R.fcell(q, ax, qa, (s + 1) / 2, (t + 1) / 2)), 2.0}}, 1.0) : kLmrZero;
            ph.push_back({R.fcell(p, ax, ga, s, t),
                          R.make(Terms{{recv, 1.0}, {T.get(R.fcell(p, ax, a1, s, t)), 3.0},
                                       {T.get(R.fcell(p, ax, a2, s, t)), -1.0}},
                                 0.25)});
          }
        } else {
          for (int t = 1; t <= n2; ++t) for (int s = 1; s <= n1; ++s) {
            Terms tt;
            for (int da = 0; da < 2; ++da) for (int dt = 0; dt < 2; ++dt) for (int ds = 0; ds < 2; ++ds)
              tt.push_back({T.get(R.fcell(q, ax, qa0 + da, 2 * s - 1 + ds, 2 * t - 1 + dt)), 1.0});
            ph.push_back({R.fcell(p, ax, ga, s, t), R.make(std::move(tt), 0.125)});
          }
        }
      }
      if (ax != 2) continue;
      // corners and edges, after the faces: prev corners #1..4, prev edges
      // #1..6, next corners, next edges (exchangepp.for:4433-4755)
      const int n3[3] = {geom[p].nx, geom[p].ny, geom[p].nz};
      auto ghost = [&](int e, int a, int m) { return e < 0 ? 0 : e > 0 ? n3[a] + 1 : m; };
      // the value p receives from q in direction D (p toward q); m: index
      // along an edge (0 for a corner); E = -D points from q toward p
      auto from = [&](int q, const int D[3], int m) -> long long {
        const int E[3] = {-D[0], -D[1], -D[2]};
        const int nq[3] = {R.nax(q, 0), R.nax(q, 1), R.nax(q, 2)};
        int c[3];
        if (rdv[p] == rdv[q]) {
          for (int a = 0; a < 3; ++a) c[a] = E[a] > 0 ? nq[a] : E[a] < 0 ? 1 : m;
          return T.get(T.id(q, c[0], c[1], c[2]));
        }
        if (rdv[q] > rdv[p]) {  // q finer: its 2x2x2 cells next to p
          int lo[3];
          for (int a = 0; a < 3; ++a) lo[a] = E[a] > 0 ? nq[a] - 1 : E[a] < 0 ? 1 : 2 * m - 1;
          Terms tt;
          for (int dk = 0; dk < 2; ++dk) for (int di = 0; di < 2; ++di) for (int dj = 0; dj < 2; ++dj)
            tt.push_back({T.get(T.id(q, lo[0] + di, lo[1] + dj, lo[2] + dk)), 1.0});
          return R.make(std::move(tt), 0.125);
        }
        // q coarser: from its cell next to p toward p; along an edge toward
        // the half of the coarse cell that holds p's cell m
        int o[3];
        for (int a = 0; a < 3; ++a) {
          c[a] = E[a] > 0 ? nq[a] : E[a] < 0 ? 1 : (m + 1) / 2;
          o[a] = E[a] != 0 ? E[a] : ((m & 1) ? -1 : +1);
        }
        Terms tt;
        for (int b = 0; b < 8; ++b) {
          const int oj = (b & 1) ? o[1] : 0, oi = (b & 2) ? o[0] : 0, ok = (b & 4) ? o[2] : 0;
          const int pc = ((b & 1) != 0) + ((b & 2) != 0) + ((b & 4) != 0);
          tt.push_back({T.get(T.id(q, c[0] + oi, c[1] + oj, c[2] + ok)), pc == 0 ? 27.0 : pc == 1 ? 9.0 : pc == 2 ? 3.0 : 1.0});
        }
        return R.make(std::move(tt), 1.0 / 64.0);
      };
      const int cp[4][2] = {{-1, -1}, {-1, +1}, {+1, +1}, {+1, -1}};
      const int cn[4][2] = {{+1, +1}, {+1, -1}, {-1, -1}, {-1, +1}};
      const int edp[6][3] = {{-1, 0, -1}, {0, +1, -1}, {+1, 0, -1}, {0, -1, -1}, {-1, -1, 0}, {-1, +1, 0}};
      const int edn[6][3] = {{+1, 0, +1}, {0, -1, +1}, {-1, 0, +1}, {0, +1, +1}, {+1, +1, 0}, {+1, -1, 0}};
      for (int side = 0; side < 2; ++side) {
        for (int c = 0; c < 4; ++c) {
          const int id = side ? d.cornext[c] : d.corprev[c];
          if (id < 0) continue;
          const int D[3] = {side ? cn[c][0] : cp[c][0], side ? cn[c][1] : cp[c][1], side ? +1 : -1};
          ph.push_back({T.id(p, ghost(D[0], 0, 0), ghost(D[1], 1, 0), ghost(D[2], 2, 0)), from(T.P(id), D, 0)});
        }
        for (int e = 0; e < 6; ++e) {
          const int id = side ? d.edgnext[e] : d.edgprev[e];
          if (id < 0) continue;
          const int *D = side ? edn[e] : edp[e];
          const int ax_e = D[0] == 0 ? 0 : D[1] == 0 ? 1 : 2;
          for (int m = 1; m <= n3[ax_e]; ++m)
            ph.push_back({T.id(p, ghost(D[0], 0, m), ghost(D[1], 1, m), ghost(D[2], 2, m)), from(T.P(id), D, m)});
        }
      }
    }
    for (auto &w : ph) T.set(w.first, w.second);
  }
  mgbound_tokens(T);
  if (periodic) exchbc_tokens(T);
  // the changed shell cells and the nodes they reach, ordered by depth
  std::vector<std::pair<long long, long long>> fin;  // (cell, token)
  for (int p : T.order) {
    const LevelGeom &G = geom[p];
    for (int k = 0; k <= G.nz + 1; ++k)
      for (int j = 0; j <= G.ny + 1; ++j)
        for (int i = 0; i <= G.nx + 1; ++i) {
          if (!TokenLevel::on_shell(G, i, j, k)) {
            i = G.nx;
            continue;
          }
          const long long c = T.id(p, i, j, k), v = T.shell[p][TokenLevel::sidx(G, i, j, k)];
          if (v != c) fin.push_back({c, v});
        }
  }
  const size_t nn = R.nodes.size();
  std::vector<int> depth(nn, 0);  // 0 = not reached
  // nodes only refer to earlier nodes, so one backward pass marks the reached
  // ones and a forward pass gives each its depth
  std::vector<char> reached(nn, 0);
  for (auto &f : fin)
    if (f.second <= -2) reached[(size_t)(-2 - f.second)] = 1;
  for (size_t n = nn; n-- > 0;)
    if (reached[n])
      for (auto &t : R.nodes[n].t)
        if (t.first <= -2) reached[(size_t)(-2 - t.first)] = 1;
  int dmax = 1;
  for (size_t n = 0; n < nn; ++n) {
    if (!reached[n]) continue;
    int dd = 1;
    for (auto &t : R.nodes[n].t)
      if (t.first <= -2) dd = std::max(dd, depth[(size_t)(-2 - t.first)] + 1);
    depth[n] = dd;
    dmax = std::max(dmax, dd);
  }
  LmrProgram out;
  // a copy of a cell the refresh does not write is applied directly with
  // the writes; a copy of one it writes becomes a one-term node of depth 1
  // (read before any write)
  std::vector<long long> dsts;
  for (auto &f : fin) dsts.push_back(f.first);
  std::sort(dsts.begin(), dsts.end());
  auto written = [&](long long c) { return std::binary_search(dsts.begin(), dsts.end(), c); };
  std::vector<long long> copy_of;
  for (auto &f : fin)
    if (f.second >= 0 && written(f.second)) copy_of.push_back(f.second);
  std::sort(copy_of.begin(), copy_of.end());
  copy_of.erase(std::unique(copy_of.begin(), copy_of.end()), copy_of.end());
  std::vector<int> newid(nn, -1);
  out.depth_start.push_back(0);
  for (int dd = 1; dd <= dmax; ++dd) {
    if (dd == 1)
      for (long long c : copy_of) {
        out.nodes.push_back(LmrProgram::Node{(int)out.terms.size(), 1, 1.0});
        out.terms.push_back(LmrProgram::Term{c, 1.0});
      }
    for (size_t n = 0; n < nn; ++n) {
      if (!reached[n] || depth[n] != dd) continue;
      newid[n] = (int)out.nodes.size();
      out.nodes.push_back(LmrProgram::Node{(int)out.terms.size(), (int)R.nodes[n].t.size(), R.nodes[n].scale});
      for (auto &t : R.nodes[n].t)
        out.terms.push_back(LmrProgram::Term{t.first <= -2 ? -2 - (long long)newid[(size_t)(-2 - t.first)] : t.first,
                                             t.second});
    }
    out.depth_start.push_back((int)out.nodes.size());
  }
  for (auto &f : fin) {
    if (f.second >= 0 && !written(f.second)) {
      out.copies.push_back({f.first, f.second});
      continue;
    }
    int node;
    if (f.second >= 0) node = (int)(std::lower_bound(copy_of.begin(), copy_of.end(), f.second) - copy_of.begin());
    else node = newid[(size_t)(-2 - f.second)];
    out.writes.push_back({f.first, node});
  }
  return out;
}

// ---------------------------------------------------------------------------
// Field exchange copy map.  exchange(op) (exchange.for:2-23) is exchange_bc
// on the periodic faces (exchange_bc.for:2-841) followed by exchange_smlvl
// (exchange.for:343-2498); for the pressure pbound follows (press.for:
// 77-137).  The sequence is replayed on tokens over the blocks' ttc arrays:
// a written cell remembers the id of the cell whose pre-exchange value it
// now holds.  Cells are numbered base[b] + (i-1) + ti*((j-1) + tj*(k-1))
// with 1-based field indices i = 1..ti.  Only written cells are stored.
// ---------------------------------------------------------------------------
namespace {

struct FieldTokens {
  const std::vector<mf3d_block_desc> &blk;
  const std::vector<long long> &base;
  int pl;
  std::vector<int> ti, tj, tk;
  std::unordered_map<int, int> pos;
  // Only ghost cells are written, so tokens are kept for the ghost region
  // of each block alone (pl-thick shell): z slabs, then per interior plane
  // the y rows, then per interior row the x ends.
  std::vector<std::vector<long long>> shell;
  FieldTokens(const std::vector<mf3d_block_desc> &b, const std::vector<long long> &bs, int pl_)
      : blk(b), base(bs), pl(pl_) {
    shell.resize(b.size());
    for (size_t q = 0; q < b.size(); ++q) {
      pos[b[q].id] = (int)q;
      ti.push_back(b[q].nx + 2 * pl);
      tj.push_back(b[q].ny + 2 * pl);
      tk.push_back(b[q].nz + 2 * pl);
      const long long W = ti[q], H = tj[q];
      shell[q].assign((size_t)(2 * pl * W * H + (long long)b[q].nz * (2 * pl * W + (long long)b[q].ny * 2 * pl)), -1);
    }
  }
  long long id(int p, int i, int j, int k) const {
    return base[p] + (i - 1) + (long long)ti[p] * ((j - 1) + (long long)tj[p] * (k - 1));
  }
  // index of a ghost cell in the shell, -1 for an interior cell
  long long sidx(int p, int i, int j, int k) const {
    const long long W = ti[p], H = tj[p];
    const int nx = ti[p] - 2 * pl, ny = tj[p] - 2 * pl, nz = tk[p] - 2 * pl;
    if (k <= pl) return ((long long)(k - 1) * H + (j - 1)) * W + (i - 1);
    if (k > nz + pl) return (pl * H + (long long)(k - nz - pl - 1) * H + (j - 1)) * W + (i - 1);
    long long o = 2 * pl * W * H + (long long)(k - pl - 1) * (2 * pl * W + (long long)ny * 2 * pl);
    if (j <= pl) return o + (long long)(j - 1) * W + (i - 1);
    if (j > ny + pl) return o + (long long)(pl + j - ny - pl - 1) * W + (i - 1);
    o += 2 * pl * W + (long long)(j - pl - 1) * 2 * pl;
    if (i <= pl) return o + (i - 1);
    if (i > nx + pl) return o + pl + (i - nx - pl - 1);
    return -1;
  }
  long long get(int p, int i, int j, int k) const {
    const long long s = sidx(p, i, j, k);
    if (s < 0) return id(p, i, j, k);
    const long long v = shell[p][(size_t)s];
    return v < 0 ? id(p, i, j, k) : v;
  }
  void set(int p, int i, int j, int k, long long v) {
    const long long s = sidx(p, i, j, k);
    if (s >= 0) shell[p][(size_t)s] = v;  // destinations are ghost cells
  }
  int P(int block_id) const {
    auto it = pos.find(block_id);
    return it == pos.end() ? -1 : it->second;
  }
};

// A field cell (block position, 1-based i, j, k).
struct FCell {
  int p, i, j, k;
};
// cell of block p at index a along axis ax and (s, t) along the others
FCell axis_cell(int p, int ax, int a, int s, int t) {
  if (ax == 0) return {p, a, s, t};
  if (ax == 1) return {p, s, a, t};
  return {p, s, t, a};
}

// Index ranges of the field: the pressure range spr..epr of every axis, and
// the field's own range lo..hi (velocities stop one face short of a high
// wall, localparameters.for:185-190).
struct FieldRange {
  int spr[3], epr[3], lo[3], hi[3], n[3];
};
FieldRange field_range(const mf3d_block_desc &d, int pl, int op) {
  FieldRange r;
  const int nn[3] = {d.nx, d.ny, d.nz};
  const int nbrn[3] = {d.inext, d.jnext, d.knext}, bcn[3] = {d.bc_east, d.bc_north, d.bc_top};
  for (int a = 0; a < 3; ++a) {
    r.n[a] = nn[a] + 2 * pl;
    r.spr[a] = pl + 1;
    r.epr[a] = nn[a] + pl;
    r.lo[a] = r.spr[a];
    r.hi[a] = r.epr[a];
    if (op == a + 1 && nbrn[a] < 0 && bcn[a] != MF3D_BC_PERIODIC) r.hi[a] -= 1;
  }
  return r;
}

// Directions of the corner and edge neighbours (x, y, z; 0 = the axis an
// edge runs along), in mf3d_block_desc's corprev/cornext/edgprev/edgnext order.
constexpr int kCP[4][3] = {{-1, -1, -1}, {-1, 1, -1}, {1, 1, -1}, {1, -1, -1}};
constexpr int kCN[4][3] = {{1, 1, 1}, {1, -1, 1}, {-1, -1, 1}, {-1, 1, 1}};
constexpr int kEP[6][3] = {{-1, 0, -1}, {0, 1, -1}, {1, 0, -1}, {0, -1, -1}, {-1, -1, 0}, {-1, 1, 0}};
constexpr int kEN[6][3] = {{1, 0, 1}, {0, -1, 1}, {-1, 0, 1}, {0, 1, 1}, {1, 1, 0}, {1, -1, 0}};

}  // namespace

std::vector<HaloPair> build_field_map(const std::vector<mf3d_block_desc> &blocks, const std::vector<long long> &base,
                                      int pl, int op, int nly, bool with_pbound) {
  FieldTokens T(blocks, base, pl);
  const int nb = (int)blocks.size();
  auto get = [&](const FCell &c) { return T.get(c.p, c.i, c.j, c.k); };
  auto set = [&](const FCell &c, long long v) { T.set(c.p, c.i, c.j, c.k, v); };
  std::vector<FieldRange> R(nb);
  bool periodic = false;
  for (int p = 0; p < nb; ++p) {
    R[p] = field_range(blocks[p], pl, op);
    const auto &d = blocks[p];
    periodic |= d.bc_west == 5 || d.bc_east == 5 || d.bc_south == 5 || d.bc_north == 5 || d.bc_bottom == 5 ||
                d.bc_top == 5;
  }
  // exchange_bc, all blocks on one rank: per layer two walks over the blocks
  // (a block alone along a periodic axis copies its own full ghost-inclusive
  // planes at once; other periodic faces pack into the partner's receive
  // plane, the second walk's pack replacing the first), then a walk that
  // unpacks the receive planes.
  if (periodic) {
    for (int ly = 0; ly <= nly; ++ly) {
      std::vector<std::vector<long long>> recv((size_t)nb * 6);
      auto bc_face = [&](int p, int f, bool unpack) {
        const auto &d = blocks[p];
        const int bcs[6] = {d.bc_west, d.bc_east, d.bc_south, d.bc_north, d.bc_bottom, d.bc_top};
        const int nbr[6] = {d.iprev, d.inext, d.jprev, d.jnext, d.kprev, d.knext};
        const int per[6] = {d.per_ip, d.per_in, d.per_jp, d.per_jn, d.per_kp, d.per_kn};
        if (!(bcs[f] == MF3D_BC_PERIODIC && nbr[f] < 0)) return;
        const int ax = f / 2;
        const bool high = f & 1, alone = nbr[f ^ 1] < 0;
        const FieldRange &r = R[p];
        const int n1 = ax == 0 ? r.n[1] : r.n[0], n2 = ax == 2 ? r.n[1] : r.n[2];
        const int ghost = high ? r.hi[ax] + 1 + ly : r.lo[ax] - 1 - ly;
        if (unpack) {
          if (alone) return;
          const auto &B = recv[(size_t)p * 6 + f];
          if (B.empty()) return;
          for (int t = 1; t <= n2; ++t)
            for (int s = 1; s <= n1; ++s) set(axis_cell(p, ax, ghost, s, t), B[(size_t)(t - 1) * n1 + (s - 1)]);
          return;
        }
        if (alone) {
          const int src = high ? r.lo[ax] + ly : r.hi[ax] - ly;
          for (int t = 1; t <= n2; ++t)
            for (int s = 1; s <= n1; ++s) set(axis_cell(p, ax, ghost, s, t), get(axis_cell(p, ax, src, s, t)));
          return;
        }
        const int q = T.P(per[f]);
        if (q < 0) return;
        // the partner's opposite face receives this face's plane
        auto &B = recv[(size_t)q * 6 + (f ^ 1)];
        B.assign((size_t)n1 * n2, 0);
        const int src = high ? r.hi[ax] - ly : r.lo[ax] + ly;
        for (int t = 1; t <= n2; ++t)
          for (int s = 1; s <= n1; ++s) B[(size_t)(t - 1) * n1 + (s - 1)] = get(axis_cell(p, ax, src, s, t));
      };
      for (int walk = 0; walk < 2; ++walk)
        for (int p = 0; p < nb; ++p)
          for (int f = 0; f < 6; ++f) bc_face(p, f, false);
      for (int p = 0; p < nb; ++p)
        for (int f = 0; f < 6; ++f) bc_face(p, f, true);
    }
  }
  // exchange_smlvl: per layer every block packs from the layer-start state
  // (faces: plane lo+ly / hi-ly of the field's range, whole ttc planes; for
  // ly = 0 also the (pl+1)^3 corner cubes and (pl+1)^2 x n edge bars, from
  // spr-1 or epr+1 inward); then each block unpacks its corners and edges
  // (cells outside the field's range in some axis) and last its faces (ghost
  // plane lo-1-ly / hi+1+ly, interior tangential range).  A phase reads the
  // state at its start, so every pair names its source token then.
  struct CP {
    FCell dst, src;
  };
  for (int ly = 0; ly <= nly; ++ly) {
    std::vector<CP> ph, faces;  // in unpack order; later pairs win
    for (int p = 0; p < nb; ++p) {
      const auto &d = blocks[p];
      const FieldRange &r = R[p];
      if (ly == 0) {
        auto ridx = [&](int ax, int dd, int m) { return dd < 0 ? r.spr[ax] - m : r.epr[ax] + m; };
        auto out = [&](int ax, int dd, int v) { return dd < 0 ? v < r.lo[ax] : v > r.hi[ax]; };
        for (int c = 0; c < 8; ++c) {
          const int *dir = c < 4 ? kCP[c] : kCN[c - 4];
          const int nbr = c < 4 ? d.corprev[c] : d.cornext[c - 4];
          if (nbr < 0) continue;
          const int q = T.P(nbr);
          if (q < 0) continue;
          const FieldRange &rq = R[q];
          // the sender sees this block on the opposite side: receiver spr-m <-> sender epr+1-m
          auto sidx = [&](int ax, int dd, int m) { return dd < 0 ? rq.epr[ax] + 1 - m : rq.spr[ax] - 1 + m; };
          for (int m1 = 0; m1 <= pl; ++m1)
            for (int m2 = 0; m2 <= pl; ++m2)
              for (int m3 = 0; m3 <= pl; ++m3) {
                const int i = ridx(0, dir[0], m1), j = ridx(1, dir[1], m2), k = ridx(2, dir[2], m3);
                if (out(0, dir[0], i) || out(1, dir[1], j) || out(2, dir[2], k))
                  ph.push_back({{p, i, j, k}, {q, sidx(0, dir[0], m1), sidx(1, dir[1], m2), sidx(2, dir[2], m3)}});
              }
        }
        for (int e = 0; e < 12; ++e) {
          const int *dir = e < 6 ? kEP[e] : kEN[e - 6];
          const int nbr = e < 6 ? d.edgprev[e] : d.edgnext[e - 6];
          if (nbr < 0) continue;
          const int q = T.P(nbr);
          if (q < 0) continue;
          const FieldRange &rq = R[q];
          auto sidx = [&](int ax, int dd, int m) { return dd < 0 ? rq.epr[ax] + 1 - m : rq.spr[ax] - 1 + m; };
          const int along = dir[0] == 0 ? 0 : dir[1] == 0 ? 1 : 2;
          const int ta = along == 0 ? 1 : 0, tb = along == 2 ? 1 : 2;
          for (int m1 = 0; m1 <= pl; ++m1)
            for (int m2 = 0; m2 <= pl; ++m2)
              for (int nn = r.spr[along]; nn <= r.epr[along]; ++nn) {
                int dst[3], src[3];
                dst[along] = src[along] = nn;
                dst[ta] = ridx(ta, dir[ta], m1);
                dst[tb] = ridx(tb, dir[tb], m2);
                if (!(out(ta, dir[ta], dst[ta]) || out(tb, dir[tb], dst[tb]))) continue;
                src[ta] = sidx(ta, dir[ta], m1);
                src[tb] = sidx(tb, dir[tb], m2);
                ph.push_back({{p, dst[0], dst[1], dst[2]}, {q, src[0], src[1], src[2]}});
              }
        }
      }
      const int nbr_p[3] = {d.iprev, d.jprev, d.kprev}, nbr_n[3] = {d.inext, d.jnext, d.knext};
      for (int ax = 0; ax < 3; ++ax) {
        const int ta = ax == 0 ? 1 : 0, tb = ax == 2 ? 1 : 2;
        for (int side = 0; side < 2; ++side) {
          const int nbr = side ? nbr_n[ax] : nbr_p[ax];
          if (nbr < 0) continue;
          const int q = T.P(nbr);
          if (q < 0) continue;
          const FieldRange &rq = R[q];
          const int g = side ? r.hi[ax] + 1 + ly : r.lo[ax] - 1 - ly;
          const int sa = side ? rq.lo[ax] + ly : rq.hi[ax] - ly;
          for (int t = r.spr[tb]; t <= r.epr[tb]; ++t)
            for (int s = r.spr[ta]; s <= r.epr[ta]; ++s)
              faces.push_back({axis_cell(p, ax, g, s, t), axis_cell(q, ax, sa, s, t)});
        }
      }
    }
    ph.insert(ph.end(), faces.begin(), faces.end());
    std::vector<long long> v(ph.size());
    for (size_t q = 0; q < ph.size(); ++q) v[q] = get(ph[q].src);
    for (size_t q = 0; q < ph.size(); ++q) set(ph[q].dst, v[q]);
  }
  // pbound: W, E, S, N, B, T on physical non-periodic faces, whole planes of
  // the ghost-inclusive range spr-1..epr+1, in order
  if (with_pbound) {
    for (int p = 0; p < nb; ++p) {
      const auto &d = blocks[p];
      const FieldRange &r = R[p];
      const int nbr[6] = {d.iprev, d.inext, d.jprev, d.jnext, d.kprev, d.knext};
      const int bcs[6] = {d.bc_west, d.bc_east, d.bc_south, d.bc_north, d.bc_bottom, d.bc_top};
      for (int f = 0; f < 6; ++f) {
        if (!(nbr[f] < 0 && bcs[f] != MF3D_BC_PERIODIC)) continue;
        const int ax = f / 2, ta = ax == 0 ? 1 : 0, tb = ax == 2 ? 1 : 2;
        const int g = (f & 1) ? r.epr[ax] + 1 : r.spr[ax] - 1, src = (f & 1) ? r.epr[ax] : r.spr[ax];
        for (int t = r.spr[tb] - 1; t <= r.epr[tb] + 1; ++t)
          for (int s = r.spr[ta] - 1; s <= r.epr[ta] + 1; ++s)
            set(axis_cell(p, ax, g, s, t), get(axis_cell(p, ax, src, s, t)));
      }
    }
  }
  // every ghost cell whose token changed, in increasing cell id
  std::vector<HaloPair> outp;
  for (int p = 0; p < nb; ++p)
    for (int k = 1; k <= T.tk[p]; ++k)
      for (int j = 1; j <= T.tj[p]; ++j)
        for (int i = 1; i <= T.ti[p]; ++i) {
          const long long si = T.sidx(p, i, j, k);
          if (si < 0) {  // skip the interior of the row
            i = T.ti[p] - pl;
            continue;
          }
          const long long v = T.shell[p][(size_t)si];
          if (v >= 0 && v != T.id(p, i, j, k)) outp.push_back({T.id(p, i, j, k), v});
        }
  return outp;
}

std::vector<double> level_widths(const double *ext, int n, double h, int ngrid, int g) {
  int W = 1 << (ngrid - 1);
  std::vector<double> e(n + 2 * W);
  for (int q = 0; q < n + 2 * W; ++q) e[q] = ext ? ext[q] : h;
  int Wg = W;
  for (int l = 2; l <= g; ++l) {
    std::vector<double> m(e.size() / 2);
    for (size_t q = 0; q < m.size(); ++q) m[q] = e[2 * q] + e[2 * q + 1];  // pairwise: exact for uniform
    e.swap(m);
    Wg /= 2;
  }
  int nl = n >> (g - 1);
  std::vector<double> w(nl + 2);
  for (int c = 0; c < nl + 2; ++c) w[c] = e[Wg - 1 + c];
  return w;
}

int face_rules(const std::vector<mf3d_block_desc> &blocks, std::vector<FaceRule> &rules) {
  std::unordered_map<int, int> pos;
  for (size_t q = 0; q < blocks.size(); ++q) pos[blocks[q].id] = (int)q;
  rules.assign(6 * blocks.size(), FaceRule{FACE_WALL, -1});
  for (size_t p = 0; p < blocks.size(); ++p) {
    const auto &d = blocks[p];
    const int nbr[6] = {d.iprev, d.inext, d.jprev, d.jnext, d.kprev, d.knext};
    const int bc[6] = {d.bc_west, d.bc_east, d.bc_south, d.bc_north, d.bc_bottom, d.bc_top};
    const int per[6] = {d.per_ip, d.per_in, d.per_jp, d.per_jn, d.per_kp, d.per_kn};
    for (int f = 0; f < 6; ++f) {
      FaceRule r{FACE_WALL, -1};
      if (nbr[f] >= 0) {
        r = {FACE_NEIGHBOUR, pos.count(nbr[f]) ? pos[nbr[f]] : -1};
      } else if (bc[f] == MF3D_BC_PERIODIC) {
        int other = nbr[f ^ 1];
        if (other < 0) r = {FACE_NEIGHBOUR, (int)p};  // alone along the axis: wrap onto itself
        else r = {FACE_NEIGHBOUR, (per[f] >= 0 && pos.count(per[f])) ? pos[per[f]] : -1};
      }
      if (r.kind == FACE_NEIGHBOUR && r.src < 0) {
        set_error("block " + std::to_string(d.id) + ": face neighbour or periodic partner not found");
        return MF3D_E_INVALID;
      }
      rules[6 * p + f] = r;
    }
  }
  return MF3D_OK;
}

}  // namespace mf3d
