// Internal host-side structures of libmf3d (not part of the C ABI).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mf3d.h"

namespace mf3d {

void set_error(const std::string &msg);

// Index geometry of one block at one multigrid level: interior n*, ghost
// shell of one cell, 0-based ghost-inclusive indices 0..n+1.
struct LevelGeom {
  int nx, ny, nz;
  long long cells() const { return (long long)(nx + 2) * (ny + 2) * (nz + 2); }
  long long lin(int i, int j, int k) const {
    return ((long long)k * (ny + 2) + j) * (nx + 2) + i;
  }
};

// A halo copy: destination cell <- source cell, as level-wide cell ids
// (block base + lin(i,j,k)).
struct HaloPair {
  long long dst, src;
};

// Composition of exchangepp + mgbound + exchbc_mgpp for one level
// (exchangepp.for:43-4763, mgsolver.for:907-992, exchangepp.for:4768-5383)
// expressed as pairs dst <- src against the state before the exchange.
// `base[b]` is the level-wide id of cell (0,0,0) of block b.
std::vector<HaloPair> build_halo_map(const std::vector<mf3d_block_desc> &blocks,
                                     const std::vector<LevelGeom> &geom,
                                     const std::vector<long long> &base);

// The same refresh on a level where blocks of different refinement meet
// (LMR, rdv differing across an interface; exchangepp.for:43-4763).  The
// values are no longer copies: a refined block's ghosts next to a coarser
// neighbour are (2 phi_coarse + 3 phi_1 - phi_2) / 4, a coarser block's the
// 8-cell averages of the refined neighbour, corner and edge ghosts of a
// refined block trilinear blends of the coarser one's cells.  The map is
// a program over the state before the exchange: nodes, each a sum
// w_0 x_0 + w_1 x_1 + ... (in that order, the reference's order) times
// `scale`, whose terms are cells or earlier nodes, evaluated in order of
// depth; then every changed ghost cell takes its node's value, or the value
// of the cell it copies where no write touches that cell.  `rdv` is
// rdv(block, g) of each block at this level (localparameters.for:47-57).
struct LmrProgram {
  struct Term {
    long long ref;  // >= 0: cell id; kLmrZero: the constant 0; <= -2: node (-2 - ref)
    double w;
  };
  struct Node {
    int t0, nt;     // terms [t0, t0 + nt)
    double scale;
  };
  std::vector<Term> terms;
  std::vector<Node> nodes;                        // in order of depth
  std::vector<int> depth_start;                   // nodes of depth d: [depth_start[d-1], depth_start[d])
  std::vector<std::pair<long long, int>> writes;  // ghost cell id <- node
  std::vector<std::pair<long long, long long>> copies;  // ghost cell id <- a cell no write touches
};
constexpr long long kLmrZero = -1;
LmrProgram build_halo_lmr(const std::vector<mf3d_block_desc> &blocks, const std::vector<LevelGeom> &geom,
                          const std::vector<long long> &base, const std::vector<int> &rdv);

// exchange(op) on field arrays (exchange.for:2-23: exchange_bc on the
// periodic faces, then exchange_smlvl with its corners, edges and faces),
// and pbound after it when `with_pbound` (press.for:77-137), as pairs
// dst <- src against the state before the exchange.  op 1, 2, 3: u, v, w
// (their index ranges), 4: p; nly: the layers exchanged (pl_ex, 0 for p).
// Cell id = base[b] + (i-1) + ti*((j-1) + tj*(k-1)), 1-based field indices.
std::vector<HaloPair> build_field_map(const std::vector<mf3d_block_desc> &blocks, const std::vector<long long> &base,
                                      int pl, int op, int nly, bool with_pbound);

// Neighbour search of alloc_dom.for:456-1150 over block extents.
int build_topology(int nblocks, const double *ext, const int *bc6, double dx,
                   double dy, double dz, mf3d_block_desc *out);

// Level-g cell widths of one axis, ghost-inclusive (n_g + 2 entries), from
// the block's extended fine widths (NULL = uniform h); see mf3d_block_desc.
std::vector<double> level_widths(const double *ext, int n, double h, int ngrid, int g);

// Face-ghost rule of one block face for the pressure field and the low-face
// velocity: which block supplies the value.
enum FaceKind { FACE_NEIGHBOUR = 0, FACE_WALL = 1 };
struct FaceRule {
  int kind;   // FACE_NEIGHBOUR (neighbour, periodic partner or self) / FACE_WALL
  int src;    // position of the source block (valid for FACE_NEIGHBOUR)
};
// rules[6*b + f], f = W,E,S,N,B,T.  Returns MF3D_OK or an error.
int face_rules(const std::vector<mf3d_block_desc> &blocks, std::vector<FaceRule> &rules);

}  // namespace mf3d
