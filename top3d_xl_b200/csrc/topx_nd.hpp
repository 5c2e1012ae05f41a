// Nested-dissection multifrontal factorisation of the coarsest-level matrix (the reference
// factors it with chol(K,'lower') and a fill-reducing permutation, TOP3D_XL.m:1052-1065, and
// applies the factor in every V-cycle, TOP3D_XL.m:767).
//
// The coarsest node grid is cut recursively along its longest axis by node planes (the
// separators) until the boxes are small; a box's separator, or a leaf box's nodes, is the
// front that eliminates them.  A front's matrix couples its eliminated DOFs (n1) with the DOFs
// of the nodes around its box (n2, all on ancestor separators).  It is assembled from the
// element operators and the children's Schur complements (extend-add), then swept by blocked
// Gauss-Jordan exchange on its first n1 columns, which leaves
//     [ F11^-1            .              ]
//     [ X = F21 F11^-1    S = F22 - X F12 ]
// so that a solve is, per tree level, f2 -= X f1 and v1 = F11^-1 f1 on the way up and
// x1 = v1 - X^T x2 on the way down: dense GEMVs with no dependent chain inside a front.
// Matrices are stored as 64 x 64 tiles (lower triangle of tiles, each tile full and row-major),
// FP64, swept on the tensor cores (mma.sync m8n8k4).
#pragma once

#include <cstdint>
#include <vector>

namespace topx {

constexpr int ND_T = 64;      // tile width
constexpr int ND_CHUNK = 4;   // tiles a solve CTA streams for one output tile (more: several CTAs)
constexpr int64_t kNdOneFrontNodes = 320;  // coarsest grids with at most this many nodes: one front
constexpr int64_t ND_MEDIUM_NODES = 2048;  // grids up to this size: leaves of ND_MEDIUM_LEAF nodes
constexpr int ND_MEDIUM_LEAF = 256, ND_LEAF = 128;

// One front of the elimination tree (device descriptor).  Positions 0 .. n1-1 are the
// eliminated DOFs (3 per separator node, in node order), n1 .. 64 T1 - 1 padding (identity),
// 64 T1 .. 64 T1 + n2 - 1 the update DOFs (3 per node around the box), then padding (zero).
struct NDFront {
  int64_t tile0;  // first tile in the tile pool: tile (i, j), i >= j, is tile0 + i (i + 1) / 2 + j
  int64_t pos0;   // first entry in the per-position arrays and the solve vectors (64 N entries)
  int64_t map0;   // first entry of its update-DOF -> parent-position map (n2 entries)
  int N, T1;      // tiles per side; leading tiles of eliminated DOFs
  int n1, n2;     // eliminated and update DOFs
  int parent;     // front index, -1 for a root
  int scr0;       // first scratch tile while its level is swept: P^-1, then R_0 .. R_{N-1} of
                  // even steps and R_0 .. R_{N-1} of odd steps
  // dataflow solve: output tiles its children complete on the way up before its forward tasks
  // may start (the sum of their N); and before its backward tasks may start, the solution tiles
  // (bwd_need = its T1) of bwd_front, the nearest ancestor that eliminates DOFs (-1: none, need 0).
  // Fronts between the two eliminate nothing, so that ancestor's solution implies all of theirs.
  int fwd_need, bwd_need, bwd_front;
};

// A launch task: front f, tile row i, tile column j.
struct NDTask {
  int32_t f;
  int16_t i, j;
};

// An assembly entry: the 3 x 3 block K[a][b] of grid nodes a (a separator node of front f, at
// node position pa) and b (at node position pb of the same front).
struct NDAsm {
  int32_t f, pa, pb, a, b;
};

struct NDLevel {
  std::vector<int> fronts;
  int maxT1 = 0;
  int64_t pos_begin = 0, pos_end = 0;  // positions of its fronts (contiguous)
  // sweep: the pivots of step 0 [piv0[0], piv0[1]); per step k, panels [s[4k], s[4k+1]) with the
  // write-back of step k-1 [s[4k+1], s[4k+2]) in one launch, then the updates [s[4k+2], s[4k+3])
  // (the pivot of step k+1 runs inside the update of its diagonal tile); the write-back of the
  // last step [fin_last[0], fin_last[1])
  int64_t piv0[2] = {0, 0};
  std::vector<int64_t> step;
  int64_t fin_last[2] = {0, 0};
  // extend-add tasks into this level's fronts, from their children of slot 0 and slot 1
  int64_t ext[3] = {0, 0, 0};
  // solve tasks (front f, output tile i, chunk j of ND_CHUNK input tiles), the chunks of one
  // output tile consecutive
  int64_t fwd[2] = {0, 0}, bwd[2] = {0, 0};
  int nscr = 0;                              // scratch tiles the level's sweep uses
};

struct NDPlan {
  std::vector<NDFront> fronts;
  std::vector<int> child_slot;          // per front: 0 or 1, its index among its parent's children
  std::vector<NDLevel> levels;          // by tree depth (0: roots); swept from the deepest up
  std::vector<NDAsm> asmb;              // assembly entries (writes of the original matrix)
  std::vector<int64_t> pad_diag;        // pool offsets of padding diagonal entries (set to 1)
  std::vector<int32_t> upd_map;         // update DOF k of front f -> position in its parent (map0 + k)
  std::vector<int32_t> sep_dof;         // per position: grid DOF (node + c * stride) of an eliminated DOF, else -1
  std::vector<int32_t> upd_dof;         // per position: grid DOF of an update DOF, else -1
  std::vector<int32_t> src[2];          // per position: solve-vector index of child slot 0 / 1's update
                                        // entry that lands here, else -1
  std::vector<NDTask> tasks;
  // the solve's tasks in dependency order for a dataflow launch: the forward tasks level by level
  // from the leaves up (the first flow_fwd entries), then the backward tasks from the root down;
  // a task depends only on tasks before it
  std::vector<NDTask> flow;
  int64_t flow_fwd = 0;
  int64_t ntiles = 0, npos = 0;
  int64_t nsolve_tasks = 0;             // upper bound of the solve tasks of one launch (partial sums)
  int nscr = 0;                         // scratch tiles (max over levels)
  int max_n1 = 0, max_n2 = 0;
  int max_t1 = 0, max_t2 = 0;           // most tiles of eliminated / update DOFs in one front
  double flops = 0;                     // sweep FLOPs (tile products) per factorisation
};

// Plan for a grid of nny x nnx x nnz nodes (y fastest), node present flags, and the stride of
// the SoA DOF vectors (component c of node n at n + c * stride).  Leaf boxes hold at most
// `leaf_nodes` grid nodes.
NDPlan nd_plan(int nny, int nnx, int nnz, int64_t stride, const std::vector<uint8_t>& present, int leaf_nodes = 64);

// Leaf size of the tree for a coarsest grid of `present` nodes: each tree level costs the solve a
// dependent phase, each larger leaf the factorisation its cube; medium grids take fewer levels.
inline int nd_leaf_nodes(int64_t present) { return present <= ND_MEDIUM_NODES ? ND_MEDIUM_LEAF : ND_LEAF; }

// Consistency checks of a plan (positions, maps, task ranges); throws on the first violation.
void nd_check_plan(const NDPlan& p);

}  // namespace topx
