// Task plan of the dataflow Gauss-Jordan inverse (k_gj_flow, topx_gjflow.cu).
//
// The blocked Gauss-Jordan exchange on 64-wide pivot blocks is cut into tile tasks per
// step k (pivot block K = k, tiles of 64 x 64):
//   PIV(k)      P^-1 of the diagonal tile (k, k)
//   PAN(k, j)   R_j = -P^-1 A[K, j]            (row panel; also written into A[K, j])
//   COL(k, i)   C_i = A[i, K] kept, A[i, K] = C_i P^-1
//   UPD(k,i,j)  A[i, j] += C_i R_j             (i, j != K)
// The chain from one pivot to the next is one task: PIV(k) for k >= 1 first does
// COL(k-1, k), PAN(k-1, k) and UPD(k-1, k, k), so the next diagonal tile goes from the
// tensor-core accumulators straight into its inversion.
// P^-1, R and C live in a ring of GF_RING step slots per matrix.  Every tile carries a
// version (steps applied to it); a task waits for the versions it reads, and PIV(k) also
// waits until all of step k - GF_RING's updates are done before it reuses that ring slot.
//
// Tasks are numbered in one global order (the tickets CTAs claim).  The order is
// topological: every dependency of a task has a smaller ticket, so the lowest unfinished
// ticket can always run and the kernel cannot deadlock however many CTAs are resident.
// The order is by "deadline": the first pivot that transitively needs a task's result.  A
// tile (i, j) updated at step k with i, j > k is needed by PIV(max(i, j)); a panel PAN(k, j)
// by PIV(j), a column COL(k, i) by PIV(i); tiles in rows or columns already pivoted are never
// read by a later pivot.  Every task of step k is due before PIV(k + GF_RING) (ring reuse).
// PIV(k) is keyed as a task of step k - 1 (the step whose critical tiles it computes).
#pragma once

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <vector>

#if defined(__CUDACC__)
#define TOPX_GF_HD __host__ __device__
#else
#define TOPX_GF_HD
#endif

namespace topx {

constexpr int GF_T = 64;    // tile (= pivot block) width
constexpr int GF_RING = 4;  // ring slots of (P^-1, R, C) per matrix
constexpr int GF_MAX_NT = 64;  // tiles per matrix side (m <= 4096)

enum GFType : uint32_t { GF_PIV = 0, GF_PAN = 1, GF_COL = 2, GF_UPD = 3 };

// code: j | i << 7 | k << 14 | mat << 21 | type << 22
inline uint32_t gf_code(uint32_t type, uint32_t mat, uint32_t k, uint32_t i, uint32_t j) {
  return j | (i << 7) | (k << 14) | (mat << 21) | (type << 22);
}
TOPX_GF_HD inline void gf_decode(uint32_t c, int& type, int& mat, int& k, int& i, int& j) {
  j = int(c & 127u);
  i = int((c >> 7) & 127u);
  k = int((c >> 14) & 127u);
  mat = int((c >> 21) & 1u);
  type = int((c >> 22) & 3u);
}

inline int gf_tiles(int m) { return (m + GF_T - 1) / GF_T; }

// control words: [0] error flag, [1] ticket, then per matrix: nt*nt tile versions, nt update
// counts per step, nt "C of row block k is in the ring" flags
constexpr int GF_CTRL_HEAD = 32;
inline size_t gf_ctrl_words(int m) {
  const size_t nt = size_t(gf_tiles(m));
  return GF_CTRL_HEAD + 2 * (nt * nt + 2 * nt);
}
// ring scratch per matrix: GF_RING slots of P^-1, nt R tiles and nt C tiles (64 x 64 each)
TOPX_GF_HD inline size_t gf_slot_doubles(int m) { return size_t(1 + 2 * ((m + GF_T - 1) / GF_T)) * GF_T * GF_T; }
inline size_t gf_scratch_doubles(int m) { return 2 * size_t(GF_RING) * gf_slot_doubles(m); }

// deadline key of a task (see the header comment)
inline int gf_deadline(int type, int nt, int k, int i, int j) {
  const int ring = k + GF_RING;
  switch (type) {
    case GF_PIV:
      return k;
    case GF_PAN:
      return j > k ? std::min(j, ring) : ring;
    case GF_COL:
      return i > k ? std::min(i, ring) : ring;
    default:
      return (i > k && j > k) ? std::min(std::max(i, j), ring) : ring;
  }
  (void)nt;
}

// The ticket order for `nset` (1 or 2) matrices of order m.
inline std::vector<uint32_t> gf_plan(int m, int nset) {
  const int nt = gf_tiles(m);
  if (nt > GF_MAX_NT) throw std::runtime_error("gj plan: matrix too large");
  struct Item {
    uint64_t key;
    uint32_t code;
  };
  std::vector<Item> items;
  items.reserve(size_t(nset) * nt * (size_t(nt) * nt + 1));
  auto add = [&](int type, int mat, int k, int i, int j) {
    const int rank = type == GF_PIV ? 0 : type == GF_UPD ? 2 : 1;
    const int kstep = (type == GF_PIV && k > 0) ? k - 1 : k;
    const uint64_t key = (uint64_t(gf_deadline(type, nt, k, i, j)) << 40) | (uint64_t(kstep) << 32) |
                         (uint64_t(rank) << 24) | (uint64_t(mat) << 16) | (uint64_t(i) << 8) | uint64_t(j);
    items.push_back(Item{key, gf_code(uint32_t(type), uint32_t(mat), uint32_t(k), uint32_t(i), uint32_t(j))});
  };
  for (int mat = 0; mat < nset; ++mat)
    for (int k = 0; k < nt; ++k) {
      add(GF_PIV, mat, k, k, k);
      for (int j = 0; j < nt; ++j)
        if (j != k && j != k + 1) add(GF_PAN, mat, k, k, j);  // PAN(k, k+1) is part of PIV(k+1)
      for (int i = 0; i < nt; ++i)
        if (i != k && i != k + 1) add(GF_COL, mat, k, i, k);  // COL(k, k+1) too
      for (int i = 0; i < nt; ++i)
        for (int j = 0; j < nt; ++j)
          if (i != k && j != k && !(i == k + 1 && j == k + 1)) add(GF_UPD, mat, k, i, j);
    }
  std::sort(items.begin(), items.end(), [](const Item& a, const Item& b) { return a.key < b.key; });
  std::vector<uint32_t> out(items.size());
  for (size_t t = 0; t < items.size(); ++t) out[t] = items[t].code;
  return out;
}

// Checks that every dependency of every task has a smaller ticket (throws otherwise).
inline void gf_check_plan(const std::vector<uint32_t>& plan, int m, int nset) {
  const int nt = gf_tiles(m);
  // ticket of each task: index [mat][k][i][j] (PIV at (k,k), PAN at (k,j), COL at (i,k))
  const size_t per = size_t(nt) * nt * nt;
  std::vector<int64_t> tk(size_t(nset) * per, -1);
  auto at = [&](int mat, int k, int i, int j) -> int64_t& { return tk[size_t(mat) * per + (size_t(k) * nt + i) * nt + j]; };
  for (size_t t = 0; t < plan.size(); ++t) {
    int type, mat, k, i, j;
    gf_decode(plan[t], type, mat, k, i, j);
    at(mat, k, i, j) = int64_t(t);
  }
  std::vector<int64_t> last_upd(size_t(nset) * nt, -1);
  for (size_t t = 0; t < plan.size(); ++t) {
    int type, mat, k, i, j;
    gf_decode(plan[t], type, mat, k, i, j);
    if (type == GF_UPD) last_upd[size_t(mat) * nt + k] = std::max(last_upd[size_t(mat) * nt + k], int64_t(t));
    if (type == GF_PIV && k > 0) {  // PIV(k) carries COL(k-1, k), PAN(k-1, k) and UPD(k-1, k, k)
      at(mat, k - 1, k, k - 1) = at(mat, k - 1, k - 1, k) = at(mat, k - 1, k, k) = int64_t(t);
      last_upd[size_t(mat) * nt + k - 1] = std::max(last_upd[size_t(mat) * nt + k - 1], int64_t(t));
    }
  }
  auto need = [&](int64_t dep, size_t t) {
    if (dep < 0 || dep >= int64_t(t)) throw std::runtime_error("gj plan: dependency not ordered before its task");
  };
  for (size_t t = 0; t < plan.size(); ++t) {
    int type, mat, k, i, j;
    gf_decode(plan[t], type, mat, k, i, j);
    if (type == GF_PIV) {
      if (k > 0) {
        need(at(mat, k - 1, k - 1, k - 1), t);  // the previous pivot
        if (k > 1) {                             // the three tiles' writers at step k-2
          need(at(mat, k - 2, k, k - 1), t);
          need(at(mat, k - 2, k - 1, k), t);
          need(at(mat, k - 2, k, k), t);
        }
      }
      if (k >= GF_RING && nt > 1) need(last_upd[size_t(mat) * nt + k - GF_RING], t);
    } else {
      need(at(mat, k, k, k), t);  // the step's pivot
      if (type == GF_UPD) {
        need(at(mat, k, k, j), t);
        need(at(mat, k, i, k), t);
      }
      if (k > 0) need(at(mat, k - 1, i, j), t);  // the tile's writer at step k-1
    }
  }
}

}  // namespace topx
