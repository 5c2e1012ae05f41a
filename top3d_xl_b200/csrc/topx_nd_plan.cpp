// Host planning of the nested-dissection multifrontal factorisation (topx_nd.hpp): the
// elimination tree of the coarsest node grid, front sizes and storage, assembly entries,
// extend-add maps and the task lists of every launch.  Depends only on the grid and on which
// nodes are present, so it is built once per engine.
#include <algorithm>
#include <stdexcept>
#include <string>

#include "topx_nd.hpp"

namespace topx {
namespace {

struct Box {
  int lo[3], hi[3];  // node coordinates [lo, hi) per axis (0: y, 1: x, 2: z)
};

struct HostFront {
  Box box;
  int parent, depth, slot;
  int child[2];
  std::vector<int32_t> sep, halo;  // grid node ids, ascending
};

struct Builder {
  int dim[3];
  const std::vector<uint8_t>& present;
  int leaf;
  std::vector<HostFront> fr;

  Builder(int ny, int nx, int nz, const std::vector<uint8_t>& pr, int lf) : present(pr), leaf(lf) {
    dim[0] = ny;
    dim[1] = nx;
    dim[2] = nz;
  }
  int64_t node(const int c[3]) const { return c[0] + int64_t(dim[0]) * (c[1] + int64_t(dim[1]) * c[2]); }

  template <typename Fn>
  void for_nodes(const Box& b, Fn&& fn) const {  // ascending grid id order
    int c[3];
    for (c[2] = b.lo[2]; c[2] < b.hi[2]; ++c[2])
      for (c[1] = b.lo[1]; c[1] < b.hi[1]; ++c[1])
        for (c[0] = b.lo[0]; c[0] < b.hi[0]; ++c[0]) fn(c, node(c));
  }

  int build(const Box& b, int parent, int depth, int slot) {
    int64_t vol = 1;
    for (int a = 0; a < 3; ++a) vol *= std::max(0, b.hi[a] - b.lo[a]);
    if (vol == 0) return -1;
    int64_t cnt = 0;
    for_nodes(b, [&](const int*, int64_t n) { cnt += present[size_t(n)] ? 1 : 0; });
    if (cnt == 0) return -1;
    const int id = int(fr.size());
    fr.push_back(HostFront{b, parent, depth, slot, {-1, -1}, {}, {}});
    if (vol <= leaf) {
      std::vector<int32_t> sep;
      for_nodes(b, [&](const int*, int64_t n) {
        if (present[size_t(n)]) sep.push_back(int32_t(n));
      });
      fr[size_t(id)].sep = std::move(sep);
    } else {
      int ax = 0;  // longest axis (the last of equals: z, then x, then y)
      for (int a = 1; a < 3; ++a)
        if (b.hi[a] - b.lo[a] >= b.hi[ax] - b.lo[ax]) ax = a;
      const int mid = (b.lo[ax] + b.hi[ax]) / 2;
      Box plane = b, c0 = b, c1 = b;
      plane.lo[ax] = mid;
      plane.hi[ax] = mid + 1;
      c0.hi[ax] = mid;
      c1.lo[ax] = mid + 1;
      std::vector<int32_t> sep;
      for_nodes(plane, [&](const int*, int64_t n) {
        if (present[size_t(n)]) sep.push_back(int32_t(n));
      });
      fr[size_t(id)].sep = std::move(sep);
      const int k0 = build(c0, id, depth + 1, 0);
      const int k1 = build(c1, id, depth + 1, 1);
      fr[size_t(id)].child[0] = k0;
      fr[size_t(id)].child[1] = k1;
    }
    // the present nodes around the box: all of them lie on ancestor separators
    Box h = b;
    for (int a = 0; a < 3; ++a) {
      h.lo[a] = std::max(0, b.lo[a] - 1);
      h.hi[a] = std::min(dim[a], b.hi[a] + 1);
    }
    std::vector<int32_t> halo;
    for_nodes(h, [&](const int* c, int64_t n) {
      bool inside = true;
      for (int a = 0; a < 3; ++a) inside = inside && c[a] >= b.lo[a] && c[a] < b.hi[a];
      if (!inside && present[size_t(n)]) halo.push_back(int32_t(n));
    });
    fr[size_t(id)].halo = std::move(halo);
    return id;
  }
};

inline int tiles_of(int n) { return (n + ND_T - 1) / ND_T; }
inline int64_t tri(int64_t i) { return i * (i + 1) / 2; }

}  // namespace

NDPlan nd_plan(int nny, int nnx, int nnz, int64_t stride, const std::vector<uint8_t>& present, int leaf_nodes) {
  if (int64_t(present.size()) != int64_t(nny) * nnx * nnz) throw std::invalid_argument("nd_plan: present size");
  if (stride * 3 > int64_t(INT32_MAX)) throw std::invalid_argument("nd_plan: grid too large");
  // a small grid is one front: its solve is then a single GEMV with no dependent phases
  int64_t npresent = 0;
  for (uint8_t v : present) npresent += v ? 1 : 0;
  const int64_t leaf = npresent <= kNdOneFrontNodes ? int64_t(nny) * nnx * nnz : std::max(8, leaf_nodes);
  Builder B(nny, nnx, nnz, present, int(std::min<int64_t>(leaf, INT32_MAX)));
  Box all{{0, 0, 0}, {nny, nnx, nnz}};
  B.build(all, -1, 0, 0);
  NDPlan P;
  const int nf = int(B.fr.size());
  if (nf == 0) throw std::invalid_argument("nd_plan: no present node");
  int depth = 0;
  for (const auto& f : B.fr) depth = std::max(depth, f.depth + 1);
  P.levels.resize(size_t(depth));
  for (int i = 0; i < nf; ++i) P.levels[size_t(B.fr[size_t(i)].depth)].fronts.push_back(i);
  // sizes, storage and positions (level by level, so a level's positions are contiguous)
  P.fronts.resize(size_t(nf));
  P.child_slot.resize(size_t(nf));
  int64_t tiles = 0, pos = 0, map = 0;
  for (auto& L : P.levels) {
    L.pos_begin = pos;
    int scr = 0;
    for (int f : L.fronts) {
      const HostFront& h = B.fr[size_t(f)];
      NDFront& d = P.fronts[size_t(f)];
      d.n1 = 3 * int(h.sep.size());
      d.n2 = 3 * int(h.halo.size());
      d.T1 = tiles_of(d.n1);
      d.N = d.T1 + tiles_of(d.n2);
      d.parent = h.parent;
      d.tile0 = tiles;
      d.pos0 = pos;
      d.map0 = map;
      d.scr0 = scr;
      tiles += tri(d.N);
      pos += int64_t(ND_T) * d.N;
      map += d.n2;
      scr += 2 * d.N + 1;
      L.maxT1 = std::max(L.maxT1, d.T1);
      P.max_n1 = std::max(P.max_n1, d.n1);
      P.max_n2 = std::max(P.max_n2, d.n2);
      P.max_t1 = std::max(P.max_t1, d.T1);
      P.max_t2 = std::max(P.max_t2, d.N - d.T1);
      P.child_slot[size_t(f)] = h.slot;
      d.fwd_need = 0;
      d.bwd_need = 0;
      d.bwd_front = -1;
    }
    L.pos_end = pos;
    L.nscr = scr;
    P.nscr = std::max(P.nscr, scr);
  }
  P.ntiles = tiles;
  P.npos = pos;
  for (int f = 0; f < nf; ++f) {
    NDFront& d = P.fronts[size_t(f)];
    if (d.parent >= 0) P.fronts[size_t(d.parent)].fwd_need += d.N;
    int a = d.parent;
    while (a >= 0 && P.fronts[size_t(a)].T1 == 0) a = P.fronts[size_t(a)].parent;
    d.bwd_front = a;
    d.bwd_need = a >= 0 ? P.fronts[size_t(a)].T1 : 0;
  }
  P.upd_map.assign(size_t(map), -1);
  P.sep_dof.assign(size_t(pos), -1);
  P.upd_dof.assign(size_t(pos), -1);
  P.src[0].assign(size_t(pos), -1);
  P.src[1].assign(size_t(pos), -1);
  // node -> position of the front whose table is current
  std::vector<int32_t> posof(present.size(), 0), stamp(present.size(), -1);
  auto set_table = [&](int f) {
    const HostFront& h = B.fr[size_t(f)];
    const NDFront& d = P.fronts[size_t(f)];
    for (size_t s = 0; s < h.sep.size(); ++s) {
      posof[size_t(h.sep[s])] = int32_t(3 * s);
      stamp[size_t(h.sep[s])] = f;
    }
    for (size_t u = 0; u < h.halo.size(); ++u) {
      posof[size_t(h.halo[u])] = int32_t(ND_T * d.T1 + 3 * int64_t(u));
      stamp[size_t(h.halo[u])] = f;
    }
  };
  const int dims[3] = {nny, nnx, nnz};
  for (int f = 0; f < nf; ++f) {
    const HostFront& h = B.fr[size_t(f)];
    const NDFront& d = P.fronts[size_t(f)];
    const int64_t P1 = int64_t(ND_T) * d.T1;
    set_table(f);
    for (size_t s = 0; s < h.sep.size(); ++s)
      for (int c = 0; c < 3; ++c) P.sep_dof[size_t(d.pos0 + 3 * int64_t(s) + c)] = int32_t(h.sep[s] + c * stride);
    for (size_t u = 0; u < h.halo.size(); ++u)
      for (int c = 0; c < 3; ++c)
        P.upd_dof[size_t(d.pos0 + P1 + 3 * int64_t(u) + c)] = int32_t(h.halo[u] + c * stride);
    for (int64_t p = d.n1; p < P1; ++p) {
      const int64_t t = p / ND_T, r = p % ND_T;
      P.pad_diag.push_back((d.tile0 + tri(t) + t) * ND_T * ND_T + r * ND_T + r);
    }
    // assembly: blocks of the separator rows with the front's own nodes (the pairs of separator
    // nodes once, the node's own block included)
    for (size_t s = 0; s < h.sep.size(); ++s) {
      const int32_t a = h.sep[s];
      int ca[3] = {int(a % nny), int((a / nny) % nnx), int(a / (int64_t(nny) * nnx))};
      for (int dz = -1; dz <= 1; ++dz)
        for (int dx = -1; dx <= 1; ++dx)
          for (int dy = -1; dy <= 1; ++dy) {
            const int cb[3] = {ca[0] + dy, ca[1] + dx, ca[2] + dz};
            bool in = true;
            for (int q = 0; q < 3; ++q) in = in && cb[q] >= 0 && cb[q] < dims[q];
            if (!in) continue;
            const int64_t b = cb[0] + int64_t(nny) * (cb[1] + int64_t(nnx) * cb[2]);
            if (!present[size_t(b)] || stamp[size_t(b)] != f) continue;  // void, or in a child's box
            const int32_t pb = posof[size_t(b)], pa = int32_t(3 * s);
            if (pb < P1 && pb > pa) continue;  // the other node of the pair writes it
            P.asmb.push_back(NDAsm{f, pa, pb, a, int32_t(b)});
          }
    }
    // children: where their update DOFs land in this front
    for (int sl = 0; sl < 2; ++sl) {
      const int c = h.child[sl];
      if (c < 0) continue;
      const HostFront& hc = B.fr[size_t(c)];
      const NDFront& dc = P.fronts[size_t(c)];
      const int64_t P1c = int64_t(ND_T) * dc.T1;
      for (size_t u = 0; u < hc.halo.size(); ++u) {
        const int32_t n = hc.halo[u];
        if (stamp[size_t(n)] != f)
          throw std::logic_error("nd_plan: a node around a child's box is not in its parent's front");
        for (int q = 0; q < 3; ++q) {
          const int64_t k = 3 * int64_t(u) + q;
          const int32_t pp = posof[size_t(n)] + q;
          P.upd_map[size_t(dc.map0 + k)] = pp;
          P.src[sl][size_t(d.pos0 + pp)] = int32_t(dc.pos0 + P1c + k);
        }
      }
    }
  }
  // task lists
  auto add = [&](int f, int i, int j) { P.tasks.push_back(NDTask{f, int16_t(i), int16_t(j)}); };
  const double tile_flops = 2.0 * ND_T * ND_T * ND_T;
  for (size_t l = 0; l < P.levels.size(); ++l) {
    NDLevel& L = P.levels[l];
    L.piv0[0] = int64_t(P.tasks.size());
    for (int f : L.fronts)
      if (P.fronts[size_t(f)].T1 > 0) add(f, 0, 0);
    L.piv0[1] = int64_t(P.tasks.size());
    for (int k = 0; k < L.maxT1; ++k) {
      L.step.push_back(int64_t(P.tasks.size()));
      for (int f : L.fronts) {
        const NDFront& d = P.fronts[size_t(f)];
        if (d.T1 > k)
          for (int j = 0; j < d.N; ++j)
            if (j != k) {
              add(f, k, j);
              P.flops += tile_flops;
            }
      }
      L.step.push_back(int64_t(P.tasks.size()));
      if (k > 0)
        for (int f : L.fronts) {
          const NDFront& d = P.fronts[size_t(f)];
          if (d.T1 >= k)
            for (int j = 0; j < d.N; ++j)
              if (j != k - 1) add(f, k - 1, j);
        }
      L.step.push_back(int64_t(P.tasks.size()));
      // the tiles whose CTA then inverts the next pivot go first: the longest tasks of the launch
      // start in its first wave instead of lengthening its tail
      auto next_pivot = [&](const NDFront& d, int i, int j) { return i == k + 1 && j == k + 1 && k + 1 < d.T1; };
      for (int f : L.fronts) {
        const NDFront& d = P.fronts[size_t(f)];
        if (d.T1 > k + 1) {
          add(f, k + 1, k + 1);
          P.flops += tile_flops;
        }
      }
      for (int f : L.fronts) {
        const NDFront& d = P.fronts[size_t(f)];
        if (d.T1 > k)
          for (int i = 0; i < d.N; ++i)
            for (int j = 0; j <= i; ++j)
              if (i != k && j != k && !next_pivot(d, i, j)) {
                add(f, i, j);
                P.flops += tile_flops;
              }
      }
      L.step.push_back(int64_t(P.tasks.size()));
    }
    L.fin_last[0] = int64_t(P.tasks.size());
    for (int f : L.fronts) {
      const NDFront& d = P.fronts[size_t(f)];
      if (d.T1 > 0 && d.T1 == L.maxT1)
        for (int j = 0; j < d.N; ++j)
          if (j != d.T1 - 1) add(f, d.T1 - 1, j);
    }
    L.fin_last[1] = int64_t(P.tasks.size());
    // extend-add into this level's fronts, child slot by child slot
    for (int sl = 0; sl < 2; ++sl) {
      L.ext[sl] = int64_t(P.tasks.size());
      for (int f : L.fronts) {
        const int c = B.fr[size_t(f)].child[sl];
        if (c < 0) continue;
        const NDFront& dc = P.fronts[size_t(c)];
        for (int i = dc.T1; i < dc.N; ++i)
          for (int j = dc.T1; j <= i; ++j) add(c, i, j);
      }
    }
    L.ext[2] = int64_t(P.tasks.size());
    auto chunks = [](int n) { return std::max(1, (n + ND_CHUNK - 1) / ND_CHUNK); };
    L.fwd[0] = int64_t(P.tasks.size());
    for (int f : L.fronts) {
      const NDFront& d = P.fronts[size_t(f)];
      for (int i = 0; i < d.N; ++i)
        for (int ch = 0; ch < chunks(d.T1); ++ch) add(f, i, ch);
    }
    L.fwd[1] = L.bwd[0] = int64_t(P.tasks.size());
    for (int f : L.fronts) {  // a front without update DOFs writes its solution going up
      const NDFront& d = P.fronts[size_t(f)];
      if (d.n2 > 0)
        for (int i = 0; i < d.T1; ++i)
          for (int ch = 0; ch < chunks(d.N - d.T1); ++ch) add(f, i, ch);
    }
    L.bwd[1] = int64_t(P.tasks.size());
    P.nsolve_tasks = std::max(P.nsolve_tasks, std::max(L.fwd[1] - L.fwd[0], L.bwd[1] - L.bwd[0]));
  }
  for (int l = int(P.levels.size()) - 1; l >= 0; --l) {
    const NDLevel& L = P.levels[size_t(l)];
    P.flow.insert(P.flow.end(), P.tasks.begin() + L.fwd[0], P.tasks.begin() + L.fwd[1]);
  }
  P.flow_fwd = int64_t(P.flow.size());
  for (const NDLevel& L : P.levels) P.flow.insert(P.flow.end(), P.tasks.begin() + L.bwd[0], P.tasks.begin() + L.bwd[1]);
  nd_check_plan(P);
  return P;
}

void nd_check_plan(const NDPlan& P) {
  auto fail = [](const std::string& m) { throw std::logic_error("nd plan check: " + m); };
  const int nf = int(P.fronts.size());
  int64_t tiles = 0, npos = 0;
  for (int f = 0; f < nf; ++f) {
    const NDFront& d = P.fronts[size_t(f)];
    if (d.N < d.T1 || d.T1 < 0 || d.n1 > ND_T * d.T1 || d.n2 > ND_T * (d.N - d.T1) || d.N > 32767)
      fail("front sizes " + std::to_string(f));
    if (d.parent >= nf || (d.parent < 0 && d.n2 != 0)) fail("parent of " + std::to_string(f));
    tiles += d.N * int64_t(d.N + 1) / 2;
    npos += int64_t(ND_T) * d.N;
    for (int64_t k = 0; k < d.n2; ++k) {
      const int32_t pp = P.upd_map[size_t(d.map0 + k)];
      if (d.parent < 0) fail("update DOFs without a parent");
      const NDFront& q = P.fronts[size_t(d.parent)];
      const bool sep = pp >= 0 && pp < q.n1;
      const bool upd = pp >= ND_T * q.T1 && pp < ND_T * q.T1 + q.n2;
      if (!sep && !upd) fail("update map of front " + std::to_string(f));
    }
  }
  if (tiles != P.ntiles || npos != P.npos) fail("storage totals");
  for (const NDTask& t : P.tasks) {
    if (t.f < 0 || t.f >= nf) fail("task front");
    const NDFront& d = P.fronts[size_t(t.f)];
    if (t.i < 0 || t.i >= d.N || t.j < 0 || t.j >= std::max(d.N, 1)) fail("task tile");
  }
  for (const NDAsm& a : P.asmb) {
    if (a.f < 0 || a.f >= nf) fail("assembly front");
    const NDFront& d = P.fronts[size_t(a.f)];
    if (a.pa < 0 || a.pa + 2 >= d.n1 || a.pb < 0 || a.pb + 2 >= ND_T * d.N) fail("assembly position");
  }
  for (const NDLevel& L : P.levels) {
    if (int64_t(L.step.size()) != 4 * int64_t(L.maxT1)) fail("step table");
    int64_t scr = 0;
    for (int f : L.fronts) {
      const NDFront& d = P.fronts[size_t(f)];
      if (d.pos0 < L.pos_begin || d.pos0 + ND_T * d.N > L.pos_end) fail("level positions");
      if (d.scr0 != scr) fail("scratch offsets");
      scr += 2 * d.N + 1;
    }
    if (scr != L.nscr || L.nscr > P.nscr) fail("scratch size");
  }
  for (int sl = 0; sl < 2; ++sl)
    for (int64_t p = 0; p < P.npos; ++p) {
      const int32_t s = P.src[sl][size_t(p)];
      if (s < -1 || s >= P.npos) fail("solve source index");
    }
  // dataflow order: every front's forward tasks after all of its children's, its backward tasks
  // after all of its parent's, every forward task before every backward task
  std::vector<int64_t> fwd_first(size_t(nf), -1), fwd_last(size_t(nf), -1), bwd_first(size_t(nf), -1),
      bwd_last(size_t(nf), -1);
  int64_t nsolve = 0;
  for (const NDLevel& L : P.levels) nsolve += (L.fwd[1] - L.fwd[0]) + (L.bwd[1] - L.bwd[0]);
  if (int64_t(P.flow.size()) != nsolve || P.flow_fwd < 0 || P.flow_fwd > nsolve) fail("flow size");
  std::vector<int> need(size_t(nf), 0);
  for (int64_t t = 0; t < nsolve; ++t) {
    const NDTask& k = P.flow[size_t(t)];
    if (k.f < 0 || k.f >= nf) fail("flow task front");
    auto& first = t < P.flow_fwd ? fwd_first : bwd_first;
    auto& last = t < P.flow_fwd ? fwd_last : bwd_last;
    if (first[size_t(k.f)] < 0) first[size_t(k.f)] = t;
    last[size_t(k.f)] = t;
  }
  for (int f = 0; f < nf; ++f) {
    const NDFront& d = P.fronts[size_t(f)];
    if (d.parent >= 0) need[size_t(d.parent)] += d.N;
    int a = d.parent;
    while (a >= 0 && P.fronts[size_t(a)].T1 == 0) a = P.fronts[size_t(a)].parent;
    if (d.bwd_front != a || d.bwd_need != (a >= 0 ? P.fronts[size_t(a)].T1 : 0))
      fail("backward wait of front " + std::to_string(f));
    if (a >= 0 && bwd_first[size_t(f)] >= 0 && P.fronts[size_t(a)].n2 > 0 && bwd_last[size_t(a)] >= bwd_first[size_t(f)])
      fail("flow: a backward task before its ancestor's");
    if (d.parent < 0 || fwd_first[size_t(d.parent)] < 0) continue;
    if (fwd_last[size_t(f)] >= fwd_first[size_t(d.parent)]) fail("flow: a forward task before its child's");
    if (bwd_first[size_t(f)] >= 0 && bwd_last[size_t(d.parent)] >= bwd_first[size_t(f)])
      fail("flow: a backward task before its parent's");
  }
  for (int f = 0; f < nf; ++f)
    if (P.fronts[size_t(f)].fwd_need != need[size_t(f)]) fail("forward need of front " + std::to_string(f));
}

}  // namespace topx
