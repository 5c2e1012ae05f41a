// Host-side voxel FEA model of TOP3D_XL (see topx_mesh.hpp).
#include "topx_mesh.hpp"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>

namespace topx {

double matlab_round(double x) {
  // MATLAB round: halves away from zero
  return x >= 0 ? std::floor(x + 0.5) : -std::floor(-x + 0.5);
}

// ---------------------------------------------------------------------------
// element matrices
// ---------------------------------------------------------------------------
static const int kHexNode[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                   {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

std::array<double, 576> element_stiffness(double nu, double cell) {
  // TOP3D_XL.m:1254-1292 gives Ke in closed form; here it is integrated exactly
  // (2x2x2 Gauss) from B^T D B, E = 1, interleaved DOFs 3a+c.
  const double lam = nu / ((1 + nu) * (1 - 2 * nu));
  const double mu = 1.0 / (2 * (1 + nu));
  double D[6][6] = {};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) D[i][j] = lam;
  for (int i = 0; i < 3; ++i) D[i][i] = lam + 2 * mu;
  D[3][3] = D[4][4] = D[5][5] = mu;
  const double g = 1.0 / std::sqrt(3.0);
  const double jac = 2.0 / cell, detJ = (cell / 2) * (cell / 2) * (cell / 2);
  std::array<double, 576> K{};
  const double gp[2] = {-g, g};
  for (double gs : gp)
    for (double gt : gp)
      for (double gq : gp) {
        double B[6][24] = {};
        for (int a = 0; a < 8; ++a) {
          const double sa = kHexNode[a][0], ta = kHexNode[a][1], pa = kHexNode[a][2];
          const double dNs = 0.125 * sa * (1 + ta * gt) * (1 + pa * gq) * jac;
          const double dNt = 0.125 * ta * (1 + sa * gs) * (1 + pa * gq) * jac;
          const double dNp = 0.125 * pa * (1 + sa * gs) * (1 + ta * gt) * jac;
          B[0][3 * a] = dNs;
          B[1][3 * a + 1] = dNt;
          B[2][3 * a + 2] = dNp;
          B[3][3 * a] = dNt;
          B[3][3 * a + 1] = dNs;
          B[4][3 * a + 1] = dNp;
          B[4][3 * a + 2] = dNt;
          B[5][3 * a] = dNp;
          B[5][3 * a + 2] = dNs;
        }
        double DB[6][24];
        for (int i = 0; i < 6; ++i)
          for (int j = 0; j < 24; ++j) {
            double s = 0;
            for (int k = 0; k < 6; ++k) s += D[i][k] * B[k][j];
            DB[i][j] = s;
          }
        for (int i = 0; i < 24; ++i)
          for (int j = 0; j < 24; ++j) {
            double s = 0;
            for (int k = 0; k < 6; ++k) s += B[k][i] * DB[k][j];
            K[i * 24 + j] += s * detJ;
          }
      }
  for (int i = 0; i < 24; ++i)
    for (int j = i + 1; j < 24; ++j) {
      const double v = 0.5 * (K[i * 24 + j] + K[j * 24 + i]);
      K[i * 24 + j] = K[j * 24 + i] = v;
    }
  return K;
}

std::vector<double> ri_operator(int span) {
  // Solving_Operator4MultiGridRestrictionAndInterpolation 'inNODE' (TOP3D_XL.m:1768-1783)
  if (span != 2 && span != 4) throw std::runtime_error("Wrong Span Width!");
  const int n = span + 1;
  std::vector<double> N(size_t(n) * n * n * 8);
  for (int kz = 0; kz < n; ++kz)
    for (int kx = 0; kx < n; ++kx)
      for (int ky = 0; ky < n; ++ky) {
        const int k = ky + n * kx + n * n * kz;
        const double s = -1.0 + 2.0 * kx / span;
        const double t = 1.0 - 2.0 * ky / span;
        const double p = -1.0 + 2.0 * kz / span;
        for (int a = 0; a < 8; ++a)
          N[size_t(k) * 8 + a] = 0.125 * (1 + kHexNode[a][0] * s) * (1 + kHexNode[a][1] * t) *
                                 (1 + kHexNode[a][2] * p);
      }
  return N;
}

std::vector<int32_t> sub_ele_nod_mat(int span) {
  // Solving_SubEleNodMat (TOP3D_XL.m:1617-1627)
  if (span != 2 && span != 4) throw std::runtime_error("Wrong Span Width!");
  const int n = span, P = (n + 1) * (n + 1);
  const int offs[8] = {0, n + 1, n, -1, P, P + n + 1, P + n, P - 1};
  std::vector<int32_t> m(size_t(n) * n * n * 8);
  for (int iz = 0; iz < n; ++iz)
    for (int ix = 0; ix < n; ++ix)
      for (int iy = 0; iy < n; ++iy) {
        const int c = iy + n * ix + n * n * iz;
        const int base = iy + (n + 1) * ix + P * iz + 2;
        for (int j = 0; j < 8; ++j) m[size_t(c) * 8 + j] = base + offs[j];
      }
  return m;
}

std::array<double, 64> pde_filter_kernel(double rmin, double eleSize) {
  // TopOpti_SetupPDEfilter_matrixFree (TOP3D_XL.m:816-853): KEF0 uses the
  // natural-coordinate derivatives with unit weights, as the reference does.
  const double g = 1.0 / std::sqrt(3.0);
  const double s[8] = {-g, g, g, -g, -g, g, g, -g};
  const double t[8] = {-g, -g, g, g, -g, -g, g, g};
  const double p[8] = {-g, -g, -g, -g, g, g, g, g};
  double N[8][8], dS[24][8];
  for (int q = 0; q < 8; ++q)
    for (int a = 0; a < 8; ++a) {
      const double sa = kHexNode[a][0], ta = kHexNode[a][1], pa = kHexNode[a][2];
      N[q][a] = 0.125 * (1 + sa * s[q]) * (1 + ta * t[q]) * (1 + pa * p[q]);
      dS[3 * q][a] = 0.125 * sa * (1 + ta * t[q]) * (1 + pa * p[q]);
      dS[3 * q + 1][a] = 0.125 * ta * (1 + sa * s[q]) * (1 + pa * p[q]);
      dS[3 * q + 2][a] = 0.125 * pa * (1 + sa * s[q]) * (1 + ta * t[q]);
    }
  const double wgt = 1.0 / 8;
  const double iR = (rmin * eleSize) / 2 / std::sqrt(3.0);
  std::array<double, 64> K{};
  for (int a = 0; a < 8; ++a)
    for (int b = 0; b < 8; ++b) {
      double k0 = 0, k1 = 0;
      for (int r = 0; r < 24; ++r) k0 += dS[r][a] * dS[r][b];
      for (int q = 0; q < 8; ++q) k1 += N[q][a] * wgt * N[q][b];
      K[a * 8 + b] = iR * iR * k0 + k1;
    }
  return K;
}

std::vector<double> child_prolongators(int span) {
  const std::vector<double> RI = ri_operator(span);
  const std::vector<int32_t> en = sub_ele_nod_mat(span);
  const int nc = span * span * span;
  std::vector<double> P(size_t(nc) * 576, 0.0);
  for (int c = 0; c < nc; ++c)
    for (int a = 0; a < 8; ++a) {
      const int k = en[size_t(c) * 8 + a] - 1;
      for (int b = 0; b < 8; ++b)
        for (int i = 0; i < 3; ++i) P[size_t(c) * 576 + (3 * a + i) * 24 + 3 * b + i] = RI[size_t(k) * 8 + b];
    }
  return P;
}

std::vector<double> galerkin_templates(const std::array<double, 576>& K, int span) {
  const std::vector<double> P = child_prolongators(span);
  const int nc = span * span * span;
  std::vector<double> T(size_t(nc) * 576, 0.0);
  for (int c = 0; c < nc; ++c) {
    const double* Pc = &P[size_t(c) * 576];
    double KP[576];
    for (int i = 0; i < 24; ++i)
      for (int j = 0; j < 24; ++j) {
        double s = 0;
        for (int k = 0; k < 24; ++k) s += K[i * 24 + k] * Pc[k * 24 + j];
        KP[i * 24 + j] = s;
      }
    for (int i = 0; i < 24; ++i)
      for (int j = 0; j < 24; ++j) {
        double s = 0;
        for (int k = 0; k < 24; ++k) s += Pc[k * 24 + i] * KP[k * 24 + j];
        T[size_t(c) * 576 + i * 24 + j] = s;
      }
  }
  return T;
}

// ---------------------------------------------------------------------------
// discretisation (TOP3D_XL.m:1629-1730) and hierarchy (TOP3D_XL.m:1076-1228)
// ---------------------------------------------------------------------------
static void discretize_grid(const std::vector<uint8_t>& solid, Level& L) {
  const int64_t ny = L.resY, nx = L.resX, nz = L.resZ;
  const int64_t nge = nx * ny * nz;
  const int64_t P = (ny + 1) * (nx + 1);
  const int64_t offs[8] = {0, ny + 1, ny, -1, P, P + ny + 1, P + ny, P - 1};
  L.eleMapBack.clear();
  L.eleMapForward.assign(nge, 0);
  for (int64_t id = 0; id < nge; ++id)
    if (solid[id]) {
      L.eleMapBack.push_back(int32_t(id + 1));
      L.eleMapForward[id] = int32_t(L.eleMapBack.size());
    }
  L.numElements = int64_t(L.eleMapBack.size());
  const int64_t ngn = L.gridNodes();
  std::vector<uint8_t> mark(ngn, 0);
  std::vector<int64_t> full(size_t(L.numElements) * 8);
  for (int64_t e = 0; e < L.numElements; ++e) {
    const int64_t id = L.eleMapBack[e] - 1;
    const int64_t iy = id % ny, ix = (id / ny) % nx, iz = id / (ny * nx);
    const int64_t base = (iy + 1) + (ny + 1) * ix + P * iz + 1;  // 1-based
    for (int j = 0; j < 8; ++j) {
      full[size_t(e) * 8 + j] = base + offs[j];
      mark[base + offs[j] - 1] = 1;
    }
  }
  L.nodMapBack.clear();
  L.nodMapForward.assign(ngn, 0);
  for (int64_t k = 0; k < ngn; ++k)
    if (mark[k]) {
      L.nodMapBack.push_back(int32_t(k + 1));
      L.nodMapForward[k] = int32_t(L.nodMapBack.size());
    }
  L.numNodes = int64_t(L.nodMapBack.size());
  L.eNodMat.resize(full.size());
  std::vector<int32_t> cnt(L.numNodes, 0);
  for (size_t i = 0; i < full.size(); ++i) {
    L.eNodMat[i] = L.nodMapForward[full[i] - 1];
    cnt[L.eNodMat[i] - 1]++;
  }
  L.nodesOnBoundary.clear();
  for (int64_t k = 0; k < L.numNodes; ++k)
    if (cnt[k] < 8) L.nodesOnBoundary.push_back(int32_t(k + 1));
}

static void build_hierarchy(Model& M) {
  int numLevels = M.numLevels;
  int nonDyadic = M.S.nonDyadic;
  if (nonDyadic == 1 && numLevels >= 4)
    numLevels -= 1;
  else
    nonDyadic = 0;
  for (int ii = 2; ii <= numLevels; ++ii) {
    const Level& F = M.levels.back();
    const int s = (ii == 2 && nonDyadic == 1) ? 4 : 2;
    Level C;
    C.resX = F.resX / s;
    C.resY = F.resY / s;
    C.resZ = F.resZ / s;
    C.span = s;
    const int64_t ny = C.resY, nx = C.resX, nz = C.resZ;
    const int64_t nce = nx * ny * nz, s3 = int64_t(s) * s * s, s1 = s + 1, s13 = s1 * s1 * s1;
    const int64_t fny = s * ny, fnx = s * nx;
    const int64_t fnny = fny + 1, fnnx = fnx + 1, fnnz = s * nz + 1;
    std::vector<uint8_t> nonempty(nce, 0);
    for (int64_t jz = 0; jz < nz; ++jz)
      for (int64_t kx = 0; kx < nx; ++kx)
        for (int64_t gy = 0; gy < ny; ++gy) {
          const int64_t ce = gy + ny * kx + ny * nx * jz;
          bool any = false;
          for (int cz = 0; cz < s && !any; ++cz)
            for (int cx = 0; cx < s && !any; ++cx)
              for (int cy = 0; cy < s && !any; ++cy) {
                const int64_t fid = (s * gy + cy) + fny * (s * kx + cx) + fny * fnx * (s * jz + cz);
                if (F.eleMapForward[fid] > 0) any = true;
              }
          nonempty[ce] = any;
        }
    // intermediate nodes: all fine nodes of non-empty coarse elements (sorted)
    std::vector<int32_t> rank(size_t(fnny * fnnx * fnnz), 0);
    for (int64_t ce = 0; ce < nce; ++ce) {
      if (!nonempty[ce]) continue;
      const int64_t gy = ce % ny, kx = (ce / ny) % nx, jz = ce / (ny * nx);
      for (int kz = 0; kz < s1; ++kz)
        for (int kxx = 0; kxx < s1; ++kxx)
          for (int ky = 0; ky < s1; ++ky)
            rank[(s * gy + ky) + fnny * (s * kx + kxx) + fnny * fnnx * (s * jz + kz)] = 1;
    }
    int64_t ni = 0;
    for (auto& r : rank)
      if (r) r = int32_t(++ni);
    C.intermediateNumNodes = ni;
    C.transferMatCoeffi.assign(ni, 0.0);
    C.eleMapBack.clear();
    for (int64_t ce = 0; ce < nce; ++ce)
      if (nonempty[ce]) C.eleMapBack.push_back(int32_t(ce + 1));
    const int64_t ne = int64_t(C.eleMapBack.size());
    C.transferMat.resize(size_t(ne * s13));
    C.elementUpwardMap.resize(size_t(ne * s3));
    for (int64_t e = 0; e < ne; ++e) {
      const int64_t ce = C.eleMapBack[e] - 1;
      const int64_t gy = ce % ny, kx = (ce / ny) % nx, jz = ce / (ny * nx);
      for (int kz = 0; kz < s1; ++kz)
        for (int kxx = 0; kxx < s1; ++kxx)
          for (int ky = 0; ky < s1; ++ky) {
            const int32_t r = rank[(s * gy + ky) + fnny * (s * kx + kxx) + fnny * fnnx * (s * jz + kz)];
            C.transferMat[size_t(e * s13 + ky + s1 * kxx + s1 * s1 * kz)] = r;
            C.transferMatCoeffi[r - 1] += 1.0;
          }
      for (int cz = 0; cz < s; ++cz)
        for (int cx = 0; cx < s; ++cx)
          for (int cy = 0; cy < s; ++cy) {
            const int64_t fid = (s * gy + cy) + fny * (s * kx + cx) + fny * fnx * (s * jz + cz);
            C.elementUpwardMap[size_t(e * s3 + cy + s * cx + s * s * cz)] = F.eleMapForward[fid];
          }
    }
    C.solidNodeMapCoarser2Finer.resize(F.numNodes);
    for (int64_t k = 0; k < F.numNodes; ++k) C.solidNodeMapCoarser2Finer[k] = rank[F.nodMapBack[k] - 1];
    discretize_grid(nonempty, C);
    M.levels.push_back(std::move(C));
  }
  M.numLevels = numLevels;
}

static void discretize_level1(Model& M, const std::vector<uint8_t>& vox) {
  // vox: (nely, nelx, nelz) column-major
  int64_t numVoxels = 0;
  for (auto v : vox) numVoxels += v ? 1 : 0;
  int L = 0;
  while (numVoxels >= M.S.coarsestResolutionControl) {
    ++L;
    numVoxels = int64_t(matlab_round(double(numVoxels) / 8.0));
  }
  L = std::max(3, L);
  const int f = 1 << L;
  Level l1;
  l1.resX = int(std::ceil(double(M.nelx) / f) * f);
  l1.resY = int(std::ceil(double(M.nely) / f) * f);
  l1.resZ = int(std::ceil(double(M.nelz) / f) * f);
  M.numLevels = L + 1;
  std::vector<uint8_t> solid(size_t(l1.gridElements()), 0);
  for (int iz = 0; iz < M.nelz; ++iz)
    for (int ix = 0; ix < M.nelx; ++ix)
      for (int iy = 0; iy < M.nely; ++iy)
        solid[size_t(iy) + size_t(l1.resY) * (ix + size_t(l1.resX) * iz)] =
            vox[size_t(iy) + size_t(M.nely) * (ix + size_t(M.nelx) * iz)] ? 1 : 0;
  discretize_grid(solid, l1);
  std::vector<uint8_t> isb(l1.numNodes + 1, 0);
  for (auto k : l1.nodesOnBoundary) isb[k] = 1;
  l1.elementsOnBoundary.clear();
  for (int64_t e = 0; e < l1.numElements; ++e) {
    bool any = false;
    for (int j = 0; j < 8; ++j) any |= isb[l1.eNodMat[size_t(e) * 8 + j]] != 0;
    if (any) l1.elementsOnBoundary.push_back(int32_t(e + 1));
  }
  M.levels.clear();
  M.levels.push_back(std::move(l1));
}

// ---------------------------------------------------------------------------
// input models (TOP3D_XL.m:442-561)
// ---------------------------------------------------------------------------
void Model::load_cuboid(const uint8_t* vox, int ny, int nx, int nz) {
  if (nx < 3 || ny < 3 || nz < 3) throw std::runtime_error("Inappropriate Input Model!");
  nely = ny;
  nelx = nx;
  nelz = nz;
  std::vector<uint8_t> v(vox, vox + size_t(nx) * ny * nz);
  discretize_level1(*this, v);
  const Level& l1 = levels[0];
  const int64_t NY = l1.resY + 1, NX = l1.resX + 1;
  fixNode.clear();
  fixState.clear();
  for (int iz = 0; iz <= nelz; ++iz)
    for (int iy = 0; iy <= nely; ++iy) {
      const int32_t k = l1.nodMapForward[iy + NY * NX * iz];
      fixNode.push_back(k);
      fixState.push_back({1, 1, 1});
    }
  const int zt = int(matlab_round(nelz / 6.0 + 1));
  LoadCase lc;
  for (int iz = 0; iz < zt; ++iz)
    for (int iy = 0; iy <= nely; ++iy) lc.node.push_back(l1.nodMapForward[iy + NY * nelx + NY * NX * iz]);
  const double fz = -1.0 / double(lc.node.size());
  lc.f.assign(lc.node.size(), {0.0, 0.0, fz});
  loads.assign(1, lc);
  objWeighting.assign(1, 1.0);
  passiveElements.clear();
}

void Model::load_topvoxel(const std::string& path) {
  // .TopVoxel v1.0 (TOP3D_XL.m:448-528) with AdaptBCExternalMdl (TOP3D_XL.m:1439-1490)
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open " + path);
  std::vector<std::string> tok;
  for (std::string t; in >> t;) tok.push_back(t);
  size_t pos = 0;
  auto take = [&]() -> const std::string& {
    if (pos >= tok.size()) throw std::runtime_error("Incompatible Mesh Data Format!");
    return tok[pos++];
  };
  for (int i = 0; i < 5; ++i) take();
  if (std::stod(take()) != 1.0) throw std::runtime_error("Unsupported Data!");
  if (take() != "Resolution:") throw std::runtime_error("Incompatible Mesh Data Format!");
  nelx = std::stoi(take());
  nely = std::stoi(take());
  nelz = std::stoi(take());
  take();
  take();
  const int withDensity = std::stoi(take());
  take();
  take();
  const int64_t nsolid = std::stoll(take());
  const int64_t nvox = int64_t(nelx) * nely * nelz;
  std::vector<uint8_t> vox(nvox, 0);
  for (int64_t i = 0; i < nsolid; ++i) {
    const int64_t v = std::stoll(take());
    if (v < 1 || v > nvox) throw std::runtime_error("voxel index out of range");
    vox[v - 1] = 1;
    if (withDensity) take();
  }
  if (take() != "Passive" || take() != "elements:") throw std::runtime_error("Incompatible Mesh Data Format!");
  const int64_t npas = std::stoll(take());
  std::vector<int64_t> passive(npas);
  for (auto& p : passive) p = std::stoll(take());
  if (take() != "Fixations:") throw std::runtime_error("Incompatible Mesh Data Format!");
  const int64_t nfix = std::stoll(take());
  std::map<int64_t, std::array<double, 3>> fix;  // unique + sorted by node id (first kept)
  for (int64_t i = 0; i < nfix; ++i) {
    const int64_t n = std::stoll(take());
    std::array<double, 3> st{std::stod(take()), std::stod(take()), std::stod(take())};
    fix.emplace(n, st);
  }
  if (take() != "Loads:") throw std::runtime_error("Incompatible Mesh Data Format!");
  std::map<int, std::map<int64_t, std::array<double, 3>>> ld;
  const int64_t nl = std::stoll(take());
  for (int64_t i = 0; i < nl; ++i) {
    const int64_t n = std::stoll(take());
    std::array<double, 3> f{std::stod(take()), std::stod(take()), std::stod(take())};
    ld[1].emplace(n, f);
  }
  take();
  take();
  const int nadd = std::stoi(take());
  for (int a = 0; a < nadd; ++a) {
    if (take() != "Loads:") throw std::runtime_error("Incompatible Mesh Data Format!");
    const int64_t k = std::stoll(take());
    const int idx = std::stoi(take());
    auto& m = ld[idx];
    for (int64_t i = 0; i < k; ++i) {
      const int64_t n = std::stoll(take());
      std::array<double, 3> f{std::stod(take()), std::stod(take()), std::stod(take())};
      m.emplace(n, f);
    }
  }
  discretize_level1(*this, vox);
  const Level& l1 = levels[0];
  set_external_bc(fix, ld);
  passiveElements.clear();
  for (auto p : passive) {
    const int64_t k = p - 1;
    const int64_t iy = k % nely, ix = (k / nely) % nelx, iz = k / (int64_t(nely) * nelx);
    const int32_t e = l1.eleMapForward[iy + int64_t(l1.resY) * (ix + int64_t(l1.resX) * iz)];
    if (e > 0) passiveElements.push_back(e);
  }
  std::sort(passiveElements.begin(), passiveElements.end());
  passiveElements.erase(std::unique(passiveElements.begin(), passiveElements.end()), passiveElements.end());
}

void Model::set_external_bc(const std::map<int64_t, std::array<double, 3>>& fix,
                            const std::map<int, std::map<int64_t, std::array<double, 3>>>& ld) {
  const Level& l1 = levels.at(0);
  // re-index an original-grid node id into the padded node grid
  const int64_t ony = nely + 1, onx = nelx + 1;
  const int64_t ANY = l1.resY + 1, ANX = l1.resX + 1;
  const int64_t nOrig = ony * onx * (int64_t(nelz) + 1);
  auto adapt = [&](int64_t n1) -> int64_t {
    if (n1 < 1 || n1 > nOrig) throw std::invalid_argument("boundary-condition node id out of range");
    const int64_t k = n1 - 1;
    const int64_t iy = k % ony, ix = (k / ony) % onx, iz = k / (ony * onx);
    return iy + ANY * ix + ANY * ANX * iz;
  };
  fixNode.clear();
  fixState.clear();
  auto solid = [&](int64_t n1) -> int32_t {
    const int32_t n = l1.nodMapForward[adapt(n1)];
    if (n <= 0) throw std::runtime_error("boundary-condition node is not a node of the solid model");
    return n;
  };
  for (auto& kv : fix) {
    fixNode.push_back(solid(kv.first));
    fixState.push_back({uint8_t(kv.second[0] == 1), uint8_t(kv.second[1] == 1), uint8_t(kv.second[2] == 1)});
  }
  loads.clear();
  const int nL = ld.empty() ? 1 : ld.rbegin()->first;
  for (int i = 1; i <= nL; ++i) {
    LoadCase lc;
    const auto it = ld.find(i);
    if (it != ld.end())
      for (auto& kv : it->second) {
        lc.node.push_back(solid(kv.first));
        lc.f.push_back(kv.second);
      }
    loads.push_back(lc);
  }
  objWeighting.assign(nL, 1.0 / nL);
}

// Common_IncludeAdjacentElements (TOP3D_XL.m:1578-1606): the elements of the 3x3x3 block of padded
// grid cells around each listed element, sorted unique compact ids
static std::vector<int32_t> include_adjacent_elements(const Level& l1, const std::vector<int32_t>& in) {
  const int64_t ny = l1.resY, nx = l1.resX, nz = l1.resZ;
  std::vector<int32_t> out;
  out.reserve(in.size() * 27);
  for (int32_t e : in) {
    const int64_t g = l1.eleMapBack[e - 1] - 1;
    const int64_t iy = g % ny, ix = (g / ny) % nx, iz = g / (ny * nx);
    for (int dz = -1; dz <= 1; ++dz)
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy) {
          const int64_t y = iy + dy, x = ix + dx, z = iz + dz;
          if (y < 0 || y >= ny || x < 0 || x >= nx || z < 0 || z >= nz) continue;
          const int32_t f = l1.eleMapForward[y + ny * (x + nx * z)];
          if (f > 0) out.push_back(f);
        }
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

void Model::set_passive_elements() {
  // TopOpti_SetPassiveElements (TOP3D_XL.m:1511-1574).  As written there, the loaded and fixed
  // node ids (compact) index the list of boundary nodes (TOP3D_XL.m:1557, 1569); an id past its end
  // is MATLAB's index error.
  const int nb = S.specifyPassiveRegions[0], nl = S.specifyPassiveRegions[1], nf = S.specifyPassiveRegions[2];
  if (nb <= 0 && nl <= 0 && nf <= 0) return;
  const Level& l1 = levels.at(0);
  std::vector<int32_t> all = passiveElements;
  if (nb > 0) {
    std::vector<int32_t> onB = l1.elementsOnBoundary;
    for (int i = 2; i <= nb; ++i) onB = include_adjacent_elements(l1, onB);
    all.insert(all.end(), onB.begin(), onB.end());
  }
  if (nl > 0 || nf > 0) {
    // node -> the boundary elements containing it (TOP3D_XL.m:1536-1548)
    std::vector<std::vector<int32_t>> nodeEles(size_t(l1.numNodes) + 1);
    std::vector<int32_t> be = l1.elementsOnBoundary;
    std::sort(be.begin(), be.end());
    for (int32_t e : be)
      for (int j = 0; j < 8; ++j) nodeEles[l1.eNodMat[size_t(e - 1) * 8 + j]].push_back(e);
    const auto& nob = l1.nodesOnBoundary;
    auto around = [&](const std::vector<int32_t>& ids) {
      std::vector<int32_t> es;
      for (int32_t id : ids) {
        if (id < 1 || size_t(id) > nob.size())
          throw std::runtime_error("passive layers near loads or fixations: node id exceeds the boundary-node list");
        const auto& v = nodeEles[nob[id - 1]];
        es.insert(es.end(), v.begin(), v.end());
      }
      std::sort(es.begin(), es.end());
      es.erase(std::unique(es.begin(), es.end()), es.end());
      return es;
    };
    if (nl > 0) {
      std::vector<int32_t> nearL;
      for (const auto& lc : loads) {
        const auto es = around(lc.node);
        nearL.insert(nearL.end(), es.begin(), es.end());
      }
      for (int i = 2; i <= nl; ++i) nearL = include_adjacent_elements(l1, nearL);
      all.insert(all.end(), nearL.begin(), nearL.end());
    }
    if (nf > 0) {
      std::vector<int32_t> nearF = around(fixNode);
      for (int i = 2; i <= nf; ++i) nearF = include_adjacent_elements(l1, nearF);
      all.insert(all.end(), nearF.begin(), nearF.end());
    }
  }
  std::sort(all.begin(), all.end());
  all.erase(std::unique(all.begin(), all.end()), all.end());
  passiveElements = all;
}

void Model::apply_boundary_condition() {
  // FEA_ApplyBoundaryCondition (TOP3D_XL.m:1294-1336)
  if (loads.empty()) throw std::runtime_error("No Loads!");
  for (auto& lc : loads) {
    std::vector<std::pair<int32_t, std::array<double, 3>>> l;
    for (size_t i = 0; i < lc.node.size(); ++i) l.push_back({lc.node[i], lc.f[i]});
    std::stable_sort(l.begin(), l.end(), [](auto& a, auto& b) { return a.first < b.first; });
    l.erase(std::unique(l.begin(), l.end(), [](auto& a, auto& b) { return a.first == b.first; }), l.end());
    std::vector<std::pair<int32_t, std::array<uint8_t, 3>>> f;
    for (size_t i = 0; i < fixNode.size(); ++i) {
      const bool loaded = std::binary_search(l.begin(), l.end(), std::make_pair(fixNode[i], std::array<double, 3>{}),
                                             [](auto& a, auto& b) { return a.first < b.first; });
      if (!loaded) f.push_back({fixNode[i], fixState[i]});
    }
    std::stable_sort(f.begin(), f.end(), [](auto& a, auto& b) { return a.first < b.first; });
    f.erase(std::unique(f.begin(), f.end(), [](auto& a, auto& b) { return a.first == b.first; }), f.end());
    if (l.empty()) throw std::runtime_error("No Loads!");
    if (f.empty()) throw std::runtime_error("No Fixations!");
    lc.node.clear();
    lc.f.clear();
    for (auto& p : l) {
      lc.node.push_back(p.first);
      lc.f.push_back(p.second);
    }
    fixNode.clear();
    fixState.clear();
    for (auto& p : f) {
      fixNode.push_back(p.first);
      fixState.push_back(p.second);
    }
  }
  for (auto n : fixNode)
    if (n <= 0) throw std::runtime_error("fixed node is not a solid node");
  for (auto& lc : loads)
    for (auto n : lc.node)
      if (n <= 0) throw std::runtime_error("loaded node is not a solid node");
  const Level& l1 = levels[0];
  fixedDOFs.assign(size_t(l1.numNodes) * 3, 0);
  for (size_t i = 0; i < fixNode.size(); ++i)
    for (int c = 0; c < 3; ++c)
      if (fixState[i][c] == 1) fixedDOFs[size_t(fixNode[i] - 1) * 3 + c] = 1;
}

void Model::setup() {
  // FEA_SetupVoxelBased (TOP3D_XL.m:1238-1252)
  Ke = element_stiffness(S.poissonRatio, S.cellSize);
  if (levels.size() == 1) build_hierarchy(*this);
  // Solving_SetupKeWithFixedDOFs (TOP3D_XL.m:1338-1423)
  const Level& l1 = levels[0];
  const auto& nob = l1.nodesOnBoundary;
  std::vector<int32_t> slot(l1.numNodes + 1, 0);
  for (size_t i = 0; i < nob.size(); ++i) slot[nob[i]] = int32_t(i + 1);
  std::vector<uint8_t> isBE(l1.numElements + 1, 0);
  for (auto e : l1.elementsOnBoundary) isBE[e] = 1;
  std::vector<int64_t> start(nob.size() + 1, 0);
  for (int64_t e = 0; e < l1.numElements; ++e)
    if (isBE[e + 1])
      for (int j = 0; j < 8; ++j) {
        const int32_t s = slot[l1.eNodMat[size_t(e) * 8 + j]];
        if (s) start[s]++;
      }
  for (size_t i = 1; i < start.size(); ++i) start[i] += start[i - 1];
  std::vector<int32_t> lists(start.back());
  std::vector<int64_t> fillp(start.begin(), start.end() - 1);
  for (int64_t e = 0; e < l1.numElements; ++e)
    if (isBE[e + 1])
      for (int j = 0; j < 8; ++j) {
        const int32_t s = slot[l1.eNodMat[size_t(e) * 8 + j]];
        if (s) lists[fillp[s - 1]++] = int32_t(e + 1);
      }
  // [~, fixedNodeIndices] = intersect(nodesOnBoundary, fixingCond(:,1))
  std::vector<size_t> fni;
  {
    std::vector<int32_t> fs(fixNode);
    std::sort(fs.begin(), fs.end());
    fs.erase(std::unique(fs.begin(), fs.end()), fs.end());
    size_t a = 0, b = 0;
    while (a < nob.size() && b < fs.size()) {
      if (nob[a] < fs[b])
        ++a;
      else if (nob[a] > fs[b])
        ++b;
      else {
        fni.push_back(a);
        ++a;
        ++b;
      }
    }
  }
  std::vector<int32_t> allfix;
  for (auto i : fni)
    for (int64_t k = start[i]; k < start[i + 1]; ++k) allfix.push_back(lists[k]);
  std::sort(allfix.begin(), allfix.end());
  allfix.erase(std::unique(allfix.begin(), allfix.end()), allfix.end());
  allElementsWithFixedDOFs = allfix;
  mapUniqueKes.assign(l1.numElements, 0);
  for (size_t i = 0; i < allfix.size(); ++i) mapUniqueKes[allfix[i] - 1] = int32_t(i + 1);
  keFreeZeroMask.assign(allfix.size(), 0u);
  keFixedDiag.assign(allfix.size(), std::array<double, 24>{});
  for (size_t ii = 0; ii < fni.size(); ++ii) {
    // the reference pairs the ii-th fixingCond row with the ii-th intersected node list
    const int32_t iNode = fixNode[ii];
    const auto st = fixState[ii];
    const size_t i = fni[ii];
    const int64_t nAdj = start[i + 1] - start[i];
    for (int64_t k = start[i]; k < start[i + 1]; ++k) {
      const int32_t e = lists[k];
      const int32_t sl = mapUniqueKes[e - 1] - 1;
      for (int a = 0; a < 8; ++a) {
        if (l1.eNodMat[size_t(e - 1) * 8 + a] != iNode) continue;
        for (int c = 0; c < 3; ++c)
          if (st[c] == 1) {
            keFreeZeroMask[sl] |= 1u << (3 * a + c);
            keFixedDiag[sl][3 * a + c] = 1.0 / double(nAdj);
          }
      }
    }
  }
  for (auto& d : keFixedDiag)
    for (auto& v : d) v = v * S.modulus * S.cellSize;
  // level-2 elements holding elements with fixed DOFs (TOP3D_XL.m:1404-1423)
  const Level& l2 = levels[1];
  const int64_t s3 = int64_t(l2.span) * l2.span * l2.span;
  isThisEle2ndLevel.assign(l2.numElements, 0);
  sonElesWithFixedDOFs.clear();
  int32_t cnt = 0;
  for (int64_t j = 0; j < l2.numElements; ++j) {
    std::vector<std::pair<int32_t, int32_t>> hit;
    for (int64_t c = 0; c < s3; ++c) {
      const int32_t e = l2.elementUpwardMap[size_t(j * s3 + c)];
      if (e > 0 && mapUniqueKes[e - 1] > 0) hit.push_back({e, int32_t(c)});
    }
    if (hit.empty()) continue;
    isThisEle2ndLevel[j] = ++cnt;
    std::sort(hit.begin(), hit.end());
    std::vector<int32_t> arr;
    for (auto& h : hit) arr.push_back(h.second);
    sonElesWithFixedDOFs.push_back(arr);
  }
}

}  // namespace topx
