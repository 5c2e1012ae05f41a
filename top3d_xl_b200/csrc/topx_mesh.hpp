// Host-side voxel FEA model of TOP3D_XL: discretisation, multigrid hierarchy,
// boundary conditions and the element matrices the device path needs.
//
// Every integer array that TOP3D_XL.m keeps 1-based (eNodMat, eleMapBack,
// nodMapBack, transferMat, ...) is produced here 1-based with the same values,
// so it can be compared bit for bit with the reference's numbering.
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <map>
#include <vector>

namespace topx {

struct Settings {
  // InitialSettings (TOP3D_XL.m:21-38)
  double modulus = 1.0;
  double poissonRatio = 0.3;
  double modulusMin = 1.0e-6;
  double SIMPpenalty = 3.0;
  double cellSize = 1.0;
  double tol = 1.0e-3;
  int maxIT = 800;
  double weightFactorJacobi = 0.6;
  int64_t coarsestResolutionControl = 50000;
  int typeVcycle = 0;  // 0 'Adapted' (the reference's setting), 1 'Standard' (TX:34)
  int specifyPassiveRegions[3] = {0, 0, 0};  // layers on the boundary, near loads, near fixations (TX:37)
  int nonDyadic = 1;
};

struct Level {
  int resX = 0, resY = 0, resZ = 0, span = 0;
  int64_t numElements = 0, numNodes = 0;
  std::vector<int32_t> eleMapBack;     // 1-based padded-grid element ids
  std::vector<int32_t> eleMapForward;  // grid element -> compact (1-based), 0 = void
  std::vector<int32_t> nodMapBack;     // 1-based grid node ids of this level's grid
  std::vector<int32_t> nodMapForward;  // grid node -> compact (1-based), 0 = absent
  std::vector<int32_t> eNodMat;        // [e*8 + j], 1-based compact node ids
  std::vector<int32_t> nodesOnBoundary;     // 1-based compact node ids (< 8 elements)
  std::vector<int32_t> elementsOnBoundary;  // level 1 only
  // coarse levels (TOP3D_XL.m:1076-1228)
  std::vector<int32_t> elementUpwardMap;  // [e*span^3 + c], compact finer ids, 0 = void
  std::vector<int32_t> transferMat;       // [e*(span+1)^3 + k], 1-based intermediate ids
  std::vector<double> transferMatCoeffi;  // per intermediate node
  std::vector<int32_t> solidNodeMapCoarser2Finer;  // per finer compact node, 1-based
  int64_t intermediateNumNodes = 0;

  int64_t gridElements() const { return int64_t(resX) * resY * resZ; }
  int64_t gridNodes() const { return int64_t(resX + 1) * (resY + 1) * (resZ + 1); }
};

struct LoadCase {
  std::vector<int32_t> node;            // compact 1-based
  std::vector<std::array<double, 3>> f;
};

struct Model {
  Settings S;
  int nelx = 0, nely = 0, nelz = 0;
  int numLevels = 0;
  std::vector<Level> levels;
  // fixingCond_: compact node id + fixing state per direction
  std::vector<int32_t> fixNode;
  std::vector<std::array<uint8_t, 3>> fixState;
  std::vector<LoadCase> loads;
  std::vector<double> objWeighting;
  std::vector<int32_t> passiveElements;  // 1-based compact element ids, sorted unique
  std::vector<uint8_t> fixedDOFs;        // per interleaved DOF (3*numNodes)
  // Solving_SetupKeWithFixedDOFs (TOP3D_XL.m:1338-1423)
  std::vector<int32_t> allElementsWithFixedDOFs;  // 1-based, sorted
  std::vector<int32_t> mapUniqueKes;              // per element, 1-based slot or 0
  std::vector<uint32_t> keFreeZeroMask;           // per slot: 24-bit mask of zeroed DOFs
  std::vector<std::array<double, 24>> keFixedDiag;  // per slot: diagonal of uniqueKesFixed_
  std::vector<int32_t> isThisEle2ndLevel;         // per level-2 element, 1-based index or 0
  std::vector<std::vector<int32_t>> sonElesWithFixedDOFs;  // 0-based child slots

  // element matrices
  std::array<double, 576> Ke{};  // row-major 24x24, unit modulus

  // build steps
  void load_cuboid(const uint8_t* vox, int ny, int nx, int nz);
  void load_topvoxel(const std::string& path);
  // fixings (node -> fixed flags per direction, a direction fixed where its value is 1) and loads
  // (load case from 1 -> node -> force) with node ids 1-based in the input model's own
  // (nely+1) x (nelx+1) x (nelz+1) node grid, as a .TopVoxel file gives them; replaces the
  // model's fixings, loads and load-case weights (AdaptBCExternalMdl, TOP3D_XL.m:1439-1490)
  void set_external_bc(const std::map<int64_t, std::array<double, 3>>& fix,
                       const std::map<int, std::map<int64_t, std::array<double, 3>>>& ld);
  void apply_boundary_condition();
  void setup();  // Ke + hierarchy + BC element matrices
  // TopOpti_SetPassiveElements (TOP3D_XL.m:1511-1574) for S.specifyPassiveRegions, after setup
  void set_passive_elements();
};

// Element matrices (TOP3D_XL.m:1254-1292, 1768-1798, 1617-1627, 816-853)
std::array<double, 576> element_stiffness(double nu, double cell);
std::vector<double> ri_operator(int span);  // (span+1)^3 x 8 row-major
std::vector<int32_t> sub_ele_nod_mat(int span);  // span^3 x 8 row-major, 1-based
std::array<double, 64> pde_filter_kernel(double rmin, double eleSize);
double matlab_round(double x);

// Derived matrices used by the coarse-operator kernels.
// Galerkin templates of a unit-modulus fine element at each child slot of a
// span-s coarse element: T_c = I_c^T K I_c  (24x24 each, row-major).
std::vector<double> galerkin_templates(const std::array<double, 576>& K, int span);
// Per child slot c of a span-s coarse element, the 24x24 map P_c from the
// coarse element's DOFs to the child's DOFs (row-major, child DOF = row).
std::vector<double> child_prolongators(int span);

}  // namespace topx
