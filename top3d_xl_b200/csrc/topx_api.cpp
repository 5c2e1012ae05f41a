// C ABI of the B200-native TOP3D_XL engine (declared in include/topx.h).
#include "../../include/topx.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "topx_engine.hpp"
#include "topx_mesh.hpp"

struct topx_ctx {
  topx_params params{};
  std::unique_ptr<topx::Model> model;
  std::unique_ptr<topx::Engine> engine;
  std::string err;
  bool begun = false;
  // the loaded input, to rebuild the model when topx_set_bc replaces its boundary conditions
  std::vector<uint8_t> vox;
  int vny = 0, vnx = 0, vnz = 0;
  std::string topvoxel;
};

namespace {

topx_status fail(topx_ctx* c, topx_status code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

template <typename F>
topx_status guarded(topx_ctx* c, F&& f) {
  if (!c) return TOPX_ERR_ARG;
  try {
    return f();
  } catch (const topx::CudaError& e) {
    return fail(c, TOPX_ERR_CUDA, e.what());
  } catch (const topx::DeviceWaitError& e) {
    return fail(c, TOPX_ERR_TIMEOUT, e.what());
  } catch (const std::invalid_argument& e) {
    return fail(c, TOPX_ERR_ARG, e.what());
  } catch (const std::runtime_error& e) {
    const std::string m = e.what();
    if (m.find("MMA") != std::string::npos) return fail(c, TOPX_ERR_NUMERIC, m);
    return fail(c, TOPX_ERR_MODEL, m);
  } catch (const std::exception& e) {
    return fail(c, TOPX_ERR_INTERNAL, e.what());
  } catch (...) {
    return fail(c, TOPX_ERR_INTERNAL, "unknown error");
  }
}

void apply_params(topx::Settings& S, const topx_params& p) {
  S.modulus = p.modulus;
  S.poissonRatio = p.poissonRatio;
  S.modulusMin = p.modulusMin;
  S.SIMPpenalty = p.SIMPpenalty;
  S.cellSize = p.cellSize;
  S.tol = p.tol;
  S.maxIT = p.maxIT;
  S.weightFactorJacobi = p.weightFactorJacobi;
  S.coarsestResolutionControl = p.coarsestResolutionControl;
  S.typeVcycle = p.typeVcycle;
  for (int i = 0; i < 3; ++i) S.specifyPassiveRegions[i] = p.specifyPassiveRegions[i];
}

// The history rows carry at most TOPX_MAX_LOAD_CASES PCG counts: refuse larger models
// instead of dropping the counts of the further load cases.
void check_load_cases(const topx::Model& m) {
  if (m.loads.size() > size_t(TOPX_MAX_LOAD_CASES))
    throw std::runtime_error("the model has " + std::to_string(m.loads.size()) + " load cases; at most " +
                             std::to_string(TOPX_MAX_LOAD_CASES) + " are supported");
}

topx_status need_model(topx_ctx* c) {
  if (!c->model) return fail(c, TOPX_ERR_STATE, "no model loaded");
  return TOPX_OK;
}

// create the device engine on first use; no CPU fallback
topx_status need_engine(topx_ctx* c) {
  topx_status s = need_model(c);
  if (s != TOPX_OK) return s;
  if (c->engine) return TOPX_OK;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n <= c->params.device)
    return fail(c, TOPX_ERR_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(e));
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, c->params.device) != cudaSuccess)
    return fail(c, TOPX_ERR_CUDA, "cannot query CUDA device");
  if (prop.major != 10)
    return fail(c, TOPX_ERR_CUDA, "libtopx is built for sm_100a (B200); device is sm_" +
                                      std::to_string(prop.major) + std::to_string(prop.minor));
  c->engine.reset(new topx::Engine(*c->model, c->params.precision, c->params.device, c->params.coarse_coop != 0));
  return TOPX_OK;
}

void fill_iter(topx_iter* out, const topx::IterRecord& r) {
  std::memset(out, 0, sizeof(*out));
  out->loop = r.loop;
  out->c = r.c;
  out->vol = r.vol;
  out->sharp = r.sharp;
  out->cons = r.cons;
  out->change = r.change;
  for (size_t i = 0; i < r.its.size() && i < size_t(TOPX_MAX_LOAD_CASES); ++i) out->its[i] = r.its[i];
  out->filter_its = r.filter_its;
  out->t_assemble = r.t_assemble;
  out->t_cg = r.t_cg;
  out->t_opt = r.t_opt;
  out->t_filter = r.t_filter;
  out->t_total = r.t_total;
}

// Restores the caller's current device when the call returns or throws.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {
    TOPX_CUDA_OK(cudaGetDevice(&prev));
    if (prev != dev) TOPX_CUDA_OK(cudaSetDevice(dev));
  }
  ~DeviceScope() {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Accept only memory that kernels on `dev` can dereference at this address.
bool on_device(const void* p, int dev) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace

extern "C" {

const char* topx_version(void) { return "topx 0.1 (sm_100a)"; }

const char* topx_profile_section_name(int section) { return topx::Engine::section_name(section); }

topx_status topx_default_params(topx_params* p) {
  if (!p) return TOPX_ERR_ARG;
  topx::Settings S;
  p->modulus = S.modulus;
  p->poissonRatio = S.poissonRatio;
  p->modulusMin = S.modulusMin;
  p->SIMPpenalty = S.SIMPpenalty;
  p->cellSize = S.cellSize;
  p->tol = S.tol;
  p->maxIT = S.maxIT;
  p->weightFactorJacobi = S.weightFactorJacobi;
  p->coarsestResolutionControl = S.coarsestResolutionControl;
  p->precision = TOPX_FP64;
  p->device = 0;
  p->coarse_coop = 1;
  p->typeVcycle = TOPX_VCYCLE_ADAPTED;
  for (int i = 0; i < 3; ++i) p->specifyPassiveRegions[i] = 0;
  return TOPX_OK;
}

topx_status topx_create(topx_ctx** ctx, const topx_params* p) {
  if (!ctx) return TOPX_ERR_ARG;
  *ctx = nullptr;
  try {
    topx_ctx* c = new topx_ctx();
    if (p)
      c->params = *p;
    else
      topx_default_params(&c->params);
    const topx_params& q = c->params;
    const bool vc_ok = q.typeVcycle == TOPX_VCYCLE_ADAPTED ||
                       (q.typeVcycle == TOPX_VCYCLE_STANDARD && q.precision == TOPX_FP64);
    if ((q.precision != TOPX_FP64 && q.precision != TOPX_MIXED && q.precision != TOPX_MIXED_F32_FILTER) || !vc_ok) {
      delete c;
      return TOPX_ERR_ARG;
    }
    *ctx = c;
    return TOPX_OK;
  } catch (...) {
    return TOPX_ERR_INTERNAL;
  }
}

topx_status topx_destroy(topx_ctx* ctx) {
  if (!ctx) return TOPX_OK;
  try {
    ctx->engine.reset();
    ctx->model.reset();
  } catch (...) {
  }
  delete ctx;
  return TOPX_OK;
}

const char* topx_last_error(const topx_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

topx_status topx_load_voxels(topx_ctx* ctx, const uint8_t* vox, int nely, int nelx, int nelz) {
  return guarded(ctx, [&]() -> topx_status {
    if (!vox || nely <= 0 || nelx <= 0 || nelz <= 0) return fail(ctx, TOPX_ERR_ARG, "bad voxel array");
    if (nelx < 3 || nely < 3 || nelz < 3) return fail(ctx, TOPX_ERR_ARG, "Inappropriate Input Model!");
    ctx->engine.reset();
    ctx->begun = false;
    std::unique_ptr<topx::Model> m(new topx::Model());
    apply_params(m->S, ctx->params);
    m->load_cuboid(vox, nely, nelx, nelz);
    m->apply_boundary_condition();
    m->setup();
    m->set_passive_elements();
    check_load_cases(*m);
    ctx->model = std::move(m);
    ctx->vox.assign(vox, vox + size_t(nely) * nelx * nelz);
    ctx->vny = nely;
    ctx->vnx = nelx;
    ctx->vnz = nelz;
    ctx->topvoxel.clear();
    return TOPX_OK;
  });
}

topx_status topx_load_topvoxel(topx_ctx* ctx, const char* path) {
  return guarded(ctx, [&]() -> topx_status {
    if (!path) return fail(ctx, TOPX_ERR_ARG, "null path");
    ctx->engine.reset();
    ctx->begun = false;
    std::unique_ptr<topx::Model> m(new topx::Model());
    apply_params(m->S, ctx->params);
    m->load_topvoxel(path);
    m->apply_boundary_condition();
    m->setup();
    m->set_passive_elements();
    check_load_cases(*m);
    ctx->model = std::move(m);
    ctx->topvoxel = path;
    ctx->vox.clear();
    return TOPX_OK;
  });
}

topx_status topx_set_bc(topx_ctx* ctx, const double* fixing, int64_t nfix, const double* loads, int64_t nload) {
  return guarded(ctx, [&]() -> topx_status {
    topx_status s = need_model(ctx);
    if (s != TOPX_OK) return s;
    if (nfix < 0 || nload < 0 || (nfix > 0 && !fixing) || (nload > 0 && !loads))
      return fail(ctx, TOPX_ERR_ARG, "bad boundary-condition arrays");
    auto node_id = [&](double v) -> int64_t {
      if (!(v >= 1.0) || v != std::floor(v)) throw std::invalid_argument("boundary-condition node id out of range");
      return int64_t(v);
    };
    // as the .TopVoxel reader: unique node ids, the first row of a node kept
    std::map<int64_t, std::array<double, 3>> fix;
    for (int64_t i = 0; i < nfix; ++i) {
      const double* r = fixing + 4 * i;
      fix.emplace(node_id(r[0]), std::array<double, 3>{r[1], r[2], r[3]});
    }
    std::map<int, std::map<int64_t, std::array<double, 3>>> ld;
    for (int64_t i = 0; i < nload; ++i) {
      const double* r = loads + 5 * i;
      if (!(r[4] >= 1.0) || r[4] != std::floor(r[4]) || r[4] > 1e6) return fail(ctx, TOPX_ERR_ARG, "bad load case");
      ld[int(r[4])].emplace(node_id(r[0]), std::array<double, 3>{r[1], r[2], r[3]});
    }
    std::unique_ptr<topx::Model> m(new topx::Model());
    apply_params(m->S, ctx->params);
    if (!ctx->topvoxel.empty())
      m->load_topvoxel(ctx->topvoxel);
    else
      m->load_cuboid(ctx->vox.data(), ctx->vny, ctx->vnx, ctx->vnz);
    m->set_external_bc(fix, ld);
    m->apply_boundary_condition();
    m->setup();
    m->set_passive_elements();
    check_load_cases(*m);
    ctx->engine.reset();
    ctx->begun = false;
    ctx->model = std::move(m);
    return TOPX_OK;
  });
}

topx_status topx_get_info(const topx_ctx* cctx, topx_info* out) {
  topx_ctx* ctx = const_cast<topx_ctx*>(cctx);
  return guarded(ctx, [&]() -> topx_status {
    if (!out) return TOPX_ERR_ARG;
    if (need_model(ctx) != TOPX_OK) return TOPX_ERR_STATE;
    const topx::Model& M = *ctx->model;
    std::memset(out, 0, sizeof(*out));
    out->numLevels = M.numLevels;
    out->nelx = M.nelx;
    out->nely = M.nely;
    out->nelz = M.nelz;
    out->numElements = M.levels[0].numElements;
    out->numNodes = M.levels[0].numNodes;
    out->numDOFs = 3 * M.levels[0].numNodes;
    for (int l = 0; l < M.numLevels && l < 8; ++l) {
      out->resX[l] = M.levels[l].resX;
      out->resY[l] = M.levels[l].resY;
      out->resZ[l] = M.levels[l].resZ;
      out->levelElements[l] = M.levels[l].numElements;
      out->levelNodes[l] = M.levels[l].numNodes;
    }
    out->numLoadCases = int(M.loads.size());
    int64_t nf = 0;
    for (auto v : M.fixedDOFs) nf += v;
    out->numFixedDOFs = nf;
    out->numPassive = int64_t(M.passiveElements.size());
    return TOPX_OK;
  });
}

topx_status topx_get_ke(const topx_ctx* cctx, double* out576) {
  topx_ctx* ctx = const_cast<topx_ctx*>(cctx);
  return guarded(ctx, [&]() -> topx_status {
    if (!out576) return TOPX_ERR_ARG;
    if (need_model(ctx) != TOPX_OK) return TOPX_ERR_STATE;
    std::memcpy(out576, ctx->model->Ke.data(), sizeof(double) * 576);
    return TOPX_OK;
  });
}

topx_status topx_get_index_array(const topx_ctx* cctx, int level, int which, int32_t* out, size_t n,
                                 size_t* n_needed) {
  topx_ctx* ctx = const_cast<topx_ctx*>(cctx);
  return guarded(ctx, [&]() -> topx_status {
    if (need_model(ctx) != TOPX_OK) return TOPX_ERR_STATE;
    const topx::Model& M = *ctx->model;
    if (level < 1 || level > M.numLevels) return fail(ctx, TOPX_ERR_ARG, "bad level");
    const topx::Level& L = M.levels[level - 1];
    std::vector<int32_t> tmp;
    const std::vector<int32_t>* src = nullptr;
    switch (which) {
      case TOPX_ARR_ENODMAT: src = &L.eNodMat; break;
      case TOPX_ARR_ELEMAPBACK: src = &L.eleMapBack; break;
      case TOPX_ARR_NODMAPBACK: src = &L.nodMapBack; break;
      case TOPX_ARR_NODESONBOUNDARY: src = &L.nodesOnBoundary; break;
      case TOPX_ARR_ELEMENTSONBOUNDARY: src = &L.elementsOnBoundary; break;
      case TOPX_ARR_ELEMENTUPWARDMAP: src = &L.elementUpwardMap; break;
      case TOPX_ARR_TRANSFERMAT: src = &L.transferMat; break;
      case TOPX_ARR_SOLIDNODEMAP: src = &L.solidNodeMapCoarser2Finer; break;
      case TOPX_ARR_FIXEDDOFS:
        tmp.assign(M.fixedDOFs.begin(), M.fixedDOFs.end());
        src = &tmp;
        break;
      case TOPX_ARR_MAPUNIQUEKES: src = &M.mapUniqueKes; break;
      case TOPX_ARR_ISTHISELE2NDLEVEL: src = &M.isThisEle2ndLevel; break;
      case TOPX_ARR_PASSIVEELEMENTS: src = &M.passiveElements; break;
      default: return fail(ctx, TOPX_ERR_ARG, "bad array id");
    }
    if (n_needed) *n_needed = src->size();
    if (!out) return TOPX_OK;
    if (n < src->size()) return fail(ctx, TOPX_ERR_ARG, "output buffer too small");
    std::memcpy(out, src->data(), sizeof(int32_t) * src->size());
    return TOPX_OK;
  });
}

topx_status topx_get_transfer_coeffi(const topx_ctx* cctx, int level, double* out, size_t n, size_t* n_needed) {
  topx_ctx* ctx = const_cast<topx_ctx*>(cctx);
  return guarded(ctx, [&]() -> topx_status {
    if (need_model(ctx) != TOPX_OK) return TOPX_ERR_STATE;
    const topx::Model& M = *ctx->model;
    if (level < 2 || level > M.numLevels) return fail(ctx, TOPX_ERR_ARG, "bad level");
    const auto& v = M.levels[level - 1].transferMatCoeffi;
    if (n_needed) *n_needed = v.size();
    if (!out) return TOPX_OK;
    if (n < v.size()) return fail(ctx, TOPX_ERR_ARG, "output buffer too small");
    std::memcpy(out, v.data(), sizeof(double) * v.size());
    return TOPX_OK;
  });
}

topx_status topx_get_load(const topx_ctx* cctx, int lc, double* out, size_t n) {
  topx_ctx* ctx = const_cast<topx_ctx*>(cctx);
  return guarded(ctx, [&]() -> topx_status {
    if (need_model(ctx) != TOPX_OK) return TOPX_ERR_STATE;
    const topx::Model& M = *ctx->model;
    if (lc < 0 || lc >= int(M.loads.size())) return fail(ctx, TOPX_ERR_ARG, "bad load case");
    const size_t nd = size_t(M.levels[0].numNodes) * 3;
    if (!out || n < nd) return fail(ctx, TOPX_ERR_ARG, "output buffer too small");
    std::fill(out, out + nd, 0.0);
    for (size_t i = 0; i < M.loads[lc].node.size(); ++i)
      for (int c = 0; c < 3; ++c) out[size_t(M.loads[lc].node[i] - 1) * 3 + c] = M.loads[lc].f[i][c];
    return TOPX_OK;
  });
}

topx_status topx_set_moduli(topx_ctx* ctx, const double* E, size_t n) {
  return guarded(ctx, [&]() -> topx_status {
    topx_status s = need_engine(ctx);
    if (s != TOPX_OK) return s;
    if (!E || n != size_t(ctx->engine->Ne)) return fail(ctx, TOPX_ERR_ARG, "moduli size mismatch");
    ctx->engine->set_moduli_host(E);
    return TOPX_OK;
  });
}

topx_status topx_ku(topx_ctx* ctx, const double* u, double* y, size_t ndof) {
  return guarded(ctx, [&]() -> topx_status {
    topx_status s = need_engine(ctx);
    if (s != TOPX_OK) return s;
    if (!u || !y || ndof != size_t(ctx->engine->Nn) * 3) return fail(ctx, TOPX_ERR_ARG, "DOF size mismatch");
    ctx->engine->apply_K(u, y);
    return TOPX_OK;
  });
}

topx_status topx_ku_noalloc(topx_ctx* ctx, const double* u_dev, double* y_dev, size_t ndof) {
  return guarded(ctx, [&]() -> topx_status {
    if (!ctx->engine)
      return fail(ctx, TOPX_ERR_STATE,
                  "topx_ku_noalloc: the context has no device state yet; create it first with an allocating "
                  "call such as topx_set_moduli");
    topx::Engine& eng = *ctx->engine;
    if (!u_dev || !y_dev || ndof != size_t(eng.Nn) * 3) return fail(ctx, TOPX_ERR_ARG, "DOF size mismatch");
    const size_t grid = size_t(eng.G[0].stride) * 3;
    const size_t need = 2 * grid * sizeof(double);
    if (need > topx::noalloc_scratch_bytes())
      return fail(ctx, TOPX_ERR_ARG,
                  "topx_ku_noalloc: this model needs " + std::to_string(need) + " bytes of scratch (2 x 3 x " +
                      std::to_string(eng.G[0].stride) + " padded grid nodes x 8 B); the fixed scratch holds " +
                      std::to_string(topx::noalloc_scratch_bytes()) + " bytes; use topx_ku for this model");
    DeviceScope scope(ctx->params.device);
    if (!on_device(u_dev, ctx->params.device) || !on_device(y_dev, ctx->params.device))
      return fail(ctx, TOPX_ERR_ARG, "topx_ku_noalloc: u and y must be device (or managed) memory of the "
                                     "context's GPU");
    double* s = topx::noalloc_scratch(ctx->params.device);
    eng.apply_K_device(u_dev, y_dev, s, s + grid);
    return TOPX_OK;
  });
}

topx_status topx_selftest_wait(topx_ctx* ctx, int which) {
  return guarded(ctx, [&]() -> topx_status {
    topx_status s = need_engine(ctx);
    if (s != TOPX_OK) return s;
    DeviceScope scope(ctx->params.device);
    ctx->engine->selftest_wait(which);
    return TOPX_OK;
  });
}

topx_status topx_assemble(topx_ctx* ctx) {
  return guarded(ctx, [&]() -> topx_status {
    topx_status s = need_engine(ctx);
    if (s != TOPX_OK) return s;
    ctx->engine->assemble();
    TOPX_CUDA_OK(cudaStreamSynchronize(ctx->engine->st));
    return TOPX_OK;
  });
}

topx_status topx_vcycle(topx_ctx* ctx, const double* r, double* z, size_t ndof) {
  return guarded(ctx, [&]() -> topx_status {
    topx_status s = need_engine(ctx);
    if (s != TOPX_OK) return s;
    if (!r || !z || ndof != size_t(ctx->engine->Nn) * 3) return fail(ctx, TOPX_ERR_ARG, "DOF size mismatch");
    ctx->engine->apply_vcycle(r, z);
    return TOPX_OK;
  });
}

topx_status topx_get_diag(topx_ctx* ctx, int level, double* out, size_t n) {
  return guarded(ctx, [&]() -> topx_status {
    topx_status s = need_engine(ctx);
    if (s != TOPX_OK) return s;
    const topx::Model& M = *ctx->model;
    if (level < 1 || level >= M.numLevels) return fail(ctx, TOPX_ERR_ARG, "bad level");
    if (!out || n != size_t(M.levels[level - 1].numNodes) * 3) return fail(ctx, TOPX_ERR_ARG, "size mismatch");
    ctx->engine->get_diag(level, out);
    return TOPX_OK;
  });
}

topx_status topx_pcg(topx_ctx* ctx, int lc, double* u, size_t ndof, int* its) {
  return guarded(ctx, [&]() -> topx_status {
    topx_status s = need_engine(ctx);
    if (s != TOPX_OK) return s;
    if (lc < 0 || lc >= int(ctx->model->loads.size())) return fail(ctx, TOPX_ERR_ARG, "bad load case");
    if (!u || ndof != size_t(ctx->engine->Nn) * 3) return fail(ctx, TOPX_ERR_ARG, "DOF size mismatch");
    const int k = ctx->engine->pcg_host(lc, u);
    if (its) *its = k;
    return TOPX_OK;
  });
}

topx_status topx_filter(topx_ctx* ctx, double rmin, const double* src, double* out, size_t ne, int* its) {
  return guarded(ctx, [&]() -> topx_status {
    topx_status s = need_engine(ctx);
    if (s != TOPX_OK) return s;
    if (!src || !out || ne != size_t(ctx->engine->Ne)) return fail(ctx, TOPX_ERR_ARG, "element size mismatch");
    if (!(rmin > 0)) return fail(ctx, TOPX_ERR_ARG, "filter radius must be positive");
    const int k = ctx->engine->filter_host(rmin, src, out);
    if (its) *its = k;
    return TOPX_OK;
  });
}

topx_status topx_unit_compliance(topx_ctx* ctx, const double* U, double* ce, size_t ne) {
  return guarded(ctx, [&]() -> topx_status {
    topx_status s = need_engine(ctx);
    if (s != TOPX_OK) return s;
    if (!U || !ce || ne != size_t(ctx->engine->Ne)) return fail(ctx, TOPX_ERR_ARG, "element size mismatch");
    ctx->engine->compliance_host(U, ce);
    return TOPX_OK;
  });
}

topx_status topx_begin(topx_ctx* ctx, int consType, double V0, int nLoop, double rMin, double rHat, double* cSolid) {
  return guarded(ctx, [&]() -> topx_status {
    if (consType != TOPX_GLOBAL && consType != TOPX_LOCAL) return fail(ctx, TOPX_ERR_ARG, "Wrong Input!");
    if (!(V0 > 0 && V0 <= 1) || nLoop < 0 || !(rMin > 0) || (consType == TOPX_LOCAL && !(rHat > 0)))
      return fail(ctx, TOPX_ERR_ARG, "Wrong Input!");
    topx_status s = need_engine(ctx);
    if (s != TOPX_OK) return s;
    ctx->engine->begin(consType, V0, nLoop, rMin, rHat);
    ctx->begun = true;
    if (cSolid) *cSolid = ctx->engine->cSolid();
    return TOPX_OK;
  });
}

topx_status topx_step(topx_ctx* ctx, topx_iter* out) {
  return guarded(ctx, [&]() -> topx_status {
    if (!ctx->begun || !ctx->engine) return fail(ctx, TOPX_ERR_STATE, "topx_begin has not been called");
    topx::IterRecord r;
    if (!ctx->engine->step(r)) return TOPX_STOP;
    if (!std::isfinite(r.c)) return fail(ctx, TOPX_ERR_NUMERIC, "non-finite compliance");
    if (out) fill_iter(out, r);
    return TOPX_OK;
  });
}

topx_status topx_run(topx_ctx* ctx, int consType, double V0, int nLoop, double rMin, double rHat, topx_iter* hist,
                     int* loops, double* cSolid) {
  topx_status s = topx_begin(ctx, consType, V0, nLoop, rMin, rHat, cSolid);
  if (s != TOPX_OK) return s;
  int k = 0;
  for (;;) {
    topx_iter it;
    s = topx_step(ctx, &it);
    if (s == TOPX_STOP) break;
    if (s != TOPX_OK) return s;
    if (hist && k < nLoop) hist[k] = it;
    ++k;
  }
  if (loops) *loops = k;
  return TOPX_OK;
}

topx_status topx_get_density(topx_ctx* ctx, double* out, size_t ne) {
  return guarded(ctx, [&]() -> topx_status {
    if (!ctx->engine) return fail(ctx, TOPX_ERR_STATE, "no run");
    if (!out || ne != size_t(ctx->engine->Ne)) return fail(ctx, TOPX_ERR_ARG, "element size mismatch");
    ctx->engine->get_xphys(out);
    return TOPX_OK;
  });
}

topx_status topx_set_density(topx_ctx* ctx, const double* xPhys, size_t ne) {
  return guarded(ctx, [&]() -> topx_status {
    topx_status s = need_engine(ctx);
    if (s != TOPX_OK) return s;
    if (!xPhys || ne != size_t(ctx->engine->Ne)) return fail(ctx, TOPX_ERR_ARG, "element size mismatch");
    ctx->engine->set_xphys(xPhys);
    return TOPX_OK;
  });
}

topx_status topx_get_displacement(topx_ctx* ctx, int lc, double* out, size_t ndof) {
  return guarded(ctx, [&]() -> topx_status {
    if (!ctx->engine) return fail(ctx, TOPX_ERR_STATE, "no run");
    if (lc < 0 || lc >= int(ctx->model->loads.size())) return fail(ctx, TOPX_ERR_ARG, "bad load case");
    if (!out || ndof != size_t(ctx->engine->Nn) * 3) return fail(ctx, TOPX_ERR_ARG, "DOF size mismatch");
    ctx->engine->get_U(lc, out);
    return TOPX_OK;
  });
}

topx_status topx_timer_start(topx_ctx* ctx) {
  return guarded(ctx, [&]() -> topx_status {
    topx_status s = need_engine(ctx);
    if (s != TOPX_OK) return s;
    ctx->engine->timer_start();
    return TOPX_OK;
  });
}

topx_status topx_timer_stop(topx_ctx* ctx, double* ms) {
  return guarded(ctx, [&]() -> topx_status {
    if (!ctx->engine) return fail(ctx, TOPX_ERR_STATE, "timer not started");
    const double v = ctx->engine->timer_stop_ms();
    if (ms) *ms = v;
    return TOPX_OK;
  });
}

topx_status topx_set_profiling(topx_ctx* ctx, int on) {
  return guarded(ctx, [&]() -> topx_status {
    topx_status s = need_engine(ctx);
    if (s != TOPX_OK) return s;
    ctx->engine->set_profiling(on != 0);
    return TOPX_OK;
  });
}

topx_status topx_get_profile(topx_ctx* ctx, topx_profile* out) {
  return guarded(ctx, [&]() -> topx_status {
    if (!out) return TOPX_ERR_ARG;
    if (!ctx->engine) return fail(ctx, TOPX_ERR_STATE, "no engine");
    out->ku_ms = ctx->engine->prof_ku_ms;
    out->ku_launches = ctx->engine->prof_ku_launches;
    out->pcg_iterations = ctx->engine->prof_pcg_its;
    for (int i = 0; i < TOPX_PROFILE_SECTIONS && i < topx::Engine::SEC_COUNT; ++i) {
      out->section_ms[i] = ctx->engine->sec_ms[i];
      out->section_count[i] = ctx->engine->sec_n[i];
    }
    return TOPX_OK;
  });
}

int64_t topx_launch_count(void) { return topx::launch_counter().load(); }

}  // extern "C"
