// Device engine of the TOP3D_XL B200 path (see topx_engine.hpp).
#include "topx_engine.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <sstream>
#include <stdexcept>
#include <type_traits>

namespace topx {

static int64_t round_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

Engine::Engine(Model& model, int precision, int device, bool coarse_coop) : M(model), prec(precision) {
  TOPX_CUDA_OK(cudaSetDevice(device));
  // non-blocking streams: no implicit ordering with the legacy default stream, so engines on
  // other host threads (and their synchronous set-up copies) never stall or break this one's
  // graph captures; every host-side copy below waits for this stream first
  TOPX_CUDA_OK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  prepare_fem_kernels();
  prepare_nd_kernels();
  nl = M.numLevels;
  if (nl < 3 || int(M.levels.size()) != nl) throw std::runtime_error("model hierarchy not built");
  for (int l = 0; l < nl; ++l) {
    const Level& L = M.levels[l];
    Grid g;
    g.ny = L.resY;
    g.nx = L.resX;
    g.nz = L.resZ;
    g.stride = round_up(g.nnodes(), 32);
    G.push_back(g);
  }
  const Level& l1 = M.levels[0];
  Ne = l1.numElements;
  Nn = l1.numNodes;
  // ---- presence masks per level -------------------------------------------
  present.resize(nl);
  epresent.resize(nl);
  for (int l = 0; l < nl; ++l) {
    const Level& L = M.levels[l];
    std::vector<uint8_t> pn(size_t(G[l].nnodes()), 0), pe(size_t(G[l].nelems()), 0);
    for (auto k : L.nodMapBack) pn[k - 1] = 1;
    for (auto k : L.eleMapBack) pe[k - 1] = 1;
    present[l].upload(pn.data(), pn.size());
    epresent[l].upload(pe.data(), pe.size());
    if (l == 0) solid1.upload(pe.data(), pe.size());
  }
  std::vector<int32_t> emb(Ne), nmb(Nn);
  for (int64_t e = 0; e < Ne; ++e) emb[e] = l1.eleMapBack[e] - 1;
  for (int64_t k = 0; k < Nn; ++k) nmb[k] = l1.nodMapBack[k] - 1;
  eleMapBack0.upload(emb.data(), emb.size());
  nodMapBack0.upload(nmb.data(), nmb.size());
  // ---- boundary conditions: global form of the per-element BC matrices -------
  // (TOP3D_XL.m:1338-1437).  Check that the element matrices reduce to
  // y = m.*K(m.*u) + (1-m).*cfix.*u before relying on it.
  std::vector<uint8_t> fb(size_t(G[0].nnodes()), 0);
  std::vector<double> cf(size_t(G[0].nnodes()), 0.0);
  for (int64_t k = 0; k < Nn; ++k) {
    uint8_t b = 0;
    for (int c = 0; c < 3; ++c)
      if (M.fixedDOFs[size_t(k) * 3 + c]) b |= uint8_t(1u << c);
    fb[nmb[k]] = b;
  }
  std::vector<double> cacc(size_t(Nn) * 3, 0.0);
  for (int a = 0; a < 8; ++a)
    for (int64_t e = 0; e < Ne; ++e) {
      const int32_t sl = M.mapUniqueKes[e];
      const int32_t node = l1.eNodMat[size_t(e) * 8 + a];
      const uint8_t nb = fb[nmb[node - 1]];
      if (sl == 0) {
        if (nb) throw std::runtime_error("unsupported boundary conditions: element without BC matrix at a fixed DOF");
        continue;
      }
      for (int c = 0; c < 3; ++c) {
        const bool zm = (M.keFreeZeroMask[sl - 1] >> (3 * a + c)) & 1u;
        if (zm != bool((nb >> c) & 1))
          throw std::runtime_error("unsupported boundary conditions: element BC matrix differs from the fixed-DOF mask");
        if (zm) cacc[size_t(node - 1) * 3 + c] += M.keFixedDiag[sl - 1][3 * a + c];
      }
    }
  for (int64_t k = 0; k < Nn; ++k) {
    double v = 0.0;
    for (int c = 0; c < 3; ++c)
      if (M.fixedDOFs[size_t(k) * 3 + c]) {
        if (v != 0.0 && cacc[size_t(k) * 3 + c] != v)
          throw std::runtime_error("unsupported boundary conditions: per-component fixed diagonal differs");
        v = cacc[size_t(k) * 3 + c];
      }
    cf[nmb[k]] = v;
  }
  fixbits.upload(fb.data(), fb.size());
  // ---- load vectors -----------------------------------------------------------
  const int nL = int(M.loads.size());
  F.resize(nL);
  U.resize(nL);
  for (int lc = 0; lc < nL; ++lc) {
    std::vector<double> f(size_t(G[0].stride) * 3, 0.0);
    for (size_t i = 0; i < M.loads[lc].node.size(); ++i) {
      const int64_t n = nmb[M.loads[lc].node[i] - 1];
      for (int c = 0; c < 3; ++c) f[n + c * G[0].stride] = M.loads[lc].f[i][c];
    }
    F[lc].upload(f.data(), f.size());
    U[lc].alloc(f.size());
  }
  // ---- element matrices ---------------------------------------------------------
  upload_ke(M.Ke.data());
  {
    std::vector<double> T2 = galerkin_templates(M.Ke, M.levels[1].span);
    const std::vector<double> P4 = child_prolongators(M.levels[1].span);
    const int nc = M.levels[1].span * M.levels[1].span * M.levels[1].span;
    // BC-modified templates of level-2 children with fixed DOFs, de-duplicated by (slot, mask)
    std::map<std::pair<int, uint32_t>, int> modid;
    const Level& l2 = M.levels[1];
    std::vector<int32_t> fe, ts;
    std::vector<double> ff;
    auto tmpl = [&](const double* Pc, const double* K, double* out) {
      double KP[576];
      for (int i = 0; i < 24; ++i)
        for (int j = 0; j < 24; ++j) {
          double s = 0;
          for (int q = 0; q < 24; ++q) s += K[i * 24 + q] * Pc[q * 24 + j];
          KP[i * 24 + j] = s;
        }
      for (int i = 0; i < 24; ++i)
        for (int j = 0; j < 24; ++j) {
          double s = 0;
          for (int q = 0; q < 24; ++q) s += Pc[q * 24 + i] * KP[q * 24 + j];
          out[i * 24 + j] = s;
        }
    };
    for (int64_t j = 0; j < l2.numElements; ++j) {
      const int32_t idx = M.isThisEle2ndLevel[j];
      if (idx == 0) continue;
      fe.push_back(l2.eleMapBack[j] - 1);
      std::vector<int32_t> sel(nc);
      for (int c = 0; c < nc; ++c) sel[c] = c;
      std::vector<double> Fj(576, 0.0);
      for (int c : M.sonElesWithFixedDOFs[idx - 1]) {
        const int32_t e = l2.elementUpwardMap[size_t(j) * nc + c];
        const int32_t sl = M.mapUniqueKes[e - 1];
        const uint32_t mask = M.keFreeZeroMask[sl - 1];
        auto key = std::make_pair(c, mask);
        auto it = modid.find(key);
        if (it == modid.end()) {
          double Kf[576], Tm[576];
          for (int r = 0; r < 24; ++r)
            for (int q = 0; q < 24; ++q)
              Kf[r * 24 + q] = ((mask >> r) & 1u) || ((mask >> q) & 1u) ? 0.0 : M.Ke[r * 24 + q];
          tmpl(&P4[size_t(c) * 576], Kf, Tm);
          const int id = nc + int(modid.size());
          T2.insert(T2.end(), Tm, Tm + 576);
          it = modid.emplace(key, id).first;
        }
        sel[c] = it->second;
        double Kx[576] = {0}, Tx[576];
        for (int r = 0; r < 24; ++r) Kx[r * 25] = M.keFixedDiag[sl - 1][r];
        tmpl(&P4[size_t(c) * 576], Kx, Tx);
        for (int k = 0; k < 576; ++k) Fj[k] += Tx[k];
      }
      ts.insert(ts.end(), sel.begin(), sel.end());
      ff.insert(ff.end(), Fj.begin(), Fj.end());
    }
    nflag = int(fe.size());
    Tall.upload(T2.data(), T2.size());
    if (nflag) {
      fl_elem.upload(fe.data(), fe.size());
      fl_tsel.upload(ts.data(), ts.size());
      fl_F.upload(ff.data(), ff.size());
    }
    // span-2 child prolongators P_c = W_c (x) I_3: their node weights
    const std::vector<double> P2 = child_prolongators(2);
    std::vector<double> w8(8 * 64);
    for (int c = 0; c < 8; ++c)
      for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 8; ++b) w8[size_t(c) * 64 + 8 * a + b] = P2[size_t(c) * 576 + (3 * a) * 24 + 3 * b];
    W8.upload(w8.data(), w8.size());
  }
  Ks.resize(nl);
  for (int l = 1; l < nl; ++l) Ks[l].alloc(size_t(G[l].nelems()) * 576);
  // ---- level-1 K*u: the tiles that own a node of the domain (when voids leave some out) -----
  {
    std::vector<uint8_t> pn(size_t(G[0].nnodes()), 0);
    for (auto k : M.levels[0].nodMapBack) pn[k - 1] = 1;
    std::vector<uint32_t> zr;
    const std::vector<uint32_t> act = ku_active_tiles(G[0], pn, &zr);
    const std::vector<uint8_t> all(pn.size(), 1);
    const size_t full = ku_active_tiles(G[0], all).size();
    if (!act.empty() && act.size() < full * 9 / 10) {
      kuTiles.upload(act.data(), act.size());
      // an empty row list (no present node on the row y = ny) launches no last-row kernel
      const std::vector<uint32_t> rows = ku_active_row_tiles(G[0], pn);
      if (!rows.empty()) kuRows.upload(rows.data(), rows.size());
      kuZr.upload(zr.data(), zr.size());
      kut = KuTiles{kuTiles.p, int(act.size()), rows.empty() ? kuTiles.p : kuRows.p, int(rows.size()), kuZr.p};
    }
    const std::vector<uint32_t> fact = filter_active_tiles(G[0], pn);
    if (!fact.empty() && fact.size() < filter_active_tiles(G[0], all).size() * 9 / 10) {
      filterTiles.upload(fact.data(), fact.size());
      fut = KuTiles{filterTiles.p, int(fact.size())};
    }
    // elementwise level-1 passes skip the 32-node chunks without a present node
    const size_t nchunk = (pn.size() + 31) / 32;
    std::vector<uint32_t> mask((nchunk + 31) / 32, 0u);
    size_t nact = 0;
    for (size_t c = 0; c < nchunk; ++c) {
      bool any = false;
      for (size_t k = 32 * c; k < std::min(pn.size(), 32 * c + 32) && !any; ++k) any = pn[k] != 0;
      if (any) {
        mask[c / 32] |= 1u << (c % 32);
        ++nact;
      }
    }
    if (nact < nchunk * 9 / 10) {
      act1Mask.upload(mask.data(), mask.size());
      act1 = act1Mask.p;
    }
    // the level-1 restriction's y pass skips (x, z) columns without a present node
    const int64_t ncol = int64_t(G[0].nnx()) * G[0].nnz(), nny1 = G[0].nny();
    std::vector<uint32_t> cm(size_t((ncol + 31) / 32), 0u);
    int64_t ncact = 0;
    for (int64_t q = 0; q < ncol; ++q) {
      bool any = false;
      for (int64_t y = 0; y < nny1 && !any; ++y) any = pn[size_t(y + nny1 * q)] != 0;
      if (any) {
        cm[size_t(q / 32)] |= 1u << (q % 32);
        ++ncact;
      }
    }
    if (ncact < ncol * 9 / 10) {
      cols1Mask.upload(cm.data(), cm.size());
      cols1 = cols1Mask.p;
    }
  }
  // ---- coarsest level: nested-dissection plan and factor storage -----------------
  {
    const Grid& g = G[nl - 1];
    const Level& Lc = M.levels[nl - 1];
    std::vector<uint8_t> pc(size_t(g.nnodes()), 0);
    for (auto k : Lc.nodMapBack) pc[k - 1] = 1;
    int64_t npc = 0;
    for (uint8_t v : pc) npc += v;
    nd = nd_plan(g.nny(), g.nnx(), g.nnz(), g.stride, pc, nd_leaf_nodes(npc));
    ndFronts.upload(nd.fronts.data(), nd.fronts.size());
    ndTasks.upload(nd.tasks.data(), nd.tasks.size());
    ndAsm.upload(nd.asmb.data(), nd.asmb.size());
    ndPad.upload(nd.pad_diag.data(), nd.pad_diag.size());
    ndMap.upload(nd.upd_map.data(), nd.upd_map.size());
    ndSep.upload(nd.sep_dof.data(), nd.sep_dof.size());
    ndUpd.upload(nd.upd_dof.data(), nd.upd_dof.size());
    ndSrc0.upload(nd.src[0].data(), nd.src[0].size());
    ndSrc1.upload(nd.src[1].data(), nd.src[1].size());
    const size_t tile = size_t(ND_T) * ND_T;
    ndPool.alloc(size_t(nd.ntiles) * tile, false);
    ndScr.alloc(size_t(nd.nscr) * tile, false);
    ndW.alloc(size_t(nd.npos));
    ndPart.alloc(size_t(std::max<int64_t>(nd.nsolve_tasks, int64_t(nd.flow.size()))) * ND_T, false);
    ndCnt.alloc(size_t(nd.npos / ND_T));
    if (pre32()) ndPool32.alloc(size_t(nd.ntiles) * tile, false);
    ndd.fronts = ndFronts.p;
    ndd.tasks = ndTasks.p;
    ndd.asmb = ndAsm.p;
    ndd.pad = ndPad.p;
    ndd.upd_map = ndMap.p;
    ndd.sep_dof = ndSep.p;
    ndd.upd_dof = ndUpd.p;
    ndd.src0 = ndSrc0.p;
    ndd.src1 = ndSrc1.p;
    ndd.pool = ndPool.p;
    ndd.scr = ndScr.p;
    ndd.wvec = ndW.p;
    ndd.part = ndPart.p;
    ndd.cnt = ndCnt.p;
    coopCtl.alloc(1);
    // an engine alone on the GPU runs the solve as one persistent launch; engines sharing the
    // GPU (the job server) launch it level by level, since a persistent launch needs all its CTAs
    // resident at once
    coopCtas = coarse_coop ? nd_solve_coop_ctas() : 0;
    ndd.coop_ctas = coopCtas;
    ndd.ctl = coopCtl.p;
    if (coopCtas) {
      ndFlow.upload(nd.flow.data(), nd.flow.size());
      ndDone.alloc(2 * nd.fronts.size());
      ndd.flow = ndFlow.p;
      ndd.flow_done = ndDone.p;
    }
  }
  // ---- workspaces ------------------------------------------------------------
  {
    const size_t S1 = size_t(G[0].stride) * 3;
    for (DevBuf<double>* b : {&kw.r, &kw.z, &kw.p, &kw.q, &kw.p2}) b->alloc(S1);
    E64.alloc(size_t(G[0].nelems()));
    cfix64.upload(cf.data(), cf.size());
    if (!pre32()) {
      alloc_vwork(v64);
      if (M.S.typeVcycle == 1) {
        vq.resize(nl);
        for (int l = 1; l < nl - 1; ++l) vq[l].alloc(size_t(G[l].stride) * 3);
      }
    } else {
      if (M.S.typeVcycle == 1) throw std::invalid_argument("the 'Standard' V-cycle runs in FP64 precision");
      alloc_vwork(v32);
    }
    if (flt32())
      alloc_fwork(f32);
    else
      alloc_fwork(f64);
  }
  // ---- reductions and scalars ---------------------------------------------------
  red1.alloc(size_t(kMaxRedBlocks) * kMaxRedSlots);
  red2.alloc(size_t(kMaxRedBlocks) * kMaxRedSlots);
  tickets.alloc(8);
  rs1 = RedScratch{red1.p, tickets.p};
  rs2 = RedScratch{red2.p, tickets.p + 1};
  scE.alloc(1);
  scF.alloc(1);
  objS.alloc(1);
  ocS.alloc(1);
  mmaS.alloc(1);
  dscal.alloc(16);
  TOPX_CUDA_OK(cudaMallocHost(&h_sc, sizeof(PcgScalars)));
  TOPX_CUDA_OK(cudaMallocHost(&h_ctl, sizeof(CoopControl)));
  h_ctl->err = 0;
  // ---- optimiser state -------------------------------------------------------
  for (DevBuf<double>* b : {&x, &xPhys, &dc, &ce, &tmpA, &tmpB, &xTilde, &xhat, &dfdx, &dxv, &volMax})
    b->alloc(size_t(Ne));
  int64_t npas = 0;
  for (auto e : M.passiveElements) npas += (e >= 1 && e <= Ne) ? 1 : 0;
  nActive_ = Ne - npas;
  if (!M.passiveElements.empty()) {
    std::vector<uint8_t> pm(size_t(Ne), 0);
    for (auto e : M.passiveElements) pm[e - 1] = 1;
    passive.upload(pm.data(), pm.size());
  }
  for (int i = 0; i < 8; ++i) {
    cudaEvent_t e;
    TOPX_CUDA_OK(cudaEventCreate(&e));
    ev.push_back(e);
  }
  for (int i = 0; i < 2; ++i) TOPX_CUDA_OK(cudaEventCreate(&tev[i]));
  TOPX_CUDA_OK(cudaEventCreateWithFlags(&ev_legacy, cudaEventDisableTiming));
  for (int i = 0; i < 16; ++i) {
    cudaEvent_t e;
    TOPX_CUDA_OK(cudaEventCreate(&e));
    pev.push_back(e);
  }
  for (int i = 0; i < 4096; ++i) {
    cudaEvent_t e;
    TOPX_CUDA_OK(cudaEventCreate(&e));
    sev.push_back(e);
  }
  sec_of.assign(sev.size() / 2, 0);
  std::ostringstream os;
  os << "levels=" << nl;
  for (int l = 0; l < nl; ++l) os << " L" << (l + 1) << "=" << G[l].nx << "x" << G[l].ny << "x" << G[l].nz;
  os << " nd(fronts=" << nd.fronts.size() << ",levels=" << nd.levels.size() << ",maxn1=" << nd.max_n1
     << ",maxn2=" << nd.max_n2 << ",tilesMB=" << (double(nd.ntiles) * ND_T * ND_T * 8 / 1e6) << ") flagged=" << nflag;
  info_ = os.str();
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
}

Engine::~Engine() {
  // no work of this engine may still be in flight when its buffers and graphs go
  if (st) cudaStreamSynchronize(st);
  for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second.exec);
  for (auto e : ev) cudaEventDestroy(e);
  for (auto e : sev) cudaEventDestroy(e);
  for (auto e : pev) cudaEventDestroy(e);
  for (auto e : tev)
    if (e) cudaEventDestroy(e);
  if (ev_legacy) cudaEventDestroy(ev_legacy);
  if (h_sc) cudaFreeHost(h_sc);
  if (h_ctl) cudaFreeHost(h_ctl);
  if (st) cudaStreamDestroy(st);
}

template <typename TC>
void Engine::alloc_vwork(VWork<TC>& v) {
  v.d1.alloc(size_t(G[0].stride) * 3);
  v.rl.resize(nl);
  v.xl.resize(nl);
  v.dl.resize(nl);
  size_t tmax = 0;
  for (int l = 1; l < nl; ++l) {
    const size_t Sl = size_t(G[l].stride) * 3;
    v.rl[l].alloc(Sl);
    v.xl[l].alloc(Sl);
    if (l < nl - 1) v.dl[l].alloc(Sl);
    const Grid& gf = G[l - 1];
    const Grid& gc = G[l];
    tmax = std::max(tmax, size_t(gc.nny()) * gf.nnx() * gf.nnz());
  }
  v.tmp1.alloc(tmax * 3);
  v.tmp2.alloc(tmax * 3);
}

template <typename TF>
void Engine::alloc_fwork(FWork<TF>& f) {
  const size_t N1 = size_t(G[0].nnodes());
  for (DevBuf<TF>* b : {&f.fr, &f.fz, &f.fp, &f.fq, &f.fy, &f.fb}) b->alloc(N1);
  f.fsrc.alloc(size_t(G[0].nelems()));
  f.fdp[0].alloc(N1);
  f.fdp[1].alloc(N1);
}

void Engine::read_scalars(PcgScalars& h, const PcgScalars* d) const {
  TOPX_CUDA_OK(cudaMemcpyAsync(h_sc, d, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
  if (coopCtas) TOPX_CUDA_OK(cudaMemcpyAsync(h_ctl, coopCtl.p, sizeof(CoopControl), cudaMemcpyDeviceToHost, st));
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  h = *h_sc;
  check_device_waits();
}

void Engine::check_coop_waits() {
  if (coopCtas) TOPX_CUDA_OK(cudaMemcpyAsync(h_ctl, coopCtl.p, sizeof(CoopControl), cudaMemcpyDeviceToHost, st));
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  check_device_waits();
}

void Engine::copy_sync(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) const {
  TOPX_CUDA_OK(cudaMemcpyAsync(dst, src, bytes, kind, st));
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
}

// The persistent coarse solve's dependency waits set an error word instead of spinning on (they
// are bounded); the word was copied into pinned memory before the caller's stream sync.  A word
// that is set is cleared (so the engine stays usable) and reported.
void Engine::check_device_waits() const {
  if (coopCtas && h_ctl->err) {
    const int err = h_ctl->err;
    h_ctl->err = 0;
    // a launch that gave up may leave chunk tickets and dependency counts behind
    TOPX_CUDA_OK(cudaMemsetAsync(coopCtl.p, 0, sizeof(CoopControl), st));
    TOPX_CUDA_OK(cudaMemsetAsync(ndCnt.p, 0, sizeof(unsigned) * ndCnt.n, st));
    if (ndDone.p) TOPX_CUDA_OK(cudaMemsetAsync(ndDone.p, 0, sizeof(unsigned) * ndDone.n, st));
    TOPX_CUDA_OK(cudaStreamSynchronize(st));
    throw DeviceWaitError(err == kCoopErrWait ? "coarse solve: a dependency wait gave up (persistent launch not co-resident)"
                                              : "coarse solve: unknown wait error");
  }
}

// Drives the persistent coarse solve's bounded dependency wait to its poll limit: one CTA waits
// for a counter that nothing raises.  The wait gives up within about a second and the check below
// throws DeviceWaitError after clearing the words.
void Engine::selftest_wait(int which) {
  if (which != 0) throw std::invalid_argument("selftest_wait: which must be 0 (the coarse solve's dependency wait)");
  if (!coopCtas)
    throw std::invalid_argument("selftest_wait: this context runs the coarse solve without a persistent launch");
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  TOPX_CUDA_OK(cudaMemsetAsync(coopCtl.p, 0, sizeof(CoopControl), st));
  launch_coop_wait_selftest(st, coopCtl.p);
  check_coop_waits();
}

// ---------------------------------------------------------------------------
// design state
// ---------------------------------------------------------------------------
void Engine::set_xphys(const double* h) {
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  copy_sync(xPhys.p, h, sizeof(double) * Ne, cudaMemcpyHostToDevice);
}
void Engine::get_xphys(double* h) const {
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  copy_sync(h, xPhys.p, sizeof(double) * Ne, cudaMemcpyDeviceToHost);
}
void Engine::get_U(int lc, double* h) const {
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  DevBuf<double> tmp;
  tmp.alloc(size_t(Nn) * 3);
  launch_grid_to_compact_nodes<double>(st, U[lc].p, tmp.p, G[0], nodMapBack0.p, Nn);
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  copy_sync(h, tmp.p, sizeof(double) * Nn * 3, cudaMemcpyDeviceToHost);
}
void Engine::set_U(int lc, const double* h) {
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  DevBuf<double> tmp;
  tmp.upload(h, size_t(Nn) * 3);
  TOPX_CUDA_OK(cudaMemsetAsync(U[lc].p, 0, U[lc].bytes(), st));
  launch_compact_to_grid_nodes<double>(st, tmp.p, U[lc].p, G[0], nodMapBack0.p, Nn);
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
}

void Engine::update_moduli(const double* d_xPhys, bool solid) {
  if (solid)
    launch_fill_scatter(st, eleMapBack0.p, Ne, M.S.modulus, E64.p, nullptr);
  else
    launch_simp_scatter(st, d_xPhys, eleMapBack0.p, Ne, M.S.modulusMin, M.S.modulus, M.S.SIMPpenalty, E64.p,
                        nullptr);
}

// ---------------------------------------------------------------------------
// Solving_AssembleFEAstencil (TOP3D_XL.m:919-1066)
// ---------------------------------------------------------------------------
void Engine::assemble() {
  run_graph("assemble", [&]() { assemble_launches(); });
  sec_harvest();
}

void Engine::assemble_launches() {
  sec_begin(SEC_DIAG);
  if (!pre32())
    launch_diag_l1<double>(st, G[0], E64.p, fixbits.p, cfix64.p, present[0].p, v64.d1.p);
  else
    launch_diag_l1<double, float>(st, G[0], E64.p, fixbits.p, cfix64.p, present[0].p, v32.d1.p);
  sec_end();
  sec_begin(SEC_GALERKIN2);
  launch_galerkin_l2(st, G[1], E64.p, Tall.p, Ks[1].p);
  launch_galerkin_l2_flagged(st, G[1], E64.p, nflag, fl_elem.p, fl_tsel.p, fl_F.p, Tall.p, Ks[1].p);
  sec_end();
  sec_begin(SEC_GALERKIN3);
  for (int l = 2; l < nl; ++l) launch_galerkin_span2(st, G[l], Ks[l - 1].p, epresent[l].p, W8.p, Ks[l].p);
  sec_end();
  sec_begin(SEC_DIAG);
  for (int l = 1; l < nl - 1; ++l) {
    if (!pre32())
      launch_diag_coarse<double>(st, G[l], Ks[l].p, present[l].p, v64.dl[l].p);
    else
      launch_diag_coarse<float>(st, G[l], Ks[l].p, present[l].p, v32.dl[l].p);
  }
  sec_end();
  factor_coarsest();
}

void Engine::factor_coarsest() {
  sec_begin(SEC_INVERSE);
  ndd.factor(st, nd, G[nl - 1], Ks[nl - 1].p);
  if (pre32()) launch_convert<double, float>(st, ndPool.p, ndPool32.p, int64_t(ndPool.n));
  sec_end();
}

// ---------------------------------------------------------------------------
// 'Adapted' V-cycle (TOP3D_XL.m:747-781)
// ---------------------------------------------------------------------------
template <typename TC>
void Engine::vcycle_t(VWork<TC>& v, bool init, PcgScalars* sc) {
  sec_begin(SEC_RESTRICT);
  launch_restrict<double, TC>(st, M.levels[1].span, kw.r.p, G[0], v.tmp1.p, v.tmp2.p, v.rl[1].p, G[1], cols1);
  for (int l = 2; l < nl; ++l)
    launch_restrict<TC, TC>(st, M.levels[l].span, v.rl[l - 1].p, G[l - 1], v.tmp1.p, v.tmp2.p, v.rl[l].p, G[l]);
  sec_end();
  sec_begin(SEC_COARSE_SOLVE);
  {
    const TC* tiles = std::is_same<TC, double>::value ? (const TC*)ndPool.p : (const TC*)ndPool32.p;
    ndd.solve<TC, TC>(st, nd, tiles, v.rl[nl - 1].p, v.xl[nl - 1].p, sc);
  }
  sec_end();
  sec_begin(SEC_PROLONG);
  const double om = M.S.weightFactorJacobi;
  for (int l = nl - 2; l >= 1; --l)
    launch_prolong_smooth<TC, TC, TC>(st, M.levels[l + 1].span, v.xl[l + 1].p, G[l + 1], v.rl[l].p, v.dl[l].p,
                                      present[l].p, v.xl[l].p, G[l], om, false, false, sc, rs1);
  launch_prolong_smooth<TC, double, TC>(st, M.levels[1].span, v.xl[1].p, G[1], kw.r.p, v.d1.p, present[0].p,
                                        kw.z.p, G[0], om, true, init, sc, rs1, act1);
  sec_end();
}

// ---------------------------------------------------------------------------
// 'Standard' V-cycle (TOP3D_XL.m:747-781 with typeVcycle_ = 'Standard'), FP64: on each level
// but the coarsest x = omega*(r/d), the residual r - K x is restricted; after the coarse-grid
// correction x += omega*(r - K x)/d.  Level 1 uses the matrix-free K*u (x in z, K x in q, both
// free while the V-cycle runs); coarser levels the stored Galerkin matrices.
// ---------------------------------------------------------------------------
void Engine::vcycle_standard(bool init, PcgScalars* sc) {
  VWork<double>& v = v64;
  const double om = M.S.weightFactorJacobi;
  sec_begin(SEC_RESTRICT);
  launch_jacobi_pre<double, double, double>(st, G[0], kw.r.p, v.d1.p, present[0].p, kw.z.p, om, sc);
  launch_ku<double>(st, KU_PLAIN, G[0], kw.z.p, nullptr, nullptr, kw.q.p, E64.p, fixbits.p, cfix64.p, sc, rs1, kut);
  launch_residual_inplace<double, double>(st, G[0], kw.r.p, kw.q.p, sc);
  launch_restrict<double, double>(st, M.levels[1].span, kw.q.p, G[0], v.tmp1.p, v.tmp2.p, v.rl[1].p, G[1], cols1);
  for (int l = 1; l < nl - 1; ++l) {
    launch_jacobi_pre<double, double, double>(st, G[l], v.rl[l].p, v.dl[l].p, present[l].p, v.xl[l].p, om, sc);
    launch_ku_coarse(st, G[l], Ks[l].p, epresent[l].p, present[l].p, v.xl[l].p, vq[l].p, sc);
    launch_residual_inplace<double, double>(st, G[l], v.rl[l].p, vq[l].p, sc);
    launch_restrict<double, double>(st, M.levels[l + 1].span, vq[l].p, G[l], v.tmp1.p, v.tmp2.p, v.rl[l + 1].p,
                                    G[l + 1]);
  }
  sec_end();
  sec_begin(SEC_COARSE_SOLVE);
  ndd.solve<double, double>(st, nd, ndPool.p, v.rl[nl - 1].p, v.xl[nl - 1].p, sc);
  sec_end();
  sec_begin(SEC_PROLONG);
  for (int l = nl - 2; l >= 1; --l) {
    launch_prolong_add<double, double, double>(st, M.levels[l + 1].span, v.xl[l + 1].p, G[l + 1], v.rl[l].p,
                                               v.dl[l].p, present[l].p, v.xl[l].p, G[l], om, sc);
    launch_ku_coarse(st, G[l], Ks[l].p, epresent[l].p, present[l].p, v.xl[l].p, vq[l].p, sc);
    launch_jacobi_correct<double, double, double>(st, G[l], v.rl[l].p, vq[l].p, v.dl[l].p, present[l].p,
                                                  v.xl[l].p, om, false, false, sc, rs1);
  }
  launch_prolong_add<double, double, double>(st, M.levels[1].span, v.xl[1].p, G[1], kw.r.p, v.d1.p, present[0].p,
                                             kw.z.p, G[0], om, sc);
  launch_ku<double>(st, KU_PLAIN, G[0], kw.z.p, nullptr, nullptr, kw.q.p, E64.p, fixbits.p, cfix64.p, sc, rs1, kut);
  launch_jacobi_correct<double, double, double>(st, G[0], kw.r.p, kw.q.p, v.d1.p, present[0].p, kw.z.p, om, true,
                                                init, sc, rs1);
  sec_end();
}

void Engine::vcycle(bool init, PcgScalars* sc) {
  if (!pre32() && M.S.typeVcycle == 1)
    vcycle_standard(init, sc);
  else if (!pre32())
    vcycle_t<double>(v64, init, sc);
  else
    vcycle_t<float>(v32, init, sc);
}

// ---------------------------------------------------------------------------
// Solving_PCG (TOP3D_XL.m:600-639) on device-resident scalars
// ---------------------------------------------------------------------------
int Engine::pcg(const double* b, double* y, bool warm, double tol, int maxIT) {
  const Grid& g = G[0];
  PcgScalars* sc = scE.p;
  char key[96];
  std::snprintf(key, sizeof(key), "pcg_init:%p:%p:%d:%.17g:%d", (const void*)b, (const void*)y, int(warm), tol, maxIT);
  run_graph(key, [&]() {
    if (warm)
      launch_ku<double>(st, KU_PLAIN, g, y, nullptr, nullptr, kw.q.p, E64.p, fixbits.p, cfix64.p, sc, rs1, kut);
    else
      TOPX_CUDA_OK(cudaMemsetAsync(kw.q.p, 0, kw.q.bytes(), st));
    launch_residual_init<double>(st, g, b, kw.q.p, kw.r.p, sc, rs1, tol, maxIT);
    vcycle(true, sc);
  });
  const int CH = 8;
  PcgScalars h{};
  int launched = 0;
  std::snprintf(key, sizeof(key), "pcg_chunk:%p:%p", (const void*)b, (const void*)y);
  while (launched < maxIT) {
    const int first = launched;
    if (!prof_ && use_graphs && launched + CH <= maxIT) {
      run_graph(key, [&]() {
        for (int c = 0; c < CH; ++c) {  // CH is even: every chunk starts from p
          double* pin = (c & 1) ? kw.p2.p : kw.p.p;
          double* pnew = (c & 1) ? kw.p.p : kw.p2.p;
          launch_ku<double>(st, KU_P_UPDATE, g, pin, kw.z.p, pnew, kw.q.p, E64.p, fixbits.p, cfix64.p, sc, rs1, kut, y);
          launch_pcg_update<double, double>(st, g, y, nullptr, pnew, kw.r.p, kw.q.p, sc, rs1, act1);
          vcycle(false, sc);
        }
      });
      launched += CH;
      read_scalars(h, sc);
      if (h.done) break;
      continue;
    }
    for (int c = 0; c < CH && launched < maxIT; ++c, ++launched) {
      if (prof_) TOPX_CUDA_OK(cudaEventRecord(pev[2 * c], st));
      double* pin = (launched & 1) ? kw.p2.p : kw.p.p;
      double* pnew = (launched & 1) ? kw.p.p : kw.p2.p;
      launch_ku<double>(st, KU_P_UPDATE, g, pin, kw.z.p, pnew, kw.q.p, E64.p, fixbits.p, cfix64.p, sc, rs1, kut, y);
      if (prof_) TOPX_CUDA_OK(cudaEventRecord(pev[2 * c + 1], st));
      sec_begin(SEC_UPDATE);
      launch_pcg_update<double, double>(st, g, y, nullptr, pnew, kw.r.p, kw.q.p, sc, rs1, act1);
      sec_end();
      vcycle(false, sc);
    }
    read_scalars(h, sc);
    if (prof_) {
      // count the launches that ran an iteration (later ones return at once)
      for (int c = 0; first + c < launched && first + c < h.its; ++c) {
        float ms = 0.f;
        TOPX_CUDA_OK(cudaEventElapsedTime(&ms, pev[2 * c], pev[2 * c + 1]));
        prof_ku_ms += ms;
        prof_ku_launches += 1;
        sec_ms[SEC_KU] += ms;
        sec_n[SEC_KU] += 1;
      }
      sec_harvest();
    }
    if (h.done) break;
  }
  read_scalars(h, sc);
  // the last iteration's solution step (each K*u applied the one before it); iteration k wrote
  // its direction into p2 (k even) or p (k odd)
  if (h.its > 0) launch_pcg_flush(st, g, y, ((h.its - 1) & 1) ? kw.p.p : kw.p2.p, sc, act1);
  if (prof_) prof_pcg_its += h.its;
  return h.its;
}

int Engine::solve(int lc) { return pcg(F[lc].p, U[lc].p, true, M.S.tol, M.S.maxIT); }

void Engine::compliance(double* d_ce) {
  for (size_t lc = 0; lc < U.size(); ++lc)
    launch_unit_compliance(st, G[0], U[lc].p, eleMapBack0.p, Ne, M.objWeighting[lc], lc > 0, d_ce);
}

// ---------------------------------------------------------------------------
// PDE filter (TOP3D_XL.m:816-917)
// ---------------------------------------------------------------------------
void Engine::setup_filter(int slot, double rmin) {
  const std::array<double, 64> KF = pde_filter_kernel(rmin, M.S.cellSize * 1.0);
  filterKe64[slot] = filter_ke<double>(KF.data());
  filterKe32[slot] = filter_ke<float>(KF.data());
  filterR[slot] = rmin;
  if (!flt32())
    launch_filter_diag<double>(st, G[0], solid1.p, filterKe64[slot], f64.fdp[slot].p);
  else
    launch_filter_diag<float>(st, G[0], solid1.p, filterKe64[slot], f32.fdp[slot].p);
}

template <>
const FilterKe<double>& Engine::filter_ke_of<double>(int slot) const {
  return filterKe64[slot];
}
template <>
const FilterKe<float>& Engine::filter_ke_of<float>(int slot) const {
  return filterKe32[slot];
}

template <typename T>
int Engine::filter_t(FWork<T>& w, int slot, const double* d_src, double* d_out) {
  const Grid& g = G[0];
  PcgScalars* sc = scF.p;
  launch_scatter_elems_t<T>(st, d_src, eleMapBack0.p, Ne, w.fsrc.p);
  launch_filter_e2n<T>(st, g, w.fsrc.p, w.fb.p, act1);
  launch_filter_residual_init<T>(st, g, w.fb.p, w.fdp[slot].p, w.fr.p, w.fz.p, w.fy.p, sc, rs1, M.S.tol / 10,
                                 M.S.maxIT, act1);
  const int CH = 8;
  PcgScalars h{};
  int launched = 0;
  // the filter matrix is captured by value: the graph key carries the radius it was built for
  char key[64];
  std::snprintf(key, sizeof(key), "filter_chunk:%d:%.17g", slot, filterR[slot]);
  const FilterKe<T>& kf = filter_ke_of<T>(slot);
  while (launched < M.S.maxIT) {
    const int n = std::min(CH, M.S.maxIT - launched);
    auto body = [&]() {
      for (int c = 0; c < n; ++c) {
        launch_filter_ku<T>(st, KU_P_UPDATE, g, kf, w.fp.p, w.fz.p, nullptr, w.fq.p, solid1.p, sc, rs1, fut);
        launch_filter_update<T>(st, g, w.fy.p, w.fp.p, w.fr.p, w.fq.p, w.fdp[slot].p, w.fz.p, sc, rs1, act1);
      }
    };
    if (n == CH)
      run_graph(key, body);
    else
      body();
    launched += n;
    read_scalars(h, sc);
    if (h.done) break;
  }
  launch_filter_n2e<T>(st, g, w.fy.p, eleMapBack0.p, Ne, d_out);
  return h.its;
}

int Engine::filter(int slot, const double* d_src, double* d_out) {
  if (!flt32()) return filter_t<double>(f64, slot, d_src, d_out);
  return filter_t<float>(f32, slot, d_src, d_out);
}

// ---------------------------------------------------------------------------
// test entry points
// ---------------------------------------------------------------------------
void Engine::apply_K(const double* h_u, double* h_y) {
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  DevBuf<double> cu, du, dy;
  cu.upload(h_u, size_t(Nn) * 3);
  du.alloc(size_t(G[0].stride) * 3);
  dy.alloc(size_t(G[0].stride) * 3);
  launch_compact_to_grid_nodes<double>(st, cu.p, du.p, G[0], nodMapBack0.p, Nn);
  launch_ku<double>(st, KU_PLAIN, G[0], du.p, nullptr, nullptr, dy.p, E64.p, fixbits.p, cfix64.p, nullptr, rs1);
  launch_grid_to_compact_nodes<double>(st, dy.p, cu.p, G[0], nodMapBack0.p, Nn);
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  copy_sync(h_y, cu.p, sizeof(double) * Nn * 3, cudaMemcpyDeviceToHost);
}

void Engine::apply_vcycle(const double* h_r, double* h_z) {
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  DevBuf<double> cu;
  cu.upload(h_r, size_t(Nn) * 3);
  PcgScalars z{};
  z.done = 0;
  copy_sync(scE.p, &z, sizeof(z), cudaMemcpyHostToDevice);
  TOPX_CUDA_OK(cudaMemsetAsync(kw.r.p, 0, kw.r.bytes(), st));
  launch_compact_to_grid_nodes<double>(st, cu.p, kw.r.p, G[0], nodMapBack0.p, Nn);
  vcycle(true, scE.p);
  launch_grid_to_compact_nodes<double>(st, kw.z.p, cu.p, G[0], nodMapBack0.p, Nn);
  check_coop_waits();
  copy_sync(h_z, cu.p, sizeof(double) * Nn * 3, cudaMemcpyDeviceToHost);
}

void Engine::timer_start() { TOPX_CUDA_OK(cudaEventRecord(tev[0], st)); }
double Engine::timer_stop_ms() {
  TOPX_CUDA_OK(cudaEventRecord(tev[1], st));
  TOPX_CUDA_OK(cudaEventSynchronize(tev[1]));
  float ms = 0.f;
  TOPX_CUDA_OK(cudaEventElapsedTime(&ms, tev[0], tev[1]));
  return double(ms);
}
void Engine::set_profiling(bool on) {
  prof_ = on;
  prof_ku_ms = 0.0;
  prof_ku_launches = 0;
  prof_pcg_its = 0;
  sev_used = 0;
  for (int i = 0; i < SEC_COUNT; ++i) {
    sec_ms[i] = 0.0;
    sec_n[i] = 0;
  }
}

void Engine::run_graph(const std::string& key, const std::function<void()>& body) {
  if (prof_ || !use_graphs) {
    body();
    return;
  }
  auto it = graphs_.find(key);
  if (it == graphs_.end()) {
    cudaGraph_t g = nullptr;
    const long long before = launch_counter().load();
    TOPX_CUDA_OK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
      body();
    } catch (...) {
      cudaStreamEndCapture(st, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    TOPX_CUDA_OK(cudaStreamEndCapture(st, &g));
    const long long recorded = launch_counter().load() - before;
    launch_counter().fetch_sub(recorded);
    cudaGraphExec_t ex = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    TOPX_CUDA_OK(e);
    it = graphs_.emplace(key, GraphExec{ex, recorded}).first;
  }
  TOPX_CUDA_OK(cudaGraphLaunch(it->second.exec, st));
  launch_counter().fetch_add(it->second.kernels);
}

const char* Engine::section_name(int s) {
  static const char* names[SEC_COUNT] = {"ku",        "pcg_update", "restrict",       "coarse_solve", "prolong",
                                         "diag",      "galerkin_l2", "galerkin_span2", "slab_assemble", "schur",
                                         "spd_inverse", "filter",    "oc",             "compliance"};
  return (s >= 0 && s < SEC_COUNT) ? names[s] : "?";
}

void Engine::sec_begin(int sec) {
  if (!prof_) return;
  if (sev_used + 2 > int(sev.size())) sec_harvest();
  sec_of[sev_used / 2] = sec;
  TOPX_CUDA_OK(cudaEventRecord(sev[sev_used], st));
}

void Engine::sec_end() {
  if (!prof_) return;
  TOPX_CUDA_OK(cudaEventRecord(sev[sev_used + 1], st));
  sev_used += 2;
}

void Engine::sec_harvest() {
  if (!prof_ || sev_used == 0) return;
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  for (int i = 0; i < sev_used; i += 2) {
    float ms = 0.f;
    TOPX_CUDA_OK(cudaEventElapsedTime(&ms, sev[i], sev[i + 1]));
    sec_ms[sec_of[i / 2]] += ms;
    sec_n[sec_of[i / 2]] += 1;
  }
  sev_used = 0;
}

void Engine::set_moduli_host(const double* h_E) {
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  copy_sync(tmpA.p, h_E, sizeof(double) * Ne, cudaMemcpyHostToDevice);
  launch_scatter_elems_t<double>(st, tmpA.p, eleMapBack0.p, Ne, E64.p);
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
}

int Engine::pcg_host(int lc, double* h_u) {
  set_U(lc, h_u);
  const int its = solve(lc);
  get_U(lc, h_u);
  return its;
}

int Engine::filter_host(double rmin, const double* h_src, double* h_out) {
  setup_filter(0, rmin);
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  copy_sync(tmpA.p, h_src, sizeof(double) * Ne, cudaMemcpyHostToDevice);
  const int its = filter(0, tmpA.p, tmpB.p);
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  copy_sync(h_out, tmpB.p, sizeof(double) * Ne, cudaMemcpyDeviceToHost);
  return its;
}

void Engine::compliance_host(const double* h_U, double* h_ce) {
  for (size_t lc = 0; lc < U.size(); ++lc) set_U(int(lc), h_U + lc * size_t(Nn) * 3);
  compliance(ce.p);
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  copy_sync(h_ce, ce.p, sizeof(double) * Ne, cudaMemcpyDeviceToHost);
}

void Engine::get_diag(int level, double* h_d) const {
  // compact interleaved diagonal of `level` (1-based, < numLevels)
  const Level& L = M.levels[level - 1];
  const Grid& g = G[level - 1];
  std::vector<double> dense(size_t(g.stride) * 3);
  if (!pre32()) {
    const double* src = level == 1 ? v64.d1.p : v64.dl[level - 1].p;
    TOPX_CUDA_OK(cudaStreamSynchronize(st));
    copy_sync(dense.data(), src, sizeof(double) * dense.size(), cudaMemcpyDeviceToHost);
  } else {
    std::vector<float> f(dense.size());
    const float* src = level == 1 ? v32.d1.p : v32.dl[level - 1].p;
    TOPX_CUDA_OK(cudaStreamSynchronize(st));
    copy_sync(f.data(), src, sizeof(float) * f.size(), cudaMemcpyDeviceToHost);
    for (size_t i = 0; i < f.size(); ++i) dense[i] = f[i];
  }
  // the engine stores reciprocal diagonals
  for (int64_t k = 0; k < L.numNodes; ++k)
    for (int c = 0; c < 3; ++c) h_d[3 * k + c] = 1.0 / dense[(L.nodMapBack[k] - 1) + c * g.stride];
}

// ---------------------------------------------------------------------------
// optimisation loop
// ---------------------------------------------------------------------------
void Engine::begin(int consType, double V0, int nLoop, double rMin, double rHat) {
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  consType_ = consType;
  V0_ = V0;
  nLoop_ = nLoop;
  rMin_ = rMin;
  rHat_ = rHat;
  loop_ = 0;
  loopbeta_ = 0;
  change_ = 1.0;
  sharp_ = 1.0;
  betaPIO_ = 1.0;
  setup_filter(0, rMin);
  if (consType == 1) setup_filter(1, rHat);
  std::vector<double> h(size_t(Ne), V0);
  for (DevBuf<double>* b : {&x, &xPhys, &xTilde, &volMax}) copy_sync(b->p, h.data(), sizeof(double) * Ne, cudaMemcpyHostToDevice);
  for (auto& u : U) TOPX_CUDA_OK(cudaMemsetAsync(u.p, 0, u.bytes(), st));
  // compliance of the fully solid domain (TOP3D_XL.m:94-104)
  update_moduli(nullptr, true);
  assemble();
  for (size_t lc = 0; lc < U.size(); ++lc) solve(int(lc));
  compliance(ce.p);
  launch_sum(st, Ne, ce.p, nullptr, dscal.p, rs1);
  double s = 0;
  TOPX_CUDA_OK(cudaMemcpyAsync(&s, dscal.p, sizeof(double), cudaMemcpyDeviceToHost, st));
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  cSolid_ = M.S.modulus * s;
}

static double ev_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return double(ms) * 1e-3;
}

bool Engine::step(IterRecord& rec) {
  if (!(loop_ < nLoop_ && change_ > 0.0001 && sharp_ > 0.01)) return false;
  const auto t_host0 = std::chrono::steady_clock::now();
  ++loop_;
  rec = IterRecord{};
  rec.loop = loop_;
  const double Emin = M.S.modulusMin, E0 = M.S.modulus, pen = M.S.SIMPpenalty;
  TOPX_CUDA_OK(cudaEventRecord(ev[0], st));
  update_moduli(xPhys.p, false);
  assemble();
  TOPX_CUDA_OK(cudaEventRecord(ev[1], st));
  for (size_t lc = 0; lc < U.size(); ++lc) rec.its.push_back(solve(int(lc)));
  TOPX_CUDA_OK(cudaEventRecord(ev[2], st));
  sec_begin(SEC_COMPLIANCE);
  compliance(ce.p);
  launch_objective(st, Ne, ce.p, xPhys.p, cSolid_, Emin, E0, pen, dc.p, objS.p, rs1);
  sec_end();
  ObjState os{};
  TOPX_CUDA_OK(cudaMemcpyAsync(&os, objS.p, sizeof(os), cudaMemcpyDeviceToHost, st));
  TOPX_CUDA_OK(cudaEventRecord(ev[3], st));
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  rec.c = os.cObj * cSolid_;
  rec.vol = os.xsum / double(Ne);
  if (consType_ == 0) {
    // sensitivity filter ft = 1 (TOP3D_XL.m:135-137)
    sec_begin(SEC_FILTER);
    launch_ewise(st, EW_MUL, Ne, x.p, dc.p, tmpA.p, 0.0);
    rec.filter_its = filter(0, tmpA.p, tmpB.p);
    launch_ewise(st, EW_DIV_MAXX, Ne, tmpB.p, x.p, dc.p, 1e-3);
    sec_end();
    TOPX_CUDA_OK(cudaEventRecord(ev[4], st));
    // OC bisection (TOP3D_XL.m:145-156)
    OcState oc{};
    oc.l1 = 0.0;
    oc.l2 = 1e9;
    oc.fval = os.xsum / double(Ne) - V0_;
    TOPX_CUDA_OK(cudaMemcpyAsync(ocS.p, &oc, sizeof(oc), cudaMemcpyHostToDevice, st));
    sec_begin(SEC_OC);
    const uint8_t* pas = passive.p;
    launch_oc_prep(st, Ne, x.p, dc.p, tmpA.p);  // tmpA is free once the filter has run
    // at most 258 steps: 60 in the first round trip (the interval test usually passes after
    // 50-60 steps from (0, 1e9)), then 15 per round trip
    static_assert(60 % kOcStepsPerLaunch == 0 && 15 % kOcStepsPerLaunch == 0, "steps per round trip");
    for (int launched = 0; launched * kOcStepsPerLaunch < 256;) {
      const int n = (launched == 0 ? 60 : 15) / kOcStepsPerLaunch;
      for (int k = 0; k < n; ++k) launch_oc_bisect(st, Ne, x.p, tmpA.p, pas, ocS.p, rs1, 0.2);
      launched += n;
      TOPX_CUDA_OK(cudaMemcpyAsync(&oc, ocS.p, sizeof(oc), cudaMemcpyDeviceToHost, st));
      TOPX_CUDA_OK(cudaStreamSynchronize(st));
      if (oc.converged) break;
    }
    launch_oc_final(st, Ne, x.p, tmpA.p, pas, xPhys.p, ocS.p, rs1, rs2, 0.2);
    sec_end();
    TOPX_CUDA_OK(cudaMemcpyAsync(&oc, ocS.p, sizeof(oc), cudaMemcpyDeviceToHost, st));
    TOPX_CUDA_OK(cudaEventRecord(ev[5], st));
    TOPX_CUDA_OK(cudaStreamSynchronize(st));
    rec.cons = oc.fval;
    rec.change = oc.change;
    rec.sharp = 4 * oc.sharpsum / double(Ne);
    rec.t_assemble = ev_ms(ev[0], ev[1]);
    rec.t_cg = ev_ms(ev[1], ev[2]);
    rec.t_filter = ev_ms(ev[3], ev[4]);
    rec.t_opt = ev_ms(ev[2], ev[3]) + ev_ms(ev[4], ev[5]);
  } else {
    step_local(rec, os);
  }
  sec_harvest();
  change_ = rec.change;
  sharp_ = rec.sharp;
  rec.t_total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_host0).count();
  return true;
}

// ---------------------------------------------------------------------------
// LOCAL: porous infill with local-volume p-norm constraint and MMA
// (TOP3D_XL.m:311-401)
// ---------------------------------------------------------------------------
void Engine::step_local(IterRecord& rec, const ObjState& os) {
  (void)os;
  const double etaPIO = 0.5;
  const int pPIO = 16;
  const double pMaxPIO = 128;
  ++loopbeta_;
  if (!xold1.p) {
    for (DevBuf<double>* b : {&xold1, &xold2, &low, &upp, &alpha, &beta, &p0, &q0, &pij, &qij, &xmma})
      b->alloc(size_t(Ne));
  }
  TOPX_CUDA_OK(cudaEventRecord(ev[3], st));
  // local volume fraction and its sensitivity (TOP3D_XL.m:333-335)
  int fits = filter(1, xPhys.p, xhat.p);
  launch_pnorm_terms(st, Ne, xhat.p, V0_, pPIO, dscal.p, rs1);
  double pnsum = 0;
  TOPX_CUDA_OK(cudaMemcpyAsync(&pnsum, dscal.p, sizeof(double), cudaMemcpyDeviceToHost, st));
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  const double pn = pnsum / double(Ne);
  launch_local_sens(st, Ne, xhat.p, xTilde.p, dc.p, V0_, pPIO, pn, betaPIO_, etaPIO, dfdx.p, dxv.p, tmpA.p);
  // filtered sensitivities (TOP3D_XL.m:338-350)
  fits += filter(0, tmpA.p, dc.p);
  fits += filter(1, dfdx.p, tmpB.p);
  launch_ewise(st, EW_MUL, Ne, tmpB.p, dxv.p, tmpA.p, 0.0);
  fits += filter(0, tmpA.p, dfdx.p);
  TOPX_CUDA_OK(cudaEventRecord(ev[4], st));
  // MMA update (TOP3D_XL.m:352-369)
  const double fval = std::pow(pnsum / double(Ne), 1.0 / pPIO) - 1;
  if (loop_ == 1) {
    TOPX_CUDA_OK(cudaMemcpyAsync(xold1.p, x.p, sizeof(double) * Ne, cudaMemcpyDeviceToDevice, st));
    TOPX_CUDA_OK(cudaMemcpyAsync(xold2.p, x.p, sizeof(double) * Ne, cudaMemcpyDeviceToDevice, st));
    TOPX_CUDA_OK(cudaMemsetAsync(low.p, 0, low.bytes(), st));
    TOPX_CUDA_OK(cudaMemsetAsync(upp.p, 0, upp.bytes(), st));
  }
  const uint8_t* pas = passive.p;
  launch_mma_gensub(st, Ne, loop_, 0.1, x.p, pas, xold1.p, xold2.p, low.p, upp.p, dc.p, dfdx.p, fval, nActive_,
                    alpha.p, beta.p, p0.p, q0.p, pij.p, qij.p, mmaS.p, rs1);
  MmaState ms{};
  for (int chunk = 0; chunk < 64; ++chunk) {
    for (int k = 0; k < 16; ++k) {
      launch_mma_newton(st, Ne, pas, low.p, upp.p, alpha.p, beta.p, p0.p, q0.p, pij.p, qij.p, mmaS.p, rs1);
      launch_mma_residual(st, Ne, pas, low.p, upp.p, alpha.p, beta.p, p0.p, q0.p, pij.p, qij.p, xmma.p, mmaS.p, rs1);
    }
    TOPX_CUDA_OK(cudaMemcpyAsync(&ms, mmaS.p, sizeof(ms), cudaMemcpyDeviceToHost, st));
    TOPX_CUDA_OK(cudaStreamSynchronize(st));
    if (ms.finished) break;
  }
  if (!ms.finished) throw std::runtime_error("MMA dual solve did not finish");
  launch_mma_finish(st, Ne, pas, xmma.p, xold1.p, x.p, mmaS.p, rs2);
  TOPX_CUDA_OK(cudaEventRecord(ev[5], st));
  // density filter + Heaviside projection with beta continuation (TOP3D_XL.m:372-382)
  fits += filter(0, x.p, xTilde.p);
  if (loopbeta_ >= 40) {
    betaPIO_ = std::min(2 * betaPIO_, pMaxPIO);
    loopbeta_ = 0;
  }
  launch_heaviside(st, Ne, xTilde.p, pas, betaPIO_, etaPIO, xPhys.p, dscal.p + 1, rs1);
  double sh = 0;
  TOPX_CUDA_OK(cudaMemcpyAsync(&sh, dscal.p + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
  TOPX_CUDA_OK(cudaMemcpyAsync(&ms, mmaS.p, sizeof(ms), cudaMemcpyDeviceToHost, st));
  TOPX_CUDA_OK(cudaEventRecord(ev[6], st));
  TOPX_CUDA_OK(cudaStreamSynchronize(st));
  rec.filter_its = fits;
  rec.cons = fval;
  rec.change = ms.change;
  rec.sharp = 4 * sh / double(Ne);
  rec.t_assemble = ev_ms(ev[0], ev[1]);
  rec.t_cg = ev_ms(ev[1], ev[2]);
  rec.t_opt = ev_ms(ev[2], ev[3]) + ev_ms(ev[4], ev[5]);
  rec.t_filter = ev_ms(ev[3], ev[4]) + ev_ms(ev[5], ev[6]);
}

template void Engine::alloc_vwork<double>(VWork<double>&);
template void Engine::alloc_vwork<float>(VWork<float>&);
template void Engine::alloc_fwork<double>(FWork<double>&);
template void Engine::alloc_fwork<float>(FWork<float>&);

}  // namespace topx
