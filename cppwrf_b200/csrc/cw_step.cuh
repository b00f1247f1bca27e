// SPDX-License-Identifier: GPL-3.0-or-later
// The RK3 step as a sequence of batched launches (CPPWRF's RK3::step, src/dyn/rk3.cpp:86-170): the launcher
// (deferred and merged halo fills, per-kernel profiling and block-shape selection) and the step's launch order.
//
// Included by the two translation units that instantiate the step's kernels, each for its own precision under
// its own floating-point options: cw_runtime.cu (FP64, no FMA contraction, IEEE division: bit-identical to the
// reference's CPU build) and cw_step_mixed.cu (FP32 fields). Everything here has internal linkage, so that each
// unit's launches refer to the kernels it compiled.
#pragma once

#include "cw_handle.cuh"

namespace {
using namespace cw;

struct Launcher {
  cw_handle* h;
  // plan: enqueue without launching, to make the batch's halo tables (device allocations) before a graph capture
  bool plan = false;
  long long count = 0;
  cudaEvent_t ev0 = nullptr;
  void begin(const char* name) {
    if (!h->profiling) return;
    cudaEvent_t a, b;
    CW_CUDA(cudaEventCreate(&a));
    CW_CUDA(cudaEventCreate(&b));
    CW_CUDA(cudaEventRecord(a, h->stream));
    h->prof_ev.push_back({name, {a, b}});
  }
  void check() {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw std::runtime_error(std::string("kernel launch: ") + cudaGetErrorString(e));
    if (h->profiling) CW_CUDA(cudaEventRecord(h->prof_ev.back().second.second, h->stream));
    ++count;
  }
  template <int NF>
  void halo_chunks(const std::vector<HaloChunk<NF>>& chunks) {
    if (plan) return;
    for (const HaloChunk<NF>& c : chunks) {
      const unsigned total = c.start[c.nf];
      if (total == 0) continue;
      const int bs = 256;
      const unsigned nb = (total + bs - 1) / bs;
      begin("k_halo");
      k_halo<NF><<<nb, bs, 0, h->stream>>>(c, 0);
      check();
      if (c.has_oddface) {
        begin("k_halo");
        k_halo<NF><<<nb, bs, 0, h->stream>>>(c, 1);
        check();
      }
    }
  }
  // halo fill points are deferred until the next kernel: consecutive fill points (nothing launched between
  // them) become one launch over the union of their fields
  std::vector<int> pend;
  void halo(int set) { pend.push_back(set); }
  // the union of the pending fill points' fields (each field once, first occurrence order)
  std::vector<HaloField> pending_fields() const {
    std::vector<HaloField> f;
    for (int set : pend)
      for (const HaloField& x : h->hs[set].f) {
        bool dup = false;
        for (const HaloField& y : f) dup |= y.p == x.p && y.ind == x.ind;
        if (!dup) f.push_back(x);
      }
    return f;
  }
  // a decomposed domain over ranks: the pending fill points' boxes between ranks (cross_plan): the packing boxes
  // into t.pk, the unpacking ones appended to x, the transfers into t
  void cross_ranks(HaloTable& t, std::vector<XchgBox>& x) {
    CrossPlan c = cross_plan(h, pend);
    const size_t esz = h->m.empty() ? 8 : size_t(h->m[0].esz);
    if (c.send_n > h->xsend_cap || c.recv_n > h->xrecv_cap) throw std::runtime_error("decomposition: exchange buffer too small");
    for (XchgBox& b : c.pk) b.dst = h->xbuf;
    for (XchgBox& b : c.unpk) {
      b.src = h->xbuf + h->xsend_cap * esz;
      x.push_back(b);
    }
    t.sends = std::move(c.sends);
    t.recvs = std::move(c.recvs);
    t.copies = std::move(c.copies);
    if (c.pk.empty()) return;
    std::vector<unsigned> st(c.pk.size() + 1);
    long long tot = 0;
    for (size_t n = 0; n < c.pk.size(); ++n) {
      st[n] = unsigned(tot);
      tot += c.pk[n].ncell;
    }
    if (tot >= (1ll << 31)) throw std::runtime_error("an exchange of more than 2^31 points");
    st[c.pk.size()] = unsigned(tot);
    t.npk = int(c.pk.size());
    t.pktotal = unsigned(tot);
    CW_CUDA(cudaMalloc(&t.pk, c.pk.size() * sizeof(XchgBox)));
    CW_CUDA(cudaMalloc(&t.pkstart, st.size() * sizeof(unsigned)));
    CW_CUDA(cudaMemcpy(t.pk, c.pk.data(), c.pk.size() * sizeof(XchgBox), cudaMemcpyHostToDevice));
    CW_CUDA(cudaMemcpy(t.pkstart, st.data(), st.size() * sizeof(unsigned), cudaMemcpyHostToDevice));
  }
  // the transfers of a fill point between ranks: NCCL point-to-point in one group on the handle's stream (captured
  // into the step's graph like the kernels), or device copies in the loopback form
  void transfer(const HaloTable& t) {
    const size_t esz = h->m.empty() ? 8 : size_t(h->m[0].esz);
    char* sbuf = h->xbuf;
    char* rbuf = h->xbuf + h->xsend_cap * esz;
    for (const XCopy& c : t.copies)
      if (c.n) CW_CUDA(cudaMemcpyAsync(rbuf + c.roff * esz, sbuf + c.soff * esz, c.n * esz, cudaMemcpyDeviceToDevice, h->stream));
    if (!t.sends.empty() || !t.recvs.empty()) nccl_exchange(h, t, sbuf, rbuf, esz);
  }
  // a batch: the pending fill points as one device table (made on first use, kept with the handle's tables)
  const HaloTable& halo_table() {
    auto it = h->halo_tabs.find(pend);
    if (it != h->halo_tabs.end()) return it->second;
    const std::vector<HaloField> f = pending_fields();
    std::vector<unsigned> st(f.size() + 1);
    long long total = 0;
    HaloTable t;
    for (size_t n = 0; n < f.size(); ++n) {
      st[n] = unsigned(total);
      total += f[n].ncell;
      t.has_oddface |= f[n].oddface_x;
    }
    if (total >= (1ll << 31)) throw std::runtime_error("a halo fill of more than 2^31 cells");
    st[f.size()] = unsigned(total);
    t.nf = int(f.size());
    t.total = unsigned(total);
    if (t.nf > 0) {
      CW_CUDA(cudaMalloc(&t.f, f.size() * sizeof(HaloField)));
      CW_CUDA(cudaMalloc(&t.start, st.size() * sizeof(unsigned)));
      CW_CUDA(cudaMemcpy(t.f, f.data(), f.size() * sizeof(HaloField), cudaMemcpyHostToDevice));
      CW_CUDA(cudaMemcpy(t.start, st.data(), st.size() * sizeof(unsigned), cudaMemcpyHostToDevice));
    }
    // a decomposed domain: the pending fill points' exchange boxes (each once)
    std::vector<XchgBox> x;
    for (int set : pend)
      for (const XchgBox& b : h->hs[set].x) {
        bool dup = false;
        for (const XchgBox& y : x)
          dup |= y.dst == b.dst && y.dst_ind == b.dst_ind && y.src == b.src && y.src_ind == b.src_ind && y.i0 == b.i0 &&
                 y.j0 == b.j0;
        if (!dup) x.push_back(b);
      }
    cross_ranks(t, x);
    if (!x.empty()) {
      std::vector<unsigned> xs(x.size() + 1);
      long long xt = 0;
      for (size_t n = 0; n < x.size(); ++n) {
        xs[n] = unsigned(xt);
        xt += x[n].ncell;
      }
      if (xt >= (1ll << 31)) throw std::runtime_error("an exchange of more than 2^31 points");
      xs[x.size()] = unsigned(xt);
      t.nx = int(x.size());
      t.xtotal = unsigned(xt);
      CW_CUDA(cudaMalloc(&t.x, x.size() * sizeof(XchgBox)));
      CW_CUDA(cudaMalloc(&t.xstart, xs.size() * sizeof(unsigned)));
      CW_CUDA(cudaMemcpy(t.x, x.data(), x.size() * sizeof(XchgBox), cudaMemcpyHostToDevice));
      CW_CUDA(cudaMemcpy(t.xstart, xs.data(), xs.size() * sizeof(unsigned), cudaMemcpyHostToDevice));
    }
    return h->halo_tabs.emplace(pend, t).first->second;
  }
  void flush() {
    if (pend.empty()) return;
    if (h->m.size() > 1 || h->decomp_px > 0) {
      const HaloTable& t = halo_table();
      if (t.pktotal > 0 && !plan) {  // a decomposed domain over ranks: the boxes other ranks receive, packed
        begin("k_exchange");
        k_exchange<<<(t.pktotal + 255u) / 256u, 256, 0, h->stream>>>(t.pk, t.pkstart, t.npk);
        check();
      }
      if (!plan) transfer(t);
      if (t.xtotal > 0 && !plan) {  // a decomposed domain: the exchange first, then the boundary fill
        begin("k_exchange");
        k_exchange<<<(t.xtotal + 255u) / 256u, 256, 0, h->stream>>>(t.x, t.xstart, t.nx);
        check();
      }
      if (t.total > 0 && !plan) {
        const unsigned nb = (t.total + 255u) / 256u;
        for (int pass = 0; pass < (t.has_oddface ? 2 : 1); ++pass) {
          begin("k_halo");
          k_halo_tab<<<nb, 256, 0, h->stream>>>(t.f, t.start, t.nf, pass);
          check();
        }
      }
      pend.clear();
      return;
    }
    if (pend.size() == 1) {
      halo_chunks(h->hs[pend[0]].small);
      halo_chunks(h->hs[pend[0]].large);
    } else {
      const std::vector<HaloField> f = pending_fields();
      if (f.size() <= size_t(kHaloSmall)) {
        std::vector<HaloChunk<kHaloSmall>> c;
        chunk_fields(f, c);
        halo_chunks(c);
      } else {
        std::vector<HaloChunk<kHaloLarge>> c;
        chunk_fields(f, c);
        halo_chunks(c);
      }
    }
    pend.clear();
  }
  void copy_list(CopyDesc* d, long long* sd, size_t n, long long total) {
    flush();
    if (!total || plan) return;
    const int bs = 256;
    begin("k_copy");
    k_copy<<<unsigned((total + bs - 1) / bs), bs, 0, h->stream>>>(d, int(n), sd);
    check();
  }
  // the block shape of a point kernel: the one being timed while tuning, else the tuned choice (0 by default)
  int shape_for(const char* name) const {
    if (h->tuning_shape >= 0) return h->tuning_shape;
    for (const auto& [n, sh] : h->shape_choice)
      if (n == name) return sh;
    return 0;
  }
  // a point kernel of fixed shape 0 over the index range kind, one launch per pack
  template <class R, int NM, class K, class... Args>
  void run(const char* name, int kind, K kern, const Packs<R, NM>& ps, Args... args) {
    flush();
    if (plan) return;
    for (size_t c = 0; c < ps.p.size(); ++c) {
      const int nb = ps.blocks[c][size_t(kind)][0];
      if (nb == 0) continue;
      begin(name);
      kern<<<nb, PX, 0, h->stream>>>(ps.p[c], args...);
      check();
    }
  }
  // a point kernel with a tunable block shape (one instantiation per shape), nq > 0: once per species
  template <class R, int NM, class K, class... Args>
  void run_t(const char* name, int kind, int nq, const std::array<K, kNumShapes>& kerns, const Packs<R, NM>& ps,
             Args... args) {
    flush();
    if (plan) return;
    const int sh = shape_for(name);
    for (size_t c = 0; c < ps.p.size(); ++c) {
      const int nb = ps.blocks[c][size_t(kind)][size_t(sh)];
      if (nb == 0 || nq == 0) continue;
      begin(name);
      kerns[size_t(sh)]<<<dim3(nb, nq), PX, 0, h->stream>>>(ps.p[c], args...);
      check();
    }
  }
  // the TMA-staged scalar update over RG_TILES: the shape is the chunk of levels a block takes (q_chunk), the planes
  // and face fluxes in dynamic shared memory
  template <class R, int NM, class K, class... Args>
  void run_q(const char* name, const std::array<K, kNumShapes>& kerns, const Packs<R, NM>& ps, Args... args) {
    flush();
    if (plan) return;
    const int sh = shape_for(name);
    const size_t smem = q_march_smem<R>(sh);
    CW_CUDA(cudaFuncSetAttribute(kerns[size_t(sh)], cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    for (size_t c = 0; c < ps.p.size(); ++c) {
      const int nb = ps.blocks[c][size_t(RG_TILES)][size_t(sh)];
      if (nb == 0) continue;
      begin(name);
      kerns[size_t(sh)]<<<nb, q_march_threads(sh), smem, h->stream>>>(ps.p[c], args...);
      check();
    }
  }
  // a column-block kernel using `arrays` shared level arrays
  template <class R, int NM, class K, class... Args>
  void run_cb(const char* name, int kind, int arrays, K kern, const Packs<R, NM>& ps, Args... args) {
    flush();
    if (plan) return;
    static_assert(CX == 32, "a column block's lanes are one warp");
    launch_cb(name, kind, arrays, kern, CNW, ps, args...);
  }
  // the same with a tunable warp count (one instantiation per shape: cb_warps(shape) warps per column block)
  template <class R, int NM, class K, class... Args>
  void run_cbt(const char* name, int kind, int arrays, const std::array<K, kNumShapes>& kerns, const Packs<R, NM>& ps,
               Args... args) {
    flush();
    if (plan) return;
    const int sh = shape_for(name);
    launch_cb(name, kind, arrays, kerns[size_t(sh)], cb_warps(sh), ps, args...);
  }
  template <class R, int NM, class K, class... Args>
  void launch_cb(const char* name, int kind, int arrays, K kern, int nw, const Packs<R, NM>& ps, Args... args) {
    const size_t smem = size_t(arrays) * h->cb_level_bytes;
    CW_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    for (size_t c = 0; c < ps.p.size(); ++c) {
      const int nb = ps.blocks[c][size_t(kind)][0];
      if (nb == 0) continue;
      begin(name);
      kern<<<nb, dim3(CX, nw), smem, h->stream>>>(ps.p[c], args...);
      check();
    }
  }
  // one block per member
  template <class R, int NM, class K>
  void run_members(const char* name, int threads, K kern, const Packs<R, NM>& ps) {
    flush();
    if (plan) return;
    for (size_t c = 0; c < ps.p.size(); ++c) {
      begin(name);
      kern<<<unsigned(ps.p[c].n), threads, 0, h->stream>>>(ps.p[c]);
      check();
    }
  }
};

// the three block-shape instantiations of a tunable point kernel
#define KV(kern) std::array{kern<R, NM, 0>, kern<R, NM, 1>, kern<R, NM, 2>}
#define KV_OP(kern, op) std::array{kern<R, NM, 0, op>, kern<R, NM, 1, op>, kern<R, NM, 2, op>}
// the same with the kernel's part (its fifth template argument)
#define KV_OP2(kern, op, x) std::array{kern<R, NM, 0, op, x>, kern<R, NM, 1, op, x>, kern<R, NM, 2, op, x>}
// the three warp-count instantiations of a tunable column kernel
#define KC(kern) std::array{kern<R, NM, cb_warps(0)>, kern<R, NM, cb_warps(1)>, kern<R, NM, cb_warps(2)>}

template <class R, int NM>
void enqueue_step(cw_handle* h, Launcher& L, const Packs<R, NM>& d) {
  const Member& M0 = h->m[0];
  bool lbc = false, terrain = false, scalars = false, any_pd = false, mp = false, open = false, dampkm = false,
       smag = false, any_plain = false;
  // every member specified on all four sides: the acoustic substeps read no halo cell of the fields the
  // per-substep fills (H_SS0, H_UV, H_AC) would refresh (the faces next to the boundary are the spec
  // zone's, updated from the boundary data), and the fills after the substeps (H_POST, H_FIN) refresh them
  // before anything reads them; those fills, and the spec zone's zero-gradient w of every substep but the
  // last (overwritten by the next one, read only after the substeps), are left out
  bool spec_all = h->decomp_px * h->decomp_py <= 1;  // a decomposed domain takes every fill: its patches read each other's points
  int nq = 0;  // the most species of a member
  for (const Member& M : h->m) {
    spec_all &= M.o.lbc != 0 && flat_x(M.g) && flat_y(M.g) && !two_d(M.g);
    nq = std::max(nq, M.o.n_scalars);
    lbc |= M.o.lbc != 0;
    open |= M.g.bc_x == CW_BC_OPEN || M.g.bc_y == CW_BC_OPEN;
    dampkm |= M.o.damp_opt == 1 && M.o.diff_opt == 1;
    smag |= M.o.km_opt == 4 && M.o.diff_opt == 1;
    mp |= M.o.mp_physics != 0;
    terrain |= !M.o.flat;
    scalars |= M.o.n_scalars > 0;
    for (int n = 0; n < M.o.n_scalars; ++n) {
      const bool pd = (n < M.o.n_moist ? M.o.moist_adv_opt : M.o.scalar_adv_opt) == 1;
      any_pd |= pd;
      any_plain |= !pd;
    }
  }
  const int n_sound = M0.n_sound;
  if (lbc) {
    L.run_members("k_advance_time", 1, k_advance_time<R, NM>, d);
  }
  if (h->cfl_on && !L.plan) CW_CUDA(cudaMemsetAsync(h->cfl_d, 0, 6 * h->m.size() * sizeof(unsigned long long), h->stream));
  L.copy_list(h->copies_d, h->copies_start_d, h->copies.size(), h->copies_total);
  L.halo(cw_handle::H_MU1);
  for (int rk = 1; rk <= 3; ++rk) {
    const int ns = rk == 1 ? 1 : (rk == 2 ? n_sound / 2 : n_sound);
    // rk_step_prep's fill (LargeStep::prep): at stages 2 and 3 the previous stage's H_FIN left these halos as this
    // fill would make them (only the scalars change in between), so only the first stage runs it (the fill merges
    // with the scalars' H_Q2 into one launch: fewer cells, not fewer launches)
    if (rk == 1) L.halo(cw_handle::H_PREP0);
    L.run_cbt("k_ls_prep", RG_COLS_STAG, 1, KC(k_ls_prep), d);
    L.halo(cw_handle::H_PREP1);
    if (rk == 1 && (dampkm || smag)) {  // DiffusionDriver::prepare: km_opt 4's and damp_opt 1's eddy viscosities
      if (smag) L.run_t("k_smag", RG_MASS, 1, KV(k_smag), d);
      if (dampkm) L.run_cb("k_dampkm", RG_COLS_MASS, 0, k_dampkm<R, NM>, d);
      L.halo(cw_handle::H_XK);
    }
    if (rk == 1) L.run_t("k_tendf_rk1", RG_STAG, 1, KV(k_tendf_rk1), d);
    if constexpr (sizeof(R) == 8) {  // FP64: the tendencies in two launches (-1.4 % per step); mixed: one (faster)
      if (open) {
        L.run_t("k_tend", RG_STAG, 1, KV_OP2(k_tend, true, 3), d, rk);
        L.run_t("k_tend_b", RG_STAG, 1, KV_OP2(k_tend, true, 12), d, rk);
      } else {
        L.run_t("k_tend", RG_STAG, 1, KV_OP2(k_tend, false, 3), d, rk);
        L.run_t("k_tend_b", RG_STAG, 1, KV_OP2(k_tend, false, 12), d, rk);
      }
    } else {
      if (open) L.run_t("k_tend", RG_STAG, 1, KV_OP(k_tend, true), d, rk);
      else L.run_t("k_tend", RG_STAG, 1, KV_OP(k_tend, false), d, rk);
    }
    if (h->cfl_on) L.run_t("k_cfl", RG_MASS, 1, KV(k_cfl), d, rk);
    if (rk == 1) L.copy_list(h->zeros_d, h->zeros_start_d, h->zeros.size(), h->zeros_total);
    L.run_cbt("k_ss_prep", RG_COLS_STAG, 3, KC(k_ss_prep), d, rk);
    if (!spec_all) L.halo(cw_handle::H_SS0);
    for (int it = 1; it <= ns; ++it) {
      L.run_t("k_uv", RG_STAG, 1, KV(k_uv), d, rk);
      if (!spec_all) L.halo(cw_handle::H_UV);
      L.run_cbt("k_ac", RG_COLS_STAG, kCbArrays, KC(k_ac), d, rk, it, ns);
      if (lbc && (!spec_all || it == ns)) L.run("k_ring", RG_RING, k_ring<R, NM>, d, int(RO_ZERO_GRAD_W), rk);
      if (!spec_all) L.halo(cw_handle::H_AC);
    }
    L.halo(cw_handle::H_POST);
    L.run_cbt("k_finish", RG_COLS_STAG, 0, KC(k_finish), d, rk, ns);
    L.halo(cw_handle::H_FIN);
    if (scalars) {
      if (rk == 1) L.run_t("k_q_tendf_rk1", RG_MASS, nq, KV(k_q_tendf_rk1), d);
      // at rk 3 the PD species take k_q_*_pd: the plain update runs only when some species is not PD
      if (rk != 3 || any_plain || !any_pd) {
        // the TMA-staged update where the tuner chose it; while tuning, the point kernel in the first round of
        // steps and the staged one in the second
        const bool march = h->q_tma && (h->tuning_shape >= 0 ? h->tune_steps_done / kNumShapes == 1 : h->q_march);
        if (march) L.run_q("k_q_march", KV(k_q_march), d, rk);
        else L.run_t("k_q_update", RG_MASS, 1, KV(k_q_update), d, rk);
      }
      if (rk == 3 && any_pd) {
        L.run_t("k_q_pre_pd", RG_MASS, nq, KV(k_q_pre_pd), d, rk);
        L.halo(cw_handle::H_Q1PD);
        L.run_t("k_q_face_pd", RG_FACES, 1, KV(k_q_face_pd), d, rk);
        L.run_t("k_q_scale_pd", RG_MASS, nq, KV(k_q_scale_pd), d, rk);
        L.halo(cw_handle::H_SCPD);
        L.run_t("k_q_update_pd", RG_MASS, nq, KV(k_q_update_pd), d, rk);
      }
      L.run_members("k_q_swap", 64, k_q_swap<R, NM>, d);
      if (lbc) L.run("k_ring", RG_RING, k_ring<R, NM>, d, int(RO_FLOW_DEP), rk);
      L.halo(cw_handle::H_Q2);
    }
  }
  if (mp) {  // the microphysics after the RK loop (PhysicsCoupling::step), then calc_p_rho_phi (rk3.cpp:146-158)
    L.run_cb("k_kessler", RG_COLS_MASS, kCbArrays, k_kessler<R, NM>, d);
    L.halo(cw_handle::H_MP);
    L.run_t("k_p_rho_phi", RG_MASS, 1, KV(k_p_rho_phi), d, 2);
    L.halo(cw_handle::H_MP_P);
  }
  if (lbc) {
    L.run("k_ring", RG_RING, k_ring<R, NM>, d, int(RO_FINAL), 3);
    L.run_t("k_p_rho_phi", RG_MASS, 1, KV(k_p_rho_phi), d, 1);
    L.halo(cw_handle::H_END_P);
  }
  if (terrain) {
    L.halo(cw_handle::H_WS0);
    L.run_cb("k_w_surface", RG_COLS_MASS, 0, k_w_surface<R, NM>, d);
    L.halo(cw_handle::H_WS1);
  }
  L.flush();
}

template <class R>
void enqueue_t(cw_handle* h, Launcher& L, const DevTables<R>& T) {
  if (h->m.size() == 1) enqueue_step<R, 1>(h, L, T.one);
  else enqueue_step<R, 0>(h, L, T.many);
}

}  // namespace
